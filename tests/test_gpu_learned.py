"""Learned per-shape SDF (3-64-64-1 SiLU network per template) on the GPU.

* The training kernel's loss and gradient against the FP64 CPU oracle
  (oracle/mlp_oracle.py) on the same parameters and points.
* Training on a periodic polydisperse scene lowers the loss, and each network's stated
  error bound (measured by the narrowphase's own tensor-core inference code over all
  grid nodes and further points) holds at every grid node.
* The tcgen05 inference agrees with the FP64 forward pass of the same weights to BF16
  rounding.
* With the network in front of the grid screen, the precision form still gives the FP64
  form's contact lists at every step and its forces to summation order.
* Ablation: from the same state, the network (sent only the nodes whose sub-cluster
  estimate lies above its rejection threshold) saves grid lookups, at most one per
  evaluation, the FP64 queue does not grow and the contacts stay the same.
"""
import sys

import numpy as np
import pytest

from conftest import ROOT
from helpers import canon

sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def test_training_gradient_matches_cpu_oracle(lsdem):
    rng = np.random.default_rng(11)
    p = mo.random_params(rng).astype(np.float32)
    pts = np.concatenate([rng.uniform(-1, 1, (256, 3)), rng.normal(0, 0.3, (256, 1))], 1).astype(np.float32)
    loss_g, grad_g, y_g = lsdem.mlp_gradient(p, pts)
    loss_o, grad_o, y_o = mo.loss_and_grad(p.astype(np.float64), pts.astype(np.float64))
    assert np.abs(y_g - y_o).max() <= 1e-4 * np.abs(y_o).max()
    assert abs(loss_g - loss_o) <= 1e-4 * loss_o
    for name, lo, hi in (("W1", mo.W1, mo.B1), ("b1", mo.B1, mo.W2), ("W2", mo.W2, mo.B2), ("b2", mo.B2, mo.W3),
                         ("w3", mo.W3, mo.B3), ("b3", mo.B3, mo.B3 + 1)):
        err = np.abs(grad_g[lo:hi] - grad_o[lo:hi]).max() / max(np.abs(grad_o[lo:hi]).max(), 1e-30)
        assert err <= 1e-3, (name, err)


def _scene(lsdem, n=1500, seed=41):
    from lsdem_b200 import scenes
    T = scenes.unit_templates(n_grid=32, n_nodes=800)
    box = 0.1 * (n / 1e5) ** (1.0 / 3.0)
    sc = scenes.polydisperse_periodic(lsdem, n=n, box=box, seed=seed, templates=T, n_grid=32, n_nodes=800)
    scenes.resolve_deep_overlaps(lsdem, sc)
    sc["dt"] = 2e-7
    return sc


def _solver(lsdem, sc, prec):
    from lsdem_b200 import scenes
    sv = lsdem.Solver()
    scenes.load_polydisperse(sv, sc)
    sv.set_precision(prec)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    return sv


@pytest.fixture(scope="module")
def trained(lsdem):
    sc = _scene(lsdem)
    sv = _solver(lsdem, sc, 2)
    loss, err = sv.train_learned_sdf(iterations=4000, batch=4096, samples=1 << 17)
    yield sc, sv, loss, err
    sv.close()


def test_training_converges_and_error_bound_holds(lsdem, trained):
    sc, sv, loss, err = trained
    for k in range(len(loss)):
        print(f"shape {k}: loss {loss[k]:.2e}", {a: round(b, 5) for a, b in sv.learned_sdf(k)[1].items()
                                                 if a != "centre"})
    rng = np.random.default_rng(0)
    for k, t in enumerate(sc["templates"]):
        params, info = sv.learned_sdf(k)
        assert info["err"] == pytest.approx(err[k])
        # mean squared error of phi / R (an untrained network starts near 1e-1)
        assert loss[k] < 5e-3, loss
        assert 0.0 <= info["err_in"] <= info["err"] and 0.0 < info["threshold_h"] < 40.0, info
        # the stated bound holds at every grid node (they are part of the validation set)
        size, o, h = np.asarray(t["size"]), np.asarray(t["origin"]), float(t["spacing"])
        ii = np.stack(np.meshgrid(*[np.arange(m) for m in size], indexing="ij"), -1).reshape(-1, 3)
        lin = ii[:, 0] + size[0] * (ii[:, 1] + size[1] * ii[:, 2])
        pts = o + ii * h
        sel = rng.choice(len(pts), 20000, replace=False)
        phi = sv.mlp_eval(k, pts[sel])
        # against the training target: phi clipped to [-0.25 R, 0.5 R]
        true = np.clip(np.asarray(t["sdf"])[lin[sel]], -0.25 * info["R"], 0.5 * info["R"])
        assert np.abs(phi - true).max() <= info["err"] * (1 + 1e-6) + 1e-12


def test_tensor_core_inference_matches_fp64_forward(lsdem, trained):
    """The tcgen05 inference (BF16 A and B operands in shared memory, FP32 accumulators
    in tensor memory) against the FP64 forward pass of the same FP32 master weights
    (oracle/mlp_oracle.py) at 4096 points of each shape's input cube: BF16 rounding of
    weights and activations bounds the difference (2 % of the output scale, mean 0.3 %).
    A wrong operand layout or descriptor would give unrelated values."""
    sc, sv, _, _ = trained
    rng = np.random.default_rng(5)
    u = rng.uniform(-1.0, 1.0, (4096, 3))
    for k in range(len(sc["templates"])):
        params, info = sv.learned_sdf(k)
        y_o = mo.forward(params.astype(np.float64), u)
        y_g = sv.mlp_eval(k, info["centre"] + info["R"] * u) / info["R"]
        scale = max(1.0, float(np.abs(y_o).max()))
        diff = np.abs(y_g - y_o)
        assert diff.max() <= 2e-2 * scale and diff.mean() <= 3e-3 * scale, (k, diff.max(), diff.mean())


def _run(lsdem, sc, prec, learned, steps, trained_sv=None):
    sv = _solver(lsdem, sc, prec)
    if learned:
        sv.train_learned_sdf(iterations=4000, batch=4096, samples=1 << 17)
        sv.set_learned_sdf(True)
    out = []
    for _ in range(steps):
        box = {}
        sv.step(sc["dt"], 1, hook=lambda t: box.update(sv.state()))
        out.append((box, {"pp": sv.contacts(lsdem.CONTACT_PARTICLE), "g": sv.contacts(lsdem.CONTACT_GHOST)}))
    sv.close()
    return out


def test_learned_form_equals_fp64_form(lsdem):
    sc = _scene(lsdem)
    ref = _run(lsdem, sc, 0, False, 3)
    got = _run(lsdem, sc, 2, True, 3)
    n_contacts = 0
    for (b0, c0), (b1, c1) in zip(ref, got):
        for k in ("pp", "g"):
            keys = ("node", "partner") if k == "pp" else ("node", "partner", "image")
            o0, o1 = canon(c0[k], keys), canon(c1[k], keys)
            assert len(o0) == len(o1), (k, len(o0), len(o1))
            for key in keys:
                assert np.array_equal(np.asarray(c0[k][key])[o0], np.asarray(c1[k][key])[o1]), (k, key)
            n_contacts += len(o0)
        for q in ("force", "torque"):
            err = np.abs(b1[q] - b0[q]).max() / np.abs(b0[q]).max()
            assert err <= 1e-10, (q, err)
    assert n_contacts > 200


def test_learned_sdf_ablation(lsdem, trained):
    sc, sv, _, _ = trained
    st = sv.state()
    res = {}
    for learned in (False, True):
        sv.set_state(pos=st["pos"], vel=st["vel"], angvel=st["angvel"], quat=st["quat"])
        sv.set_learned_sdf(learned)
        sv.set_screen_stats(True)
        sv.step(sc["dt"], 1)
        res[learned] = (sv.screen_stats(), sv.contacts(lsdem.CONTACT_PARTICLE))
        sv.set_screen_stats(False)
    (s0, c0), (s1, c1) = res[False], res[True]
    print("without network:", s0)
    print("with network:   ", s1)
    assert s1["net_evals"] > 0 and s0["net_evals"] == 0
    # the network may also reject nodes the grid screen had to queue (near its grid
    # boundary): the FP64 queue can only shrink, the contacts stay the same
    assert s1["nodes_queued"] <= s0["nodes_queued"]
    # the network only sees nodes it may reject (the others take the grid test in the
    # screen); every node it rejects saves a grid lookup
    rejected = s0["grid_lookups"] - s1["grid_lookups"]
    print(f"network: {s1['net_evals']:.0f} evaluations, {rejected:.0f} grid lookups saved "
          f"({rejected / max(s1['net_evals'], 1):.1%} of its evaluations)")
    assert 0 < rejected <= s1["net_evals"], (s0["grid_lookups"], s1["grid_lookups"], s1["net_evals"])
    o0, o1 = canon(c0), canon(c1)
    assert np.array_equal(np.asarray(c0["node"])[o0], np.asarray(c1["node"])[o1])
    sv.set_learned_sdf(False)

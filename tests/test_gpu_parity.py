"""Step parity of the CUDA path against the FP64 CPU oracle, from identical state.

The external-force hook runs after the contact forces of a step and before the
second half kick, so the state it sees (positions, orientations, velocities,
forces, torques) is exactly the state the step's detection and forces were
computed from. The oracle recomputes hash, sorted order, cell ranges,
contact lists and forces from that state (with the GPU's previous contact list
as history) and the results are compared:

* integer outputs (cell keys, sorted order, cell ranges, per-node contact pairs
  with their partner) bit-exact;
* contact geometry, carried-over springs, forces and torques within a relative
  tolerance of 1e-9 (FP64; the device normalises with rsqrt and contracts FMAs,
  the CPU oracle does neither).

Each step test runs in the plain FP64 form and in both precision forms (FP32
screening on FP16 / BF16 SDF templates): the screen only rejects nodes that the
FP64 test provably rejects, so all three must meet the same bounds.
"""
import numpy as np
import pytest

from conftest import load_oracle
from helpers import canon, dense_ellipsoid_scene, history_from_gpu, load_scene

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def _capture(sv):
    box = {}

    def hook(t):
        box.update(sv.state())
        box["t"] = t
    return box, hook


def _oracle_from(sv, lsdem, st, sc, periodic=0):
    ora = load_oracle()
    model = ora.model_from_solver(sv)
    for k in ("pos", "vel", "angvel", "quat"):
        model["particles"][k] = st[k].copy()
    if model["walls"] is not None:
        model["walls"].update({k: v for k, v in sv.wall_state().items()})
    model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"], periodic=periodic)
    return ora.OracleSim(model)


def _close(a, b, rtol=RTOL, scale=None):
    a, b = np.asarray(a), np.asarray(b)
    s = scale if scale is not None else max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() <= rtol * s


def _compare_lists(gpu, orc, n_tot, label):
    og = canon(gpu)
    oo = canon({"node": orc["node"], "partner": orc["partner"]})
    assert len(og) == len(oo), f"{label}: {len(og)} GPU contacts vs {len(oo)} oracle"
    assert np.array_equal(gpu["node"][og], orc["node"][oo]), f"{label}: node ids differ"
    assert np.array_equal(gpu["partner"][og], orc["partner"][oo]), f"{label}: partners differ"
    cnt = np.bincount(gpu["node"], minlength=n_tot)
    assert np.array_equal(cnt, orc["count"]), f"{label}: per-node counts differ"
    if len(og):
        h = float(np.abs(orc["point"]).max())
        assert _close(gpu["point"][og], orc["point"][oo], scale=h), f"{label}: contact points"
        assert _close(gpu["normal"][og], orc["normal"][oo], rtol=1e-9, scale=1.0), f"{label}: normals"
        assert _close(gpu["overlap"][og], orc["overlap"][oo], rtol=1e-6), f"{label}: overlaps"
    return og, oo


@pytest.mark.parametrize("prec", [0, 1, 2])
@pytest.mark.parametrize("seed", [7, 11])
def test_step_parity_particles_and_floor(lsdem, seed, prec):
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=seed)
    sv = load_scene(lsdem, scenes, sc, precision=prec)
    dt = 1e-6
    prev = None
    for step in range(3):
        box, hook = _capture(sv)
        sv.step(dt, 1, hook=hook)
        sim = _oracle_from(sv, lsdem, box, sc)
        n_tot = sim.nodes.total
        if prev is not None:
            sim.old["pp"] = history_from_gpu(prev["pp"], n_tot)
            sim.old["pw"] = history_from_gpu(prev["pw"], n_tot)
        sim.detect_all()
        # broadphase: keys, stable order, cell ranges
        hh = sv.hash()
        assert np.array_equal(hh["key"], sim.last_hash["key"])
        assert np.array_equal(hh["sorted_idx"], sim.last_hash["sorted_idx"])
        assert np.array_equal(hh["sorted_key"], sim.last_hash["sorted_key"])
        assert np.array_equal(hh["start"], sim.last_hash["start"])
        assert np.array_equal(hh["end"], sim.last_hash["end"])
        cpp = sv.contacts(lsdem.CONTACT_PARTICLE, geometry=True)
        cpw = sv.contacts(lsdem.CONTACT_WALL, geometry=True)
        assert len(cpp["node"]) > 50 and len(cpw["node"]) > 10, "scene must produce contacts"
        og, oo = _compare_lists(cpp, sim.last["pp"], n_tot, "particle")
        wg, wo = _compare_lists(cpw, sim.last["pw"], n_tot, "wall")
        sim.forces(dt)
        # springs after the force update (FP64 history)
        s_scale = max(np.abs(sim.last["pp"]["spring"]).max(), 1e-300)
        assert _close(cpp["spring"][og], sim.last["pp"]["spring"][oo], rtol=1e-7, scale=s_scale)
        if step > 0:
            assert np.abs(cpp["spring"]).max() > 0, "history must carry non-zero springs"
        f_scale = np.abs(sim.F).max()
        t_scale = np.abs(sim.T).max()
        assert _close(box["force"], sim.F, rtol=1e-7, scale=f_scale), np.abs(box["force"] - sim.F).max() / f_scale
        assert _close(box["torque"], sim.T, rtol=1e-7, scale=t_scale), np.abs(box["torque"] - sim.T).max() / t_scale
        prev = {"pp": cpp, "pw": cpw}


def test_trajectory_matches_oracle(lsdem):
    """20 steps from the same initial state: GPU and oracle trajectories agree to FP64 round-off growth."""
    from lsdem_b200 import scenes
    ora = load_oracle()
    sc = dense_ellipsoid_scene(scenes, n=27, seed=3)
    sv = load_scene(lsdem, scenes, sc)
    model = ora.model_from_solver(sv)
    model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"])
    model["walls"].update(sv.wall_state())
    sim = ora.OracleSim(model)
    dt = 2e-6
    for _ in range(20):
        sim.step(dt)
    sv.step(dt, 20)
    st = sv.state()
    L = 5e-3
    assert np.abs(st["pos"] - sim.P["pos"]).max() < 1e-9 * L
    vmax = np.abs(sim.P["vel"]).max()
    assert np.abs(st["vel"] - sim.P["vel"]).max() < 1e-6 * vmax
    assert np.abs(st["quat"] - sim.P["quat"]).max() < 1e-9

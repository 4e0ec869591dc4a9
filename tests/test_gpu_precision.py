"""Precision forms (FP32 screening on FP16 / BF16 SDF templates, FP64 contact evaluation)
against the plain FP64 form, on a periodic polydisperse scene with random velocities.

The FP32 screen rejects a node only when its error bounds prove that the FP64 node test
rejects it; every other node and every contact goes through the FP64 code. So from the
same initial state the three forms must produce identical contact lists (node, partner,
image) at every step, and forces / torques that differ only by the order of the FP64
summation (relative 1e-10 of the largest value bounds that with a wide margin over the
few steps compared here).
"""
import numpy as np
import pytest

from helpers import canon

pytestmark = pytest.mark.gpu


def _scene(lsdem, n, seed, n_grid, n_nodes):
    from lsdem_b200 import scenes
    T = scenes.unit_templates(n_grid=n_grid, n_nodes=n_nodes)
    box = 0.1 * (n / 1e5) ** (1.0 / 3.0)
    sc = scenes.polydisperse_periodic(lsdem, n=n, box=box, seed=seed, templates=T, n_grid=n_grid, n_nodes=n_nodes)
    scenes.resolve_deep_overlaps(lsdem, sc)
    return sc


def _run(lsdem, sc, prec, steps):
    from lsdem_b200 import scenes
    sv = lsdem.Solver()
    scenes.load_polydisperse(sv, sc)
    sv.set_precision(prec)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    out = []
    for _ in range(steps):
        box = {}
        sv.step(sc["dt"], 1, hook=lambda t: box.update(sv.state()))
        c = {"pp": sv.contacts(lsdem.CONTACT_PARTICLE), "g": sv.contacts(lsdem.CONTACT_GHOST)}
        out.append((box, c))
    sv.close()
    return out


@pytest.mark.parametrize("prec", [1, 2])
def test_precision_form_equals_fp64_form(lsdem, prec):
    sc = _scene(lsdem, n=1500, seed=41, n_grid=32, n_nodes=800)
    sc["dt"] = 2e-7
    ref = _run(lsdem, sc, 0, 4)
    got = _run(lsdem, sc, prec, 4)
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
            s = np.abs(b0[q]).max()
            err = np.abs(b1[q] - b0[q]).max() / s
            assert err <= 1e-10, (q, err)
    assert n_contacts > 200, "scene must produce contacts"

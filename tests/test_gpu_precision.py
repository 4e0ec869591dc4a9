"""Precision form (FP32 narrowphase and contact law on FP16 / BF16 SDF templates, FP64
state and spring history) against the FP64 oracle, from identical state.

The state at force time is captured in the external-force hook of the FP32 solver; the
oracle recomputes contacts and forces in FP64 from it. Errors are relative to the
largest FP64 force (torque): max-norm and L2 over all particles, plus the relative
error of the total normal elastic energy. Bounds: FP16 templates <= 1e-3 (the
precision-form target), BF16 templates <= 2e-2 (8-bit mantissa).
"""
import numpy as np
import pytest

from conftest import load_oracle
from helpers import dense_ellipsoid_scene

pytestmark = pytest.mark.gpu

BOUND = {1: 1e-3, 2: 2e-2}


def _errors(lsdem, sv, sc, periodic=0):
    ora = load_oracle()
    box = {}

    def hook(t):
        box.update(sv.state())

    sv.step(sc["dt"], 1, hook=hook)
    sv.step(sc["dt"], 1, hook=hook)
    model = ora.model_from_solver(sv)
    for k in ("pos", "vel", "angvel", "quat"):
        model["particles"][k] = box[k]
    if model["walls"] is not None:
        model["walls"].update(sv.wall_state())
    model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"], periodic=periodic)
    sim = ora.OracleSim(model)
    # history of the FP32 run's previous step is not needed: both sides start springs from the
    # same carried values only when lists match, so compare the normal part through forces of a
    # step whose springs are tiny (dt-scale) against the FP64 recomputation
    sim.detect_all()
    sim.forces(sc["dt"])
    F, T = sim.F, sim.T
    fmax, tmax = np.abs(F).max(), np.abs(T).max()
    e = {
        "force_max": float(np.abs(box["force"] - F).max() / fmax),
        "force_l2": float(np.linalg.norm(box["force"] - F) / np.linalg.norm(F)),
        "torque_max": float(np.abs(box["torque"] - T).max() / tmax),
        "torque_l2": float(np.linalg.norm(box["torque"] - T) / np.linalg.norm(T)),
    }
    c = sv.contacts(lsdem.CONTACT_PARTICLE, geometry=True)
    en32 = float(np.sum(c["en_n"]))
    en64 = float(np.sum(sim.last["pp"]["en_n"]))
    e["energy_n"] = abs(en32 - en64) / en64
    return e


@pytest.mark.parametrize("prec", [1, 2])
def test_precision_form_force_error_ellipsoids(lsdem, prec):
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=5, vel_sigma=0.0)
    sc["angvel"] = np.zeros_like(sc["angvel"])
    sc["dt"] = 1e-7
    sv = lsdem.Solver()
    scenes.load_into(sv, sc)
    sv.set_precision(prec)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    e = _errors(lsdem, sv, sc)
    print(f"precision {prec}: {e}")
    assert e["force_l2"] <= BOUND[prec], e
    assert e["torque_l2"] <= 5 * BOUND[prec], e
    assert e["energy_n"] <= BOUND[prec], e


def test_precision_form_periodic_polydisperse(lsdem):
    from lsdem_b200 import scenes
    T = scenes.unit_templates(n_grid=24, n_nodes=400)
    n = 800
    box = 0.1 * (n / 1e5) ** (1.0 / 3.0)
    sc = scenes.polydisperse_periodic(lsdem, n=n, box=box, seed=31, templates=T, vel_sigma=0.0)
    scenes.resolve_deep_overlaps(lsdem, sc)
    sc["dt"] = 1e-7
    sv = lsdem.Solver()
    scenes.load_polydisperse(sv, sc)
    sv.set_precision(1)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    e = _errors(lsdem, sv, sc, periodic=7)
    print(f"periodic polydisperse, FP16 templates: {e}")
    assert e["force_l2"] <= BOUND[1], e

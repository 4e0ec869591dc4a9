"""Sector periodicity on the GPU against the oracle.

The quarter domain x >= 0, y >= 0 about the z axis through the domain minimum
(addPeriodicBoundarySector, LSSolver.h:448-452; PeriodicBoundary.h:313-420): particles
leaving across x = 0 or y = 0 are turned by -/+90 degrees (position, velocity,
orientation), images turned by 90, 180 and 270 degrees stand in for the neighbours
across the cut planes.

* Step parity from identical state (captured in the external-force hook): particle,
  wall and image contact lists (per image set, codes 8, 16, 32) bit-exact, forces and
  torques within 1e-7 of the largest, in the FP64 form and the BF16 screen.
* Trajectory: a column of particles starts outside the quarter domain, so it is
  turned by the wrap in the first step; 10 steps of the GPU and of the oracle from the
  same initial state agree in positions, velocities and orientations.
"""
import numpy as np
import pytest

from conftest import load_oracle
from helpers import canon, dense_ellipsoid_scene, history_from_gpu, load_scene

pytestmark = pytest.mark.gpu

SECTOR = 8


def _scene(lsdem, outside=False, seed=9):
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=seed, vel_sigma=0.05)
    # first lattice row and column 3.5 mm from the cut planes x = 0 and y = 0
    sc["pos"][:, 0] -= sc["pos"][:, 0].min() - 3.5e-3
    sc["pos"][:, 1] -= sc["pos"][:, 1].min() - 3.5e-3
    sc["min"] = np.zeros(3)
    if outside:
        col = sc["pos"][:, 0] < 4e-3
        sc["pos"][col, 0] = -1.0e-3  # left of x = 0: turned by -90 degrees in the first step
        sc["vel"][col, 0] = -0.2
    return sc


def _load(lsdem, sc, prec):
    from lsdem_b200 import scenes
    sv = load_scene(lsdem, scenes, sc, precision=prec)
    sv.set_periodic(SECTOR)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    return sv


def _oracle(ora, sv, st, sc):
    model = ora.model_from_solver(sv)
    for k in ("pos", "vel", "angvel", "quat"):
        model["particles"][k] = st[k].copy()
    model["walls"].update(sv.wall_state())
    model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"], periodic=SECTOR)
    return ora.OracleSim(model)


@pytest.mark.parametrize("prec", [0, 2])
def test_sector_step_parity(lsdem, prec):
    ora = load_oracle()
    sc = _scene(lsdem)
    sv = _load(lsdem, sc, prec)
    prev = None
    total_img = 0
    for step in range(3):
        box = {}
        sv.step(1e-6, 1, hook=lambda t: box.update(sv.state()))
        sim = _oracle(ora, sv, box, sc)
        nt = sim.nodes.total
        if prev is not None:
            sim.old["pp"] = history_from_gpu(prev["pp"], nt)
            sim.old["pw"] = history_from_gpu(prev["pw"], nt)
            for m, c in prev["g"].items():
                sim.old[f"g{m}"] = history_from_gpu(c, nt)
        sim.detect_all()
        lists = {"pp": sv.contacts(lsdem.CONTACT_PARTICLE), "pw": sv.contacts(lsdem.CONTACT_WALL)}
        for name in ("pp", "pw"):
            g, o = lists[name], sim.last[name]
            a, b = canon(g), canon({"node": o["node"], "partner": o["partner"]})
            assert len(a) == len(b), (name, len(a), len(b))
            assert np.array_equal(g["node"][a], o["node"][b]) and np.array_equal(g["partner"][a], o["partner"][b])
        cg = sv.contacts(lsdem.CONTACT_GHOST)
        assert set(np.unique(cg["image"])) <= {8, 16, 32}
        gl = {}
        for m in (8, 16, 32):
            sel = cg["image"] == m
            sub = {k: v[sel] for k, v in cg.items()}
            gl[m] = sub
            o = sim.last[f"g{m}"]
            a, b = canon(sub), canon({"node": o["node"], "partner": o["partner"]})
            assert len(a) == len(b), (m, len(a), len(b))
            assert np.array_equal(sub["node"][a], o["node"][b]) and np.array_equal(sub["partner"][a], o["partner"][b])
            total_img += len(a)
        sim.forces(1e-6)
        assert np.abs(box["force"] - sim.F).max() <= 1e-7 * np.abs(sim.F).max(), step
        assert np.abs(box["torque"] - sim.T).max() <= 1e-7 * np.abs(sim.T).max(), step
        prev = {"pp": lists["pp"], "pw": lists["pw"], "g": gl}
    assert total_img > 20, "particles must touch the turned images"
    sv.close()


def test_sector_wrap_trajectory(lsdem):
    ora = load_oracle()
    sc = _scene(lsdem, outside=True)
    sv = _load(lsdem, sc, 0)
    model = ora.model_from_solver(sv)
    model["walls"].update(sv.wall_state())
    model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"], periodic=SECTOR)
    sim = ora.OracleSim(model)
    out = sc["pos"][:, 0] < 0
    dt = 1e-6
    for _ in range(10):
        sim.step(dt)
    sv.step(dt, 10)
    st = sv.state()
    # the column left of x = 0 was turned onto the y > 0 side
    assert out.sum() >= 4 and (st["pos"][out, 0] >= 0).all() and (st["pos"][out, 1] >= 0).all()
    assert np.abs(st["vel"][out, 1]).max() > 0.1  # turned by -90 degrees: -0.2 m/s along x became +0.2 along y
    L = 5e-3
    assert np.abs(st["pos"] - sim.P["pos"]).max() < 1e-9 * L
    vmax = np.abs(sim.P["vel"]).max()
    assert np.abs(st["vel"] - sim.P["vel"]).max() < 1e-6 * vmax
    assert np.abs(st["quat"] - sim.P["quat"]).max() < 1e-9
    sv.close()

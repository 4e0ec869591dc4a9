"""A rotating curved wall on the GPU against the FP64 oracle, from identical state.

A small closed drum (radius 20 mm, length 30 mm, turning at 10 rad/s about x) with
superquadric particles (templates from subdivided superquadric meshes, grids built
on the GPU) pressed against its lower half and a second ring of particles inside
them. The reference tests every surface node against every wall of its cell
neighbourhood; the solver lists a wall for a particle only when the particle's
bounding sphere can reach phi <= 0 in the wall's grid (candidate stage) and then
screens the whole body before its clusters, so this test checks that these culls
drop no contact: per step, the wall and particle contact lists bit-exact, forces
and torques within 1e-7 of the largest, for the FP64 form and the BF16 screen.
The wall's rotation (quaternion integration, wall velocity in the contact law) is
checked by the same comparison over several steps.
"""
import math

import numpy as np
import pytest

from conftest import load_oracle
from helpers import canon, history_from_gpu

pytestmark = pytest.mark.gpu


def _drum_scene(lsdem, seed=5):
    from lsdem_b200 import scenes
    rng = np.random.default_rng(seed)
    T = scenes.superquadric_templates(lsdem, rng, 2, (2.5, 6.0), (2.0e-3, 3.0e-3), 20, 300, level=3)
    tm = scenes._unit_density_templates(lsdem, T)
    R, L = 0.02, 0.03
    b = max(t["bound"] for t in tm)
    pos = []
    for x in (-0.009, 0.0, 0.009):
        for th in np.linspace(-150, -30, 6):  # outer ring: reaches into the wall
            t = math.radians(th)
            pos.append((x, (R - 0.85 * b) * math.cos(t), (R - 0.85 * b) * math.sin(t)))
        for th in np.linspace(-140, -40, 4):  # inner ring: touches the outer one
            t = math.radians(th)
            pos.append((x, (R - 2.7 * b) * math.cos(t), (R - 2.7 * b) * math.sin(t)))
    pos = np.array(pos)
    n = len(pos)
    shape = rng.integers(0, len(tm), n).astype(np.int32)
    scale = np.ones(n)
    inv_mass, inv_inertia = scenes._body_arrays(tm, shape, scale, 2500.0)
    w = scenes.drum_wall(R, L, 5e-4, mu=0.5, e=0.6)
    w.update(pos=np.zeros(3), quat=np.array([1.0, 0, 0, 0]), angvel=np.array([10.0, 0, 0]))
    return {"templates": tm, "shape": shape, "scale": scale, "pos": pos, "quat": scenes.random_quaternions(rng, n),
            "vel": rng.normal(0, 0.05, (n, 3)), "angvel": rng.normal(0, 5.0, (n, 3)), "inv_mass": inv_mass,
            "inv_inertia": inv_inertia, "kn": 1e5, "ks": 8e4, "mu": 0.5, "e": 0.6, "dt": 1e-6,
            "min": np.array([-L / 2, -R, -R]), "max": np.array([L / 2, R, R]), "gravity": np.array([0, 0, -9.81]),
            "periodic": 0, "walls": [w]}


def _compare(gpu, orc, label):
    og = canon(gpu)
    oo = canon({"node": orc["node"], "partner": orc["partner"]})
    assert len(og) == len(oo), f"{label}: {len(og)} GPU contacts vs {len(oo)} oracle"
    assert np.array_equal(np.asarray(gpu["node"])[og], orc["node"][oo]), label
    assert np.array_equal(np.asarray(gpu["partner"])[og], orc["partner"][oo]), label
    return og, oo


@pytest.mark.parametrize("prec", [0, 2])
def test_rotating_drum_wall_parity(lsdem, prec):
    from lsdem_b200 import scenes
    ora = load_oracle()
    sc = _drum_scene(lsdem)
    sv = lsdem.Solver()
    scenes.load_polydisperse(sv, sc)
    sv.set_precision(prec)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    dt = sc["dt"]
    prev = None
    n_wall = 0
    for step in range(4):
        box = {}
        sv.step(dt, 1, hook=lambda t: box.update(sv.state()))
        model = ora.model_from_solver(sv)
        for k in ("pos", "vel", "angvel", "quat"):
            model["particles"][k] = box[k]
        model["walls"].update(sv.wall_state())
        model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"])
        sim = ora.OracleSim(model)
        nt = sim.nodes.total
        if prev is not None:
            sim.old["pp"] = history_from_gpu(prev["pp"], nt)
            sim.old["pw"] = history_from_gpu(prev["pw"], nt)
        sim.detect_all()
        cpp = sv.contacts(lsdem.CONTACT_PARTICLE)
        cpw = sv.contacts(lsdem.CONTACT_WALL)
        _compare(cpp, sim.last["pp"], "particle")
        _compare(cpw, sim.last["pw"], "wall")
        n_wall += len(cpw["node"])
        sim.forces(dt)
        fs, ts = np.abs(sim.F).max(), np.abs(sim.T).max()
        assert np.abs(box["force"] - sim.F).max() <= 1e-7 * fs, step
        assert np.abs(box["torque"] - sim.T).max() <= 1e-7 * ts, step
        prev = {"pp": cpp, "pw": cpw}
    ws = sv.wall_state()
    # the drum turned: its quaternion left the identity by 4 steps of 10 rad/s
    assert abs(ws["quat"][0, 1]) > 0.5 * 4 * dt * 10.0 / 2.0
    sv.close()
    assert n_wall > 40, "particles must press on the wall"

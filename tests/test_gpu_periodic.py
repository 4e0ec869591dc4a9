"""Periodic images on the GPU against the oracle: wrap, image sets, image cell keys,
contacts with images (per image set) and the resulting forces, from identical state,
in the plain FP64 form and in both precision forms.

Uses a small, dense, triply periodic polydisperse scene of the four scaled templates, so
that many particles touch images across the faces.
"""
import numpy as np
import pytest

from conftest import load_oracle
from helpers import canon

pytestmark = pytest.mark.gpu


def _scene(lsdem, n=600, seed=21):
    from lsdem_b200 import scenes
    T = scenes.unit_templates(n_grid=16, n_nodes=200)
    box = 0.1 * (n / 1e5) ** (1.0 / 3.0)
    return scenes.polydisperse_periodic(lsdem, n=n, box=box, seed=seed, templates=T, n_grid=16, n_nodes=200)


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_periodic_step_parity(lsdem, prec):
    from lsdem_b200 import scenes
    ora = load_oracle()
    sc = _scene(lsdem)
    sv = lsdem.Solver()
    scenes.load_polydisperse(sv, sc)
    sv.set_precision(prec)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    box = {}

    def hook(t):
        box.update(sv.state())

    for step in range(2):
        sv.step(sc["dt"], 1, hook=hook)
        model = ora.model_from_solver(sv)
        for k in ("pos", "vel", "angvel", "quat"):
            model["particles"][k] = box[k]
        model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"], periodic=7)
        sim = ora.OracleSim(model)
        if step > 0:
            from helpers import history_from_gpu
            nt = sim.nodes.total
            sim.old["pp"] = history_from_gpu(prev_pp, nt)
            for m, c in prev_g.items():
                sim.old[f"g{m}"] = history_from_gpu(c, nt)
        sim.detect_all()
        cpp = sv.contacts(lsdem.CONTACT_PARTICLE, geometry=True)
        o = sim.last["pp"]
        og, oo = canon(cpp), canon({"node": o["node"], "partner": o["partner"]})
        assert len(og) == len(oo) and len(og) > 100
        assert np.array_equal(cpp["node"][og], o["node"][oo])
        assert np.array_equal(cpp["partner"][og], o["partner"][oo])
        cg = sv.contacts(lsdem.CONTACT_GHOST, geometry=True)
        total = 0
        prev_g = {}
        for m in (1, 2, 4, 3, 5, 6, 7):
            sel = cg["image"] == m
            sub = {k: v[sel] for k, v in cg.items()}
            prev_g[m] = sub
            ol = sim.last[f"g{m}"]
            a, b = canon(sub), canon({"node": ol["node"], "partner": ol["partner"]})
            assert len(a) == len(b), (m, len(a), len(b))
            assert np.array_equal(sub["node"][a], ol["node"][b]), m
            assert np.array_equal(sub["partner"][a], ol["partner"][b]), m
            if len(a):
                assert np.abs(sub["point"][a] - ol["point"][b]).max() < 1e-12
            total += len(a)
        assert total > 20, "scene must produce contacts with images"
        prev_pp = cpp
        sim.forces(sc["dt"])
        fs = np.abs(sim.F).max()
        assert np.abs(box["force"] - sim.F).max() < 1e-7 * fs
        assert np.abs(box["torque"] - sim.T).max() < 1e-7 * np.abs(sim.T).max()
    assert (sv.state()["pos"] >= sc["min"]).all() and (sv.state()["pos"] < sc["max"]).all()

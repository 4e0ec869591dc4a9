"""Steps replayed from CUDA graphs against steps launched kernel by kernel.

The same scenes stepped with graph replay (lsdem_set_graphs on, the default) and with
every kernel launched (off) give the same contact lists and the same state: positions,
velocities and orientations within 1e-12 of their scale (only the order of the FP64
force atomics can differ between runs), in the FP64 and BF16 forms, with periodic
images and with a wall, with and without an external-force hook (the graph then ends
before the hook, the second half kick follows it); a capacity growth inside the run
(re-capture) included.
"""
import numpy as np
import pytest

from helpers import canon, dense_ellipsoid_scene, load_scene

pytestmark = pytest.mark.gpu


def _run(lsdem, sc, prec, graphs, steps, periodic=0, cap=None, hook=False):
    from lsdem_b200 import scenes
    sv = load_scene(lsdem, scenes, sc, precision=prec, **(cap or {}))
    sv.set_graphs(graphs)
    if periodic:
        sv.set_periodic(periodic)
        sv.initialize(sc["min"], sc["max"], sc["gravity"])
    times = []
    sv.step(2e-6, steps, hook=(lambda t: times.append(t)) if hook else None)
    if hook:
        assert len(times) >= steps  # called every step (again for re-run batches)
    st = sv.state()
    c = sv.contacts(lsdem.CONTACT_PARTICLE)
    launches = sv.num(8)
    sv.close()
    return st, c, launches


@pytest.mark.parametrize("hook", [False, True])
@pytest.mark.parametrize("prec", [0, 2])
@pytest.mark.parametrize("periodic", [0, 3])
def test_graph_replay_equals_eager(lsdem, prec, periodic, hook):
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=5)
    cap = {"pp": 2, "contacts": 64}  # small capacities: the run grows them (batch re-run, new capture)
    a, ca, la = _run(lsdem, sc, prec, True, 40, periodic, cap, hook)
    b, cb, lb = _run(lsdem, sc, prec, False, 40, periodic, cap, hook)
    assert la == lb > 0
    oa, ob = canon(ca), canon(cb)
    assert len(oa) == len(ob) > 20
    assert np.array_equal(ca["node"][oa], cb["node"][ob]) and np.array_equal(ca["partner"][oa], cb["partner"][ob])
    for k in ("pos", "vel", "angvel", "quat"):
        scale = max(np.abs(b[k]).max(), 1e-30)
        assert np.abs(a[k] - b[k]).max() <= 1e-12 * scale, k

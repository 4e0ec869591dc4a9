"""Step contract across calls: solve() phases, the external-force hook and snapshots.

* A second lsdem_initialize after steps (the drop-in's next solve() phase) continues from
  the current state with the last step's forces and contact history, as the reference
  keeps its host mirrors, forces and contact arrays between phases (LSSolver.h:478-505,
  612-623, SolidInteraction.h:24-27): 20 + 20 steps in two phases equal 40 steps in one,
  contact springs included.
* The hook runs exactly once per step, after complete forces, also when the step's lists
  overflow and it is re-run with grown capacities (LSSolver.h:1000-1011 calls it once).
* lsdem_snapshot_save / lsdem_snapshot_load: a solver restored from a snapshot takes the
  same steps as the one that saved it; a snapshot of another model is rejected.

States are compared within 1e-12 of their scale (only the order of FP64 force atomics
differs between runs), contact lists exactly.
"""
import numpy as np
import pytest

from helpers import canon, dense_ellipsoid_scene, load_scene

pytestmark = pytest.mark.gpu

DT = 2e-6


def _same(a, b, keys=("pos", "vel", "angvel", "quat")):
    for k in keys:
        scale = max(np.abs(b[k]).max(), 1e-30)
        assert np.abs(a[k] - b[k]).max() <= 1e-12 * scale, (k, np.abs(a[k] - b[k]).max() / scale)


def _same_contacts(ca, cb):
    oa, ob = canon(ca), canon(cb)
    assert len(oa) == len(ob) and len(oa) > 0
    assert np.array_equal(ca["node"][oa], cb["node"][ob]) and np.array_equal(ca["partner"][oa], cb["partner"][ob])
    s = np.abs(cb["spring"]).max()
    assert s > 0
    assert np.abs(ca["spring"][oa] - cb["spring"][ob]).max() <= 1e-10 * s


def _scene():
    from lsdem_b200 import scenes
    return dense_ellipsoid_scene(scenes, n=64, seed=17, vel_sigma=0.2)


@pytest.mark.parametrize("prec", [0, 2])
def test_two_phases_equal_one(lsdem, prec):
    from lsdem_b200 import scenes
    sc = _scene()
    one = load_scene(lsdem, scenes, sc, precision=prec)
    one.step(DT, 40)
    a, ca = one.state(), one.contacts(lsdem.CONTACT_PARTICLE)
    one.close()
    two = load_scene(lsdem, scenes, sc, precision=prec)
    two.step(DT, 20)
    mid = two.contacts(lsdem.CONTACT_PARTICLE)
    assert len(mid["node"]) > 0 and np.abs(mid["spring"]).max() > 0  # history to carry
    two.initialize(sc["min"], sc["max"], sc["gravity"])  # the next phase
    assert two.time == 0.0
    two.step(DT, 20)
    b, cb = two.state(), two.contacts(lsdem.CONTACT_PARTICLE)
    two.close()
    _same(b, a)
    _same_contacts(cb, ca)


def test_host_edit_between_phases(lsdem):
    """Between phases the host copy of the state is the device's (the reference downloads it
    at every output): reading it after a host-side edit gives the state the first phase
    reached, the next phase starts from it, and the edit (the floor's angular velocity)
    applies from then on."""
    from lsdem_b200 import scenes
    sc = _scene()
    w = np.array([0.0, 0.0, 30.0])
    sv = load_scene(lsdem, scenes, sc)
    sv.step(DT, 15)
    s1 = sv.state()
    sv.set_wall_angular_velocity(0, w)
    _same(sv.state(), s1)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    _same(sv.state(), s1)
    sv.step(DT, 15)
    ws = sv.wall_state()
    assert np.allclose(ws["angvel"][0], w)
    th = 30.0 * 15 * DT
    assert np.abs(ws["quat"][0] - [np.cos(th / 2), 0.0, 0.0, np.sin(th / 2)]).max() < 1e-9
    assert np.abs(sv.state()["pos"] - s1["pos"]).max() > 0
    sv.close()


def test_hook_once_per_step_through_overflow(lsdem):
    from lsdem_b200 import scenes
    sc = _scene()
    big = load_scene(lsdem, scenes, sc, pp=64, wall=8, contacts=1 << 18)
    big.step(DT, 12)
    a = big.state()
    big.close()
    small = load_scene(lsdem, scenes, sc, pp=1, wall=1, contacts=64)  # overflows in the first steps
    calls = []

    def hook(t):
        calls.append(t)

    small.step(DT, 12, hook=hook)
    assert small.num(7) > 0, "the run must have re-run overflowing steps"
    assert len(calls) == 12
    assert np.allclose(np.diff(calls), DT, rtol=1e-9, atol=0.0) and calls[0] == 0.0
    _same(small.state(), a)
    small.close()


@pytest.mark.parametrize("prec", [0, 2])
def test_snapshot_restores_the_run(lsdem, tmp_path, prec):
    from lsdem_b200 import scenes
    sc = _scene()
    path = tmp_path / "state.snp"
    sv = load_scene(lsdem, scenes, sc, precision=prec)
    sv.step(DT, 25)
    sv.snapshot_save(path)
    t_saved, steps_saved = sv.time, sv.num(6)
    sv.step(DT, 20)
    a, ca = sv.state(), sv.contacts(lsdem.CONTACT_PARTICLE)
    sv.close()
    sv = load_scene(lsdem, scenes, sc, precision=prec)
    sv.snapshot_load(path)
    assert sv.time == t_saved and sv.num(6) == steps_saved
    sv.step(DT, 20)
    b, cb = sv.state(), sv.contacts(lsdem.CONTACT_PARTICLE)
    sv.close()
    _same(b, a)
    _same_contacts(cb, ca)
    # a snapshot of another model is rejected
    other = dense_ellipsoid_scene(scenes, n=27, seed=3)
    sv = load_scene(lsdem, scenes, other)
    with pytest.raises(lsdem.LSDEMError):
        sv.snapshot_load(path)
    sv.close()

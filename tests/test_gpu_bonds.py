"""V-bonds on the GPU against the FP64 oracle, from identical state.

Bonds are created from the contacts of a dense ellipsoid scene (createBondsFromContacts,
LSSolver.h:385-418: one bond per particle-particle contact), then the scene is stepped in
a new phase, which keeps the contact history of the step before.
Before each step the bond flags and state are read; the external-force hook captures the
state the step's forces were computed from; the oracle recomputes contacts (with the
GPU's previous contact list as history) and contact + bond forces from it
(contactKernel.cu:273-351). Checked: bond flags after the step bit-exact (breakage),
bond state (displacement and moment measures, peak stresses, bond point) within 1e-9
relative, total forces and torques within 1e-7 of the largest — in the FP64 form and in
the BF16 precision form (bonds are FP64 in both).
"""
import numpy as np
import pytest

from conftest import load_oracle
from helpers import dense_ellipsoid_scene, history_from_gpu, load_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("strength", [2e6, 1e12])
@pytest.mark.parametrize("prec", [0, 2])
def test_bond_step_parity(lsdem, prec, strength):
    from lsdem_b200 import scenes
    ora = load_oracle()
    sc = dense_ellipsoid_scene(scenes, n=27, seed=13)
    sv = load_scene(lsdem, scenes, sc, precision=prec)
    dt = 1e-6
    sv.step(dt, 1)
    # the next phase keeps this step's contact history (as the reference's contact arrays)
    prev = {"pp": sv.contacts(lsdem.CONTACT_PARTICLE), "pw": sv.contacts(lsdem.CONTACT_WALL)}
    sv.create_bonds_from_contacts(1.0e-3, 1.0e-4, 1e8, 0.3, strength, strength, 0.3)
    nb = sv.num(2)
    assert nb > 20, "the scene must produce bonds"
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    broken = 0
    for step in range(3):
        before = sv.bonds()
        box = {}
        sv.step(dt, 1, hook=lambda t: box.update(sv.state()))
        after = sv.bonds()
        model = ora.model_from_solver(sv)
        for k in ("pos", "vel", "angvel", "quat"):
            model["particles"][k] = box[k]
        model["walls"].update(sv.wall_state())
        model["bonds"]["bonded"] = before["bonded"].copy()
        model["bonds"]["state"] = before["state"].copy()
        model.update(domain=(sc["min"], sc["max"]), gravity=sc["gravity"])
        sim = ora.OracleSim(model)
        if prev is not None:
            nt = sim.nodes.total
            sim.old["pp"] = history_from_gpu(prev["pp"], nt)
            sim.old["pw"] = history_from_gpu(prev["pw"], nt)
        sim.detect_all()
        sim.forces(dt)
        assert np.array_equal(sim.bonds["bonded"], after["bonded"]), step
        live = after["bonded"] == 1
        s_ref, s_gpu = sim.bonds["state"][live], after["state"][live]
        d = np.abs(s_gpu - s_ref)
        # normal / shear displacement (m), bending / twist measure (rad), peak normal and
        # shear stress (Pa), bond point (m): round-off scaled tolerances
        assert (d[:, 0:2] <= 1e-12).all() and (d[:, 6:9] <= 1e-12).all(), step
        assert (d[:, 2:4] <= 1e-9).all(), step
        if live.any():
            assert (d[:, 4:6] <= 1e-7 * np.abs(s_ref[:, 4:6]).max() + 1e-3).all(), step
        fs, ts = np.abs(sim.F).max(), np.abs(sim.T).max()
        assert np.abs(box["force"] - sim.F).max() <= 1e-7 * fs, step
        assert np.abs(box["torque"] - sim.T).max() <= 1e-7 * ts, step
        broken += int((before["bonded"] == 1).sum() - live.sum())
        prev = {"pp": sv.contacts(lsdem.CONTACT_PARTICLE), "pw": sv.contacts(lsdem.CONTACT_WALL)}
    print(f"strength {strength:g}: {nb} bonds, {broken} broke during the 3 steps")
    if strength > 1e9:
        assert broken == 0 and (sv.bonds()["bonded"] == 1).all(), "unbreakable bonds must survive"
    else:
        assert broken > 0, "weak bonds must break"


def test_bonds_from_contacts_built_on_device_equal_host_routine(lsdem):
    """lsdem_create_bonds_from_contacts builds the bonds on the device (bonds.cu). The same
    contacts added one by one through lsdem_add_bond (the host routine, VBondedInteraction::add,
    VBondedInteraction.h:74-195), in the contact list's order, give the same bonds bit for bit:
    topology, stiffness constants, local frames and points."""
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=19)
    args = (1.0e-3, 1.0e-4, 1e8, 0.3, 2e6, 2e6, 0.3)
    dev = load_scene(lsdem, scenes, sc)
    dev.step(1e-6, 2)
    c = dev.contacts(lsdem.CONTACT_PARTICLE, geometry=True)
    st = dev.state()
    nb = dev.particle_params()["node_base"]
    owner = np.searchsorted(nb, c["node"], side="right") - 1
    dev.create_bonds_from_contacts(*args)
    host = load_scene(lsdem, scenes, sc)
    host.set_state(pos=st["pos"], vel=st["vel"], angvel=st["angvel"], quat=st["quat"])
    for k in range(len(owner)):
        host.add_bond(int(owner[k]), int(c["partner"][k]), c["point"][k], c["normal"][k], *args)
    assert dev.num(2) == host.num(2) == len(owner) > 50
    bd, bh = dev.bonds(), host.bonds()
    assert np.array_equal(bd["ids"], bh["ids"])
    assert np.array_equal(bd["state"], bh["state"])
    pd, ph = dev.bond_params(), host.bond_params()
    for k in ("B", "geo", "frames"):
        assert np.array_equal(pd[k], ph[k]), k
    dev.close()
    host.close()

"""Frame output on the GPU (lsdem_write_vtu) against the solver's own state.

The files of one frame (the reference's LSSolver::output set: surface-node mesh,
particle centres, particle contacts, bonds, wall mesh, wall contacts) are read back
with a plain VTK XML reader (tests/helpers.py: base64 of an 8-byte byte count and
the data) and every array is checked against values computed here from the
solver's state, templates and contact lists:

* node world positions p + R(q) (s n) and velocities v + w x (x - p), as float32,
  within float rounding; particle ids and triangle connectivity (offset by each
  body's first node) exact;
* particle centres, velocities, angular velocities, orientations, radii;
* contacts (points, normals, sliding directions = normalised springs, energies) as
  sets; bonds (ids, flags, state); walls (vertices in world coordinates);
* a scene of 3.2M surface nodes (38 MB per vector array) crosses the writer's
  32 MB chunk boundary, so the base64 stream is carried across chunks.
"""
import time

import numpy as np
import pytest

from helpers import dense_ellipsoid_scene, load_scene, read_vtu

pytestmark = pytest.mark.gpu


def _rot(q, v):
    """Rotate rows of v by unit quaternions q (q0 scalar first)."""
    w, x, y, z = q[:, 0:1], q[:, 1:2], q[:, 2:3], q[:, 3:4]
    qv = np.concatenate([x, y, z], 1)
    t = 2.0 * np.cross(qv, v)
    return v + w * t + np.cross(qv, t)


def _expected_nodes(sv):
    from conftest import load_oracle
    ora = load_oracle()
    model = ora.model_from_solver(sv)
    pp = sv.particle_params()
    st = sv.state()
    shapes = model["shapes"]
    nodes, owner = [], []
    for p in range(sv.n_particles):
        loc = np.asarray(shapes[pp["shape"][p]]["nodes"]).reshape(-1, 3) * pp["scale"][p]
        nodes.append(loc)
        owner.append(np.full(len(loc), p))
    loc, owner = np.concatenate(nodes), np.concatenate(owner)
    q = st["quat"][owner]
    pw = st["pos"][owner] + _rot(q, loc)
    vw = st["vel"][owner] + np.cross(st["angvel"][owner], pw - st["pos"][owner])
    return pw, vw, owner, pp


def _close32(got, ref, scale):
    return np.abs(np.asarray(got, np.float64) - ref).max() <= 2e-7 * scale + 1e-30


def test_frame_files_match_state(lsdem, tmp_path):
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=7)
    sv = load_scene(lsdem, scenes, sc, precision=2)
    nn = 300
    tris = np.arange(3 * (nn // 3), dtype=np.int32).reshape(-1, 3)[::3]  # every third node triple
    for p in range(0, sv.n_particles, 2):  # half of the particles carry triangles
        sv.set_triangles(0, p, tris)
    sv.set_triangles(1, 0, np.array([[0, 1, 2], [0, 2, 3]]))
    sv.step(1e-6, 2)
    sv.create_bonds_from_contacts(1.0e-3, 1.0e-4, 1e8, 0.3, 1e12, 1e12, 0.3)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    sv.step(1e-6, 2)
    sv.write_vtu(tmp_path, 7, 123, 0.5)
    d = tmp_path
    # particles
    P = read_vtu(d / "LSParticle" / "Particle_0007.vtu")
    st = sv.state()
    pp = sv.particle_params()
    L = float(np.abs(st["pos"]).max())
    assert P["n_points"] == sv.n_particles and P["n_cells"] == 0
    assert np.float32(P["TIME"][0]) == np.float32(0.5) and P["STEP"][0] == 123
    assert _close32(P["points"], st["pos"], L)
    assert _close32(P["velocity"], st["vel"], np.abs(st["vel"]).max())
    assert _close32(P["angularVelocity"], st["angvel"], np.abs(st["angvel"]).max())
    assert _close32(P["orientation"], st["quat"], 1.0)
    assert _close32(P["radius"], pp["radius"], pp["radius"].max())
    # surface-node mesh
    M = read_vtu(d / "LSParticle" / "LSObjectMesh_0007.vtu")
    pw, vw, owner, pp = _expected_nodes(sv)
    assert M["n_points"] == len(pw)
    assert _close32(M["points"], pw, L)
    assert _close32(M["velocity"], vw, np.abs(vw).max())
    assert np.array_equal(M["particleID"], owner)
    base = np.concatenate([[0], np.cumsum(np.bincount(owner, minlength=sv.n_particles))])
    conn = np.concatenate([tris + base[p] for p in range(0, sv.n_particles, 2)])
    assert M["n_cells"] == len(conn)
    assert np.array_equal(M["connectivity"].reshape(-1, 3), conn)
    assert np.array_equal(M["offsets"], 3 * np.arange(1, len(conn) + 1))
    assert (M["types"] == 5).all()
    # contacts (sets: the writer's order is the solver's, the reference's is by node)
    for sub, kind in (("LSParticleInteraction", lsdem.CONTACT_PARTICLE),
                      ("LSParticle-WallInteraction", lsdem.CONTACT_WALL)):
        C = read_vtu(d / sub / "LSInteraction_0007.vtu")
        c = sv.contacts(kind, geometry=True)
        assert C["n_points"] == C["n_cells"] == len(c["node"]) > 0
        order_g = np.lexsort(C["points"].T[::-1])
        order_r = np.lexsort(c["point"].astype(np.float32).T[::-1])
        assert _close32(C["points"][order_g], c["point"][order_r], L)
        assert _close32(C["contactNormal"][order_g], c["normal"][order_r], 1.0)
        s = c["spring"][order_r]
        n = np.linalg.norm(s, axis=1)
        sd = np.where(n[:, None] > 1e-10, s / np.maximum(n, 1e-300)[:, None], 0.0)
        assert _close32(C["slidingDirection"][order_g], sd, 1.0)
        assert _close32(C["normalElasticEnergy"][order_g], c["en_n"][order_r], np.abs(c["en_n"]).max())
        assert _close32(C["slidingElasticEnergy"][order_g], c["en_s"][order_r], max(np.abs(c["en_s"]).max(), 1e-30))
        assert np.array_equal(C["connectivity"], np.arange(len(c["node"])))
        assert (C["types"] == 1).all()
    # bonds
    B = read_vtu(d / "LSParticleInteraction" / "VBondedInteraction_0007.vtu")
    b = sv.bonds()
    assert B["n_points"] == len(b["bonded"]) > 0
    assert np.array_equal(B["masterObjectID"], b["ids"][:, 0]) and np.array_equal(B["slaveObjectID"], b["ids"][:, 1])
    assert np.array_equal(B["activated"], b["bonded"])
    assert _close32(B["points"], b["state"][:, 6:9], L)
    for k, name in enumerate(("normalElasticEnergy", "shearElasticEnergy", "bendingElasticEnergy",
                              "torsionElasticEnergy", "maxNormalStress", "maxShearStress")):
        assert _close32(B[name], b["state"][:, k], max(np.abs(b["state"][:, k]).max(), 1e-30)), name
    # wall mesh
    W = read_vtu(d / "Wall" / "LSObjectMesh_0007.vtu")
    ws = sv.wall_state()
    verts = np.asarray(sc["floor"]["verts"])
    exp = ws["pos"][0] + _rot(np.repeat(ws["quat"][:1], len(verts), 0), verts)
    assert _close32(W["points"], exp, L)
    assert np.array_equal(W["connectivity"].reshape(-1, 3), [[0, 1, 2], [0, 2, 3]])
    assert (W["particleID"] == 0).all()
    sv.close()


def test_large_frame_crosses_chunks(lsdem, tmp_path):
    from lsdem_b200 import scenes
    sc = scenes.ellipsoid_falling(n=3200, n_nodes=1000, n_grid=16, seed=3)
    sv = lsdem.Solver()
    scenes.load_into(sv, sc)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    sv.step(1e-6, 2)
    sv.write_vtu(tmp_path, 1, 2, 2e-6)
    M = read_vtu(tmp_path / "LSParticle" / "LSObjectMesh_0001.vtu")
    pw, vw, owner, _ = _expected_nodes(sv)
    assert len(pw) == 3_200_000 and 12 * len(pw) > (32 << 20)
    L = float(np.abs(sv.state()["pos"]).max())
    assert _close32(M["points"], pw, L)
    assert _close32(M["velocity"], vw, max(np.abs(vw).max(), 1e-30))
    assert np.array_equal(M["particleID"], owner)
    assert M["n_cells"] == 0 and len(M["connectivity"]) == 0
    # a second frame from the same writer after more steps (timed: the writer is set up)
    sv.step(1e-6, 3)
    t0 = time.perf_counter()
    sv.write_vtu(tmp_path, 2, 5, 5e-6)
    dt = time.perf_counter() - t0
    size = sum(p.stat().st_size for p in tmp_path.rglob("*_0002.vtu"))
    print(f"frame of {len(pw)} surface nodes: {size / 1e6:.0f} MB of VTU in {dt * 1e3:.0f} ms "
          f"({size / dt / 1e9:.2f} GB/s)")
    M2 = read_vtu(tmp_path / "LSParticle" / "LSObjectMesh_0002.vtu")
    pw2, _, _, _ = _expected_nodes(sv)
    assert _close32(M2["points"], pw2, L)
    sv.close()

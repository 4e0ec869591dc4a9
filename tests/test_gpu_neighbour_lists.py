"""Step-to-step reuse of the broadphase against sorting and walking every step.

With lsdem_set_neighbour_lists on (the default) the candidate search tests each
particle's list from the last rebuild, and the cell sort and the rebuild run only
when a particle moved more than the rebuild distance; off, every step sorts and
walks the 27 cells as the reference does (LSSolver.h:1000-1011). The same scenes
stepped both ways give, after every batch, the same numbers of candidate pairs
(particles, walls, images) and contacts, and at the end the same contact lists and
the same state (within 1e-12 of its scale: only the order of the FP64 force atomics
differs between runs). Moving particles make the lists rebuild during the run, and
so do particles moved by the host between batches and periodic wraps; between
rebuilds a particle changes cells (placed 0.02 mm from a cell face, then moved
0.1 mm across it by the host), which the lists follow.
"""
import numpy as np
import pytest

from helpers import canon, dense_ellipsoid_scene, load_scene

pytestmark = pytest.mark.gpu

DT = 2e-6
CAP = {"pp": 48, "wall": 8, "ghost": 48, "contacts": 1 << 18}  # no capacity growth (which rebuilds) in the run


def _run(lsdem, sc, j, prec, reuse, periodic, batches=30, per=10):
    from lsdem_b200 import scenes
    sv = load_scene(lsdem, scenes, sc, precision=prec, **CAP)
    sv.set_neighbour_lists(reuse)
    if periodic:
        sv.set_periodic(periodic)
        sv.initialize(sc["min"], sc["max"], sc["gravity"])
    stats = []
    moved_cells = 0  # batches whose particles changed cells without a rebuild
    keys, builds = None, 0
    g = sv.grid()
    for b in range(batches):
        if b == 1:
            # particle j crosses its cell face: 0.1 mm, less than the rebuild distance
            pos = sv.state()["pos"]
            pos[j, 0] += sc["nudge"]
            sv.set_state(pos=pos)
        if b in (batches // 2, batches - 5):
            # the host moves a particle by 0.3 mm: more than the rebuild distance
            pos = sv.state()["pos"]
            pos[b % 7] += np.array([3e-4, 0.0, 0.0])
            sv.set_state(pos=pos)
        sv.step(DT, per)
        # cells from the positions (the hash accessor would sort and so force a rebuild)
        k1, b1 = np.floor((sv.state()["pos"] - g["min"]) * g["inv"]).astype(np.int64), sv.num(9)
        if keys is not None and b1 == builds and not np.array_equal(k1, keys):
            moved_cells += 1
        keys, builds = k1, b1
        s = sv.step_stats()
        stats.append((s["pairs_particle"], s["pairs_ghost"], s["pairs_wall"], s["contacts"]))
    st = sv.state()
    c = sv.contacts(lsdem.CONTACT_PARTICLE)
    counts = (sv.num(6), sv.num(9), moved_cells)
    sv.close()
    return st, c, stats, counts


def _scene(lsdem):
    """A 9 mm lattice of the (5, 4, 3) mm ellipsoids (bounding spheres overlap, so the
    lattice has contacts without the violent start of a denser one), shifted along x
    so that one particle j sits 0.02 mm from a cell face; after 10 steps the host
    moves it 0.1 mm across the face (less than the rebuild distance, 0.04 of the
    largest bounding radius = 0.2 mm)."""
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=64, seed=11, vel_sigma=0.3, spacing=9e-3)
    sv = load_scene(lsdem, scenes, sc)
    g = sv.grid()
    sv.close()
    cell = 1.0 / g["inv"][0]
    u = (sc["pos"][:, 0] - g["min"][0]) / cell
    frac = u - np.floor(u)
    up = (1.0 - frac) * cell - 2e-5    # shift that puts the particle 0.02 mm before its upper face
    down = -(frac * cell - 2e-5)       # ... 0.02 mm past its lower face
    j_up, j_dn = int(np.argmin(np.abs(up))), int(np.argmin(np.abs(down)))
    if abs(up[j_up]) <= abs(down[j_dn]):
        shift, j, nudge = up[j_up], j_up, 1e-4
    else:
        shift, j, nudge = down[j_dn], j_dn, -1e-4
    assert abs(shift) < 3e-3
    sc["pos"][:, 0] += shift
    sc["nudge"] = nudge
    return sc, j


@pytest.mark.parametrize("prec", [0, 2])
@pytest.mark.parametrize("periodic", [0, 3])
def test_reuse_equals_full_walk(lsdem, prec, periodic):
    sc, j = _scene(lsdem)
    a, ca, sa, (steps, builds, moved) = _run(lsdem, sc, j, prec, True, periodic)
    b, cb, sb, (_, builds_off, _) = _run(lsdem, sc, j, prec, False, periodic)
    assert sa == sb
    assert builds_off == 0  # counted only while the lists are on
    # the lists were rebuilt during the run (moves, the host's moves, wraps), not every
    # step, and a particle changed cells between rebuilds
    assert 3 <= builds < steps // 2, (builds, steps)
    assert moved >= 1
    oa, ob = canon(ca), canon(cb)
    assert len(oa) == len(ob)
    assert sum(x[3] for x in sa) > 100  # contacts over the batches
    assert np.array_equal(ca["node"][oa], cb["node"][ob]) and np.array_equal(ca["partner"][oa], cb["partner"][ob])
    for k in ("pos", "vel", "angvel", "quat"):
        scale = max(np.abs(b[k]).max(), 1e-30)
        assert np.abs(a[k] - b[k]).max() <= 1e-12 * scale, k


def _two_pair_scene(lsdem):
    """Two pairs of (5, 4, 3) mm ellipsoids with their long axes on the line of centres,
    2.05 bounding radii apart (0.25 mm gap) across two cell faces: the lower-index body
    sits 0.05 mm before a face, so at the build its partner is two cells away, outside its
    27-cell window, but within reach plus the margin. The bodies then close the gap by
    0.19 mm each, less than the rebuild distance (0.2 mm), and touch: the walk finds the
    pairs in the window of the moved cells, so the lists must hold them. Pair 1 lies along
    +x (the partner above the owner's cell), pair 2 along -z (below it)."""
    from lsdem_b200 import scenes
    shp = scenes.make_ellipsoid((5e-3, 4e-3, 3e-3), 16, 300)
    probe = {"shape": shp, "pos": np.array([[0.05, 0.05, 0.05]]), "quat": np.array([[1.0, 0, 0, 0]]),
             "vel": np.zeros((1, 3)), "kn": 1e5, "ks": 8e4, "mu": 0.5, "e": 0.6, "density": 2500.0,
             "min": np.zeros(3), "max": np.full(3, 0.1), "gravity": np.zeros(3), "floor": None}
    sv = load_scene(lsdem, scenes, probe)
    r = float(sv.particle_params()["radius"][0])
    w = 1.0 / sv.grid()["inv"]
    sv.close()
    assert np.allclose(w, w[0]) and 2 * r <= w[0] < 2.1 * r
    d = 2.05 * r
    eps = 5e-5
    s = np.sqrt(0.5)
    qz = np.array([s, 0.0, -s, 0.0])  # body x axis along world z
    pos = np.array([[3 * w[0] - eps, 0.05, 0.05], [3 * w[0] - eps + d, 0.05, 0.05],
                    [0.08, 0.08, 6 * w[0] + eps], [0.08, 0.08, 6 * w[0] + eps - d]])
    quat = np.array([[1.0, 0, 0, 0], [1.0, 0, 0, 0], qz, qz])
    v = 4.0
    vel = np.array([[v, 0, 0], [-v, 0, 0], [0, 0, -v], [0, 0, v]])
    return dict(probe, pos=pos, quat=quat, vel=vel), r


@pytest.mark.parametrize("prec", [0, 2])
def test_lists_hold_partners_beyond_the_27_cells(lsdem, prec):
    from lsdem_b200 import scenes
    sc, r = _two_pair_scene(lsdem)
    dt, steps = 2e-6, 24
    assert v_moved(sc, dt, steps) < 0.4 * 0.1 * r  # below the rebuild distance
    runs = []
    for reuse in (True, False):
        sv = load_scene(lsdem, scenes, sc, precision=prec, **CAP)
        sv.set_neighbour_lists(reuse)
        per = []
        for _ in range(steps):
            sv.step(dt, 1)
            s = sv.step_stats()
            per.append((s["pairs_particle"], s["contacts"]))
        runs.append((per, sv.num(9), sv.contacts(lsdem.CONTACT_PARTICLE), sv.state()))
        sv.close()
    (pa, builds, ca, sa), (pb, _, cb, sb) = runs
    assert builds == 1  # the lists were built once, before the bodies moved
    assert pb[0] == (0, 0) and max(x[0] for x in pb) == 2 and max(x[1] for x in pb) > 0  # both pairs touch
    assert pa == pb
    oa, ob = canon(ca), canon(cb)
    assert np.array_equal(ca["node"][oa], cb["node"][ob]) and np.array_equal(ca["partner"][oa], cb["partner"][ob])
    for k in ("pos", "vel"):
        assert np.abs(sa[k] - sb[k]).max() <= 1e-12 * np.abs(sb[k]).max(), k


def v_moved(sc, dt, steps):
    return float(np.abs(sc["vel"]).max()) * dt * steps

"""The geometry behind the support tables of the candidate separation test (CPU).

The tables (k_support_tables) bound, per cube-map cell of directions, v . p for every v in
the cell by c . p + delta |p|, with c the cell's centre direction and delta the largest
distance from c to the cell's four corner directions; and they take the maximum over the
solid's dilated grid set from its points with a 6-neighbour outside the set. Both premises
are checked here on a restatement of the mapping (same face order and gnomonic
coordinates as sup_cell_f / sup_dir): sampled directions lie within delta of their cell's
centre, and on a template's grid the boundary maximum equals the maximum over the whole
dilated set, for many directions.
"""
import numpy as np

M = 24


def sup_dir(f, p, q):
    sg = -1.0 if f & 1 else 1.0
    v = np.array([sg, p, q]) if f < 2 else (np.array([q, sg, p]) if f < 4 else np.array([p, q, sg]))
    return v / np.linalg.norm(v)


def sup_cell(u):
    a = np.abs(u)
    if a[0] >= a[1] and a[0] >= a[2]:
        f, m, p, q = (0 if u[0] >= 0 else 1), a[0], u[1], u[2]
    elif a[1] >= a[2]:
        f, m, p, q = (2 if u[1] >= 0 else 3), a[1], u[2], u[0]
    else:
        f, m, p, q = (4 if u[2] >= 0 else 5), a[2], u[0], u[1]
    i = min(max(int(np.floor((p / m + 1.0) * 0.5 * M)), 0), M - 1)
    j = min(max(int(np.floor((q / m + 1.0) * 0.5 * M)), 0), M - 1)
    return f, i, j


def cell_geometry(f, i, j):
    h = 2.0 / M
    p0, q0 = -1.0 + h * i, -1.0 + h * j
    c = sup_dir(f, p0 + 0.5 * h, q0 + 0.5 * h)
    delta = max(np.linalg.norm(sup_dir(f, p0 + h * (k & 1), q0 + h * (k >> 1)) - c) for k in range(4))
    return c, delta


def test_directions_lie_within_delta_of_their_cell_centre():
    rng = np.random.default_rng(3)
    worst = 0.0
    for u in rng.normal(size=(20000, 3)):
        u /= np.linalg.norm(u)
        c, delta = cell_geometry(*sup_cell(u))
        worst = max(worst, np.linalg.norm(u - c) / delta)
        assert np.linalg.norm(u - c) <= delta * (1 + 1e-12)
    assert worst > 0.9  # the bound is reached near the corners, so it is not loose


def test_support_over_dilated_set_is_reached_on_its_boundary():
    from conftest import load_package
    lsdem = load_package()
    from lsdem_b200 import scenes
    t = scenes.unit_templates(n_grid=16, n_nodes=200)[3]  # capsule
    nx, ny, nz = t["size"]
    phi = np.asarray(t["sdf"]).reshape(nz, ny, nx)
    m = phi <= 0
    for ax in range(3):  # dilation by one point along each axis: the 27-neighbourhood
        d = m.copy()
        a, b = [slice(None)] * 3, [slice(None)] * 3
        a[ax], b[ax] = slice(1, None), slice(None, -1)
        d[tuple(a)] |= m[tuple(b)]
        d[tuple(b)] |= m[tuple(a)]
        m = d
    pad = np.pad(m, 1)
    interior = m & pad[2:, 1:-1, 1:-1] & pad[:-2, 1:-1, 1:-1] & pad[1:-1, 2:, 1:-1] & pad[1:-1, :-2, 1:-1] \
        & pad[1:-1, 1:-1, 2:] & pad[1:-1, 1:-1, :-2]
    interior[[0, -1], :, :] = False
    interior[:, [0, -1], :] = False
    interior[:, :, [0, -1]] = False
    boundary = m & ~interior
    assert boundary.sum() < m.sum()

    def points(mask):
        z, y, x = np.nonzero(mask)
        return np.stack([t["origin"][0] + t["spacing"] * x, t["origin"][1] + t["spacing"] * y,
                         t["origin"][2] + t["spacing"] * z], 1)

    pa, pb = points(m), points(boundary)
    rng = np.random.default_rng(4)
    for u in rng.normal(size=(500, 3)):
        u /= np.linalg.norm(u)
        c, delta = cell_geometry(*sup_cell(u))
        full = (pa @ c + delta * np.linalg.norm(pa, axis=1)).max()
        edge = (pb @ c + delta * np.linalg.norm(pb, axis=1)).max()
        assert edge == full

"""The geometry behind the support tables of the candidate separation test (CPU).

The tables bound the support h(w) = max p . w of a point set along every direction from its
values at the cube map's vertex directions (+-1, p, q): h is convex, so inside each half of a
gnomonic cell it lies below the linear interpolation of its corner values. The solid's point
set is built from the SDF grid refined by two: every point where the trilinear phi is <= 0
must lie in the convex hull of the set, and the largest projection of the set must be reached
on its boundary points (the ones the host uploads). Checked here on the restatement in
support_restate.py: the interpolated bound is above the exact support for many directions and
tight to a small fraction of the body size; sampled points with phi <= 0 never project beyond
the set's support; and the boundary points reach the same support as the whole set.
"""
import numpy as np

import support_restate as sr


def _template(k=3):
    from conftest import load_package
    load_package()
    from lsdem_b200 import scenes
    return scenes.unit_templates(n_grid=16, n_nodes=200)[k]


def _phi(t, x):
    """Trilinear phi at points x (FP64, the reference's interpolation)."""
    gx, gy, gz = (int(v) for v in t["size"])
    phi = np.asarray(t["sdf"], np.float64).reshape(gz, gy, gx)
    g = (x - np.asarray(t["origin"])) / t["spacing"]
    i = np.clip(np.floor(g).astype(int), 0, [gx - 2, gy - 2, gz - 2])
    f = g - i
    out = 0.0
    for k in range(8):
        dx, dy, dz = k & 1, (k >> 1) & 1, k >> 2
        w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2])
        out = out + w * phi[i[:, 2] + dz, i[:, 1] + dy, i[:, 0] + dx]
    return out


def test_interpolated_bound_is_above_the_support():
    t = _template(0)
    rng = np.random.default_rng(3)
    for pts in (np.asarray(t["nodes"]), sr.solid_points(t)):
        tab = sr.vertex_table(pts)
        rad = np.linalg.norm(pts, axis=1).max()
        worst = 0.0
        for u in rng.normal(size=(4000, 3)):
            H, m = sr.sup_bound_exact(tab, u)
            bound = H * m / np.linalg.norm(u)
            exact = (pts @ (u / np.linalg.norm(u))).max()
            assert bound >= exact - 1e-15 * rad
            worst = max(worst, (bound - exact) / rad)
        assert worst < 2e-2  # second-order in the cell size: far tighter than a cone bound


def test_points_with_nonpositive_phi_lie_within_the_solid_set():
    for k in range(4):
        t = _template(k)
        P = sr.lattice_points(t, sr.refined_solid_mask(t))
        o = np.asarray(t["origin"])
        hi = o + t["spacing"] * (np.asarray(t["size"]) - 1)
        rng = np.random.default_rng(10 + k)
        x = o + (hi - o) * rng.random((200000, 3))
        solid = x[_phi(t, x) <= 0.0]
        assert len(solid) > 1000
        W = rng.normal(size=(300, 3))
        W /= np.linalg.norm(W, axis=1)[:, None]
        sup = (P @ W.T).max(0)
        assert np.all((solid @ W.T).max(0) <= sup + 1e-15)


def test_support_over_refined_set_is_reached_on_its_boundary():
    t = _template(3)  # capsule
    m = sr.refined_solid_mask(t)
    b = sr.boundary(m)
    assert b.sum() < m.sum()
    pa, pb = sr.lattice_points(t, m), sr.lattice_points(t, b)
    W = np.random.default_rng(4).normal(size=(500, 3))
    assert np.array_equal((pa @ W.T).max(0), (pb @ W.T).max(0))

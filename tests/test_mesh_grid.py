"""Level-set grid generation against the reference's own generator (CPU).

tests/golden/mesh_grid.npz holds the output of the reference's host header
FunDEM/kernel/helper/LevelSetObjectGenerator.h (run by
tests/golden/make_mesh_grid_golden.py): superellipsoid meshes
(LevelSetObject::Superellipsoid), their analytic grids (F / |grad F|), and mesh
grids (TriangleMeshParticle: nearest-triangle distance with the solid-angle sign,
:122-224, 454-500, 758-802) including a non-convex torus.

Checked here: the superellipsoid mesh construction restated in scenes.py (same
triangles, vertices to 1 ulp), the grid box rule of the C ABI (bit-exact), the
oracle's mesh grid (bit-exact) and the analytic grid restatement (1e-12
relative). The device builder is checked in test_gpu_mesh_grid.py.
"""
import numpy as np
import pytest

from conftest import ROOT

G = np.load(ROOT / "tests" / "golden" / "mesh_grid.npz")
SUPER = ("super_p4", "super_mixed", "ellipsoid")
CASES = SUPER + ("torus",)


@pytest.mark.parametrize("case", SUPER)
def test_superellipsoid_mesh_matches_reference(lsdem, case):
    from lsdem_b200 import scenes
    rx, ry, rz, ee, en, level, _, _ = G[f"{case}_params"]
    v, f = scenes.superellipsoid_mesh((rx, ry, rz), ee, en, int(level))
    assert np.array_equal(f, G[f"{case}_tris"])
    assert np.abs(v - G[f"{case}_verts"]).max() <= 4e-16 * max(rx, ry, rz)


@pytest.mark.parametrize("case", CASES)
def test_grid_box_matches_reference(lsdem, case):
    h = float(G[f"{case}_mesh_h"])
    pad = int(G[f"{case}_params"][-1])
    origin, size = lsdem.mesh_grid_box(G[f"{case}_verts"], h, pad)
    assert np.array_equal(origin, G[f"{case}_mesh_origin"]) and np.array_equal(size, G[f"{case}_mesh_size"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_mesh_grid_matches_reference(ora, case):
    ref = G[f"{case}_mesh"]
    out = ora.mesh_grid(G[f"{case}_verts"], G[f"{case}_tris"], G[f"{case}_mesh_origin"], G[f"{case}_mesh_size"],
                        float(G[f"{case}_mesh_h"]))
    assert np.array_equal(out, ref)
    assert (ref < 0).sum() > 100 and (ref > 0).sum() > 100


@pytest.mark.parametrize("case", SUPER)
def test_analytic_superellipsoid_grid_matches_reference(lsdem, case):
    from lsdem_b200 import scenes
    rx, ry, rz, ee, en, _, h, _ = G[f"{case}_params"]
    pts = scenes.grid_points(G[f"{case}_analytic_size"], G[f"{case}_analytic_origin"], h)
    F, g = scenes.superellipsoid_value_gradient(pts, (rx, ry, rz), ee, en)
    gn = np.sqrt(g[:, 0] ** 2 + g[:, 1] ** 2 + g[:, 2] ** 2)
    got = np.where(gn > 1e-12, F / np.maximum(gn, 1e-300), np.where(F <= 0, -0.5 * h, 0.5 * h))
    ref = G[f"{case}_analytic"]
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) <= 1e-12


def test_mesh_grid_rejects_invalid_mesh(lsdem):
    # the reference's TriangleMeshParticle::isValid (LevelSetObjectGenerator.h:872-886): no grid
    v = G["ellipsoid_verts"]
    t = G["ellipsoid_tris"].copy()
    for bad in (np.array([[0, 0, 1]]), np.array([[0, 1, len(v)]]), np.array([[-1, 1, 2]])):
        with pytest.raises(lsdem.LSDEMError):
            lsdem.mesh_grid(v, np.concatenate([t, bad]), 0.1)
    with pytest.raises(lsdem.LSDEMError):
        lsdem.mesh_grid_box(v[:0], 0.1)

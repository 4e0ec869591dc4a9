"""Synthetic level-set scenes (seeded) for tests and benchmarks.

No public dataset is involved: every scene is generated from a seed. Shapes are
SDF grids with a uniform spacing and surface nodes, in the data layout of the
reference solver (grid index ix + nx*(iy + ny*iz), phi < 0 inside; walls have
phi > 0 on the free side), built with published methods:

* exact point-ellipsoid distance by the bisection method of D. Eberly,
  "Distance from a Point to an Ellipse, an Ellipsoid, or a Hyperellipsoid" (2013);
* surface nodes from a Fibonacci sphere projected radially onto the surface
  (the same radial-projection idea as the reference's node generator,
  FunDEM/kernel/helper/LevelSetObjectGenerator.h:1013-1044);
* grid padding of two spacings around the body (LevelSetObjectGenerator.h:122-145);
* uniform random rotations by K. Shoemake's method, as the reference tutorials
  (FunDEM/apps/tutorial/tutorial1-LSParticleFalling.cpp:7-24);
* base seed 12345 (SpherePackingGenerator.h:80 default), per-config streams.
"""
from __future__ import annotations

import math
import struct

import numpy as np

# ---------------------------------------------------------------------------
# Shapes


def _eberly_root3(r0, r1, z0, z1, z2, g, iters=90):
    n0 = r0 * z0
    n1 = r1 * z1
    s0 = z2 - 1.0
    s1 = np.where(g < 0, 0.0, np.sqrt(n0 * n0 + n1 * n1 + z2 * z2) - 1.0)
    s = np.zeros_like(z0)
    for _ in range(iters):
        s = 0.5 * (s0 + s1)
        ratio0 = n0 / (s + r0)
        ratio1 = n1 / (s + r1)
        ratio2 = z2 / (s + 1.0)
        gg = ratio0 * ratio0 + ratio1 * ratio1 + ratio2 * ratio2 - 1.0
        s0 = np.where(gg > 0, s, s0)
        s1 = np.where(gg > 0, s1, s)
    return s


def ellipsoid_distance(p, axes):
    """Signed distance from points p (N,3) to the ellipsoid with semi-axes `axes` (negative inside).

    Eberly's method in the first octant with sorted axes e0 >= e1 >= e2; coordinates are floored
    at 1e-12 * e0 so that points on a symmetry plane use the general branch (distance error < 1e-12 e0)."""
    p = np.asarray(p, np.float64)
    ax = np.asarray(axes, np.float64)
    order = np.argsort(-ax)
    e0, e1, e2 = ax[order]
    y = np.maximum(np.abs(p[:, order]), 1e-12 * e0)
    y0, y1, y2 = y[:, 0], y[:, 1], y[:, 2]
    z0, z1, z2 = y0 / e0, y1 / e1, y2 / e2
    g = z0 * z0 + z1 * z1 + z2 * z2 - 1.0
    r0 = (e0 / e2) ** 2
    r1 = (e1 / e2) ** 2
    sbar = _eberly_root3(r0, r1, z0, z1, z2, g)
    x = np.stack([r0 * y0 / (sbar + r0), r1 * y1 / (sbar + r1), y2 / (sbar + 1.0)], 1)
    d = np.linalg.norm(y - x, axis=1)
    return np.where(g < 0, -d, d)


def fibonacci_directions(n):
    k = np.arange(n, dtype=np.float64) + 0.5
    z = 1.0 - 2.0 * k / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = k * math.pi * (3.0 - math.sqrt(5.0))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)


def grid_for(half_extent, n, pad=2):
    """Cubic-spacing grid of n nodes per axis covering +-half_extent (max axis) with `pad` spacings."""
    hmax = float(np.max(half_extent))
    h = 2.0 * hmax / (n - 1 - 2 * pad)
    origin = -0.5 * (n - 1) * h * np.ones(3)
    return h, origin


def grid_points(size, origin, h):
    nx, ny, nz = size
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pts = np.stack([origin[0] + x * h, origin[1] + y * h, origin[2] + z * h], -1).reshape(-1, 3)
    return pts  # index ix + nx*(iy + ny*iz)


def make_ellipsoid(axes, n_grid=32, n_nodes=1000, pad=2):
    axes = np.asarray(axes, np.float64)
    h, origin = grid_for(axes, n_grid, pad)
    size = np.array([n_grid] * 3, np.int32)
    sdf = ellipsoid_distance(grid_points(size, origin, h), axes)
    u = fibonacci_directions(n_nodes)
    t = 1.0 / np.sqrt((u[:, 0] / axes[0]) ** 2 + (u[:, 1] / axes[1]) ** 2 + (u[:, 2] / axes[2]) ** 2)
    nodes = u * t[:, None]
    return {"nodes": nodes, "sdf": sdf, "size": size, "origin": origin, "spacing": h, "bound": float(axes.max())}


def superellipsoid_value_gradient(p, axes, ee, en):
    """Implicit function F = (|x/rx|^(2/ee) + |y/ry|^(2/ee))^(ee/en) + |z/rz|^(2/en) - 1 and its
    gradient, as the reference's superellipsoid generator evaluates them
    (FunDEM/kernel/helper/LevelSetObjectGenerator.h:1264-1341: |v|^e by pow, magnitudes floored
    at 1e-30 in the derivatives, sign(0) = +1)."""
    p = np.asarray(p, np.float64)
    rx, ry, rz = (float(a) for a in axes)
    exy, ez, outer = 2.0 / ee, 2.0 / en, ee / en
    ax, ay, az = np.abs(p[:, 0] / rx), np.abs(p[:, 1] / ry), np.abs(p[:, 2] / rz)
    sxy = ax ** exy + ay ** exy
    F = sxy ** outer + az ** ez - 1.0
    tiny = 1e-30
    sgn = lambda v: np.where(v >= 0.0, 1.0, -1.0)
    o1 = np.maximum(sxy, tiny) ** (outer - 1.0)
    gx = outer * o1 * exy * np.maximum(ax, tiny) ** (exy - 1.0) * sgn(p[:, 0]) / rx
    gy = outer * o1 * exy * np.maximum(ay, tiny) ** (exy - 1.0) * sgn(p[:, 1]) / ry
    gz = ez * np.maximum(az, tiny) ** (ez - 1.0) * sgn(p[:, 2]) / rz
    return F, np.stack([gx, gy, gz], 1)


def make_superellipsoid(axes, ee, en, n_grid=64, n_nodes=1500, pad=2):
    """Superellipsoid template with the reference generator's grid values: F / |grad F| at each
    grid node, or -+h/2 where |grad F| <= 1e-12 (LevelSetObjectGenerator.h:185-205). Surface
    nodes: Fibonacci directions u scaled onto the surface in closed form, t = S(u)^(-en/2) with
    S(u) = (|ux/rx|^(2/ee) + |uy/ry|^(2/ee))^(ee/en) + |uz/rz|^(2/en), the radial projection the
    generator applies to its mesh vertices (LevelSetObjectGenerator.h:1013-1044). A single
    exponent p for all axes is ee = en = 2/p."""
    axes = np.asarray(axes, np.float64)
    h, origin = grid_for(axes, n_grid, pad)
    size = np.array([n_grid] * 3, np.int32)
    F, g = superellipsoid_value_gradient(grid_points(size, origin, h), axes, ee, en)
    gn = np.sqrt(g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1] + g[:, 2] * g[:, 2])
    sdf = np.where(gn > 1e-12, F / np.maximum(gn, 1e-300), np.where(F <= 0.0, -0.5 * h, 0.5 * h))
    u = fibonacci_directions(n_nodes)
    exy, ez, outer = 2.0 / ee, 2.0 / en, ee / en
    S = (np.abs(u[:, 0] / axes[0]) ** exy + np.abs(u[:, 1] / axes[1]) ** exy) ** outer + np.abs(u[:, 2] / axes[2]) ** ez
    nodes = u * (S ** (-0.5 * en))[:, None]
    return {"nodes": nodes, "sdf": sdf, "size": size, "origin": origin, "spacing": h,
            "bound": float(np.max(np.linalg.norm(nodes, axis=1)))}


# The 12 vertices (before normalisation) and 20 faces of the regular icosahedron in the
# numbering of the common icosphere construction, which the reference's superellipsoid
# generator also uses (LevelSetObjectGenerator.h:1069-1118); the same numbering is kept so
# that meshes come out vertex for vertex as the reference's.
_GR = 0.5 * (1.0 + math.sqrt(5.0))
_ICO_V = [(-1.0, _GR, 0.0), (1.0, _GR, 0.0), (-1.0, -_GR, 0.0), (1.0, -_GR, 0.0),
          (0.0, -1.0, _GR), (0.0, 1.0, _GR), (0.0, -1.0, -_GR), (0.0, 1.0, -_GR),
          (_GR, 0.0, -1.0), (_GR, 0.0, 1.0), (-_GR, 0.0, -1.0), (-_GR, 0.0, 1.0)]
_ICO_F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
          (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
          (6, 2, 10), (8, 6, 7), (9, 8, 1)]


def _normalize_rows(v):
    l2 = v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]
    inv = np.where(np.abs(l2) <= 1e-20, 0.0, 1.0 / np.sqrt(np.where(l2 > 0, l2, 1.0)))
    return v * inv[:, None]


def _orient_outward(v, f):
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    centre = (a + b + c) * (1.0 / 3.0)
    n = np.cross(b - a, c - a)
    flip = (n * centre).sum(1) < 0.0
    f[flip] = f[flip][:, [0, 2, 1]]
    return f


def superellipsoid_mesh(axes, ee, en, level=4):
    """Closed triangle mesh of the superellipsoid (|x/rx|^(2/ee) + |y/ry|^(2/ee))^(ee/en) +
    |z/rz|^(2/en) = 1 built as the reference's generator builds it
    (LevelSetObjectGenerator.h:1013-1200): icosahedron on the unit sphere, `level` midpoint
    subdivisions (each new vertex the normalised midpoint of an edge, created in triangle
    order), triangles turned to face outward after every stage, then every vertex scaled
    radially onto the surface by t = S(u)^(-en/2). Returns (vertices (n, 3), triangles (m, 3))."""
    rx, ry, rz = (float(a) for a in axes)
    v = _normalize_rows(np.array(_ICO_V, np.float64))
    f = _orient_outward(v, np.array(_ICO_F, np.int64))
    verts = [tuple(r) for r in v]
    for _ in range(max(0, min(int(level), 8))):
        cache = {}
        out = np.empty((4 * len(f), 3), np.int64)
        pend = []

        def mid(i, j):
            key = (i, j) if i < j else (j, i)
            k = cache.get(key)
            if k is None:
                k = len(verts) + len(pend)
                cache[key] = k
                pend.append(key)
            return k
        for t, (i0, i1, i2) in enumerate(f.tolist()):
            i01, i12, i20 = mid(i0, i1), mid(i1, i2), mid(i2, i0)
            out[4 * t:4 * t + 4] = ((i0, i01, i20), (i1, i12, i01), (i2, i20, i12), (i01, i12, i20))
        V = np.array(verts, np.float64)
        pa = np.array(pend, np.int64).reshape(-1, 2)
        m = _normalize_rows((V[pa[:, 0]] + V[pa[:, 1]]) * 0.5)
        verts.extend(tuple(r) for r in m)
        f = _orient_outward(np.array(verts, np.float64), out)
    V = np.array(verts, np.float64)
    l2 = V[:, 0] * V[:, 0] + V[:, 1] * V[:, 1] + V[:, 2] * V[:, 2]
    d = V * (1.0 / np.sqrt(l2))[:, None]
    exy, ez, outer = 2.0 / ee, 2.0 / en, ee / en
    S = np.power(np.power(np.abs(d[:, 0] / rx), exy) + np.power(np.abs(d[:, 1] / ry), exy), outer) + \
        np.power(np.abs(d[:, 2] / rz), ez)
    V = d * np.power(S, -0.5 * en)[:, None]
    f = _orient_outward(V, f)
    return V, f.astype(np.int32)


def make_mesh_template(lsdem, verts, tris, spacing, n_nodes_dirs=None, nodes=None, pad=2, device=0):
    """Template from a closed triangle mesh: the level-set grid computed on the GPU by the
    reference's buildGrid rule (lsdem.mesh_grid) and the given surface nodes."""
    sdf, size, origin = lsdem.mesh_grid(verts, tris, spacing, pad=pad, device=device)
    return {"nodes": np.asarray(nodes, np.float64), "sdf": sdf, "size": size, "origin": origin,
            "spacing": float(spacing), "verts": np.asarray(verts), "tris": np.asarray(tris),
            "bound": float(np.max(np.linalg.norm(nodes, axis=1)))}


def superellipsoid_nodes(axes, ee, en, n_nodes):
    """Fibonacci directions scaled radially onto the superellipsoid surface (closed form)."""
    u = fibonacci_directions(n_nodes)
    exy, ez, outer = 2.0 / ee, 2.0 / en, ee / en
    S = (np.abs(u[:, 0] / axes[0]) ** exy + np.abs(u[:, 1] / axes[1]) ** exy) ** outer + \
        np.abs(u[:, 2] / axes[2]) ** ez
    return u * (S ** (-0.5 * en))[:, None]


def _surface_along_rays(f, u, rmax, iters=60):
    lo = np.zeros(len(u))
    hi = np.full(len(u), rmax)
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        inside = f(u * mid[:, None]) < 0
        lo = np.where(inside, mid, lo)
        hi = np.where(inside, hi, mid)
    return u * (0.5 * (lo + hi))[:, None]


def make_from_sdf(f, half_extent, n_grid, n_nodes, pad=2, exact=True, surf_samples=200_000):
    """Template from a signed distance (exact=True) or an inside-outside function (exact=False,
    distance then measured to a dense surface sample, sign from f)."""
    h, origin = grid_for(np.asarray(half_extent), n_grid, pad)
    size = np.array([n_grid] * 3, np.int32)
    pts = grid_points(size, origin, h)
    rmax = 2.0 * float(np.linalg.norm(half_extent))
    if exact:
        sdf = f(pts)
    else:
        from scipy.spatial import cKDTree

        surf = _surface_along_rays(f, fibonacci_directions(surf_samples), rmax)
        d, _ = cKDTree(surf).query(pts)
        sdf = np.where(f(pts) < 0, -d, d)
    nodes = _surface_along_rays(f, fibonacci_directions(n_nodes), rmax)
    return {"nodes": nodes, "sdf": sdf, "size": size, "origin": origin, "spacing": h,
            "bound": float(np.max(np.linalg.norm(nodes, axis=1)))}


def superquadric_fn(axes, eps):
    """Inside-outside function of |x/a|^p + |y/b|^p + |z/c|^p = 1 with p = eps (negative inside)."""
    a, b, c = axes

    def f(p):
        v = np.abs(p[:, 0] / a) ** eps + np.abs(p[:, 1] / b) ** eps + np.abs(p[:, 2] / c) ** eps
        return v ** (1.0 / eps) - 1.0
    return f


def rounded_box_sdf(half, r):
    half = np.asarray(half, np.float64)

    def f(p):
        q = np.abs(p) - (half - r)
        return np.linalg.norm(np.maximum(q, 0.0), axis=1) + np.minimum(np.max(q, axis=1), 0.0) - r
    return f


def capsule_sdf(half_len, r):
    def f(p):
        z = np.clip(p[:, 2], -half_len, half_len)
        d = p - np.stack([np.zeros_like(z), np.zeros_like(z), z], 1)
        return np.linalg.norm(d, axis=1) - r
    return f


def make_plane_wall(extent_xy, h=None):
    """Floor wall: phi = z (free side above). Grid 5 x 5 x 3 with spacing `h` (phi linear -> exact)."""
    h = h or 0.5 * float(max(extent_xy))
    size = np.array([5, 5, 3], np.int32)
    origin = np.array([-2 * h, -2 * h, -h])
    sdf = grid_points(size, origin, h)[:, 2].copy()
    ex, ey = 0.5 * extent_xy[0], 0.5 * extent_xy[1]
    verts = np.array([[-ex, -ey, 0.0], [ex, -ey, 0.0], [ex, ey, 0.0], [-ex, ey, 0.0]])
    return {"verts": verts, "sdf": sdf, "size": size, "origin": origin, "spacing": h}


# ---------------------------------------------------------------------------
# Placement helpers


def random_quaternions(rng, n):
    """Uniform random unit quaternions (Shoemake), q0 scalar first."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    s1, s2 = np.sqrt(1.0 - u1), np.sqrt(u1)
    a, b = 2.0 * math.pi * u2, 2.0 * math.pi * u3
    return np.stack([s2 * np.cos(b), s1 * np.sin(a), s1 * np.cos(a), s2 * np.sin(b)], 1)


def rsa_positions(rng, n, radii, lo, hi, max_tries=200, periodic=False, placed_out=None):
    """Random sequential addition of non-overlapping spheres (radii per particle) in the box [lo, hi].
    placed_out (optional boolean array of n): a sphere that finds no room is skipped (marked
    False there, position NaN) instead of raising."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    L = hi - lo
    rmax = float(np.max(radii))
    cell = 2.0 * rmax
    dims = np.maximum(1, (L / cell).astype(int))
    grid = {}
    pos = np.zeros((n, 3))
    placed = 0
    for i in range(n):
        r = radii[i]
        for _ in range(max_tries):
            p = (lo + r + rng.random(3) * (L - 2 * r)) if not periodic else (lo + rng.random(3) * L)
            c = np.minimum(((p - lo) / cell).astype(int), dims - 1)
            ok = True
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        cc = c + (dx, dy, dz)
                        if periodic:
                            cc = cc % dims
                        for j in grid.get(tuple(cc), ()):
                            d = pos[j] - p
                            if periodic:
                                d -= L * np.round(d / L)
                            if d @ d < (r + radii[j]) ** 2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pos[i] = p
                grid.setdefault(tuple(c), []).append(i)
                placed += 1
                if placed_out is not None:
                    placed_out[i] = True
                break
        else:
            if placed_out is None:
                raise RuntimeError(f"RSA could not place particle {i} (fraction too high)")
            placed_out[i] = False
            pos[i] = np.nan
    return pos


def cluster_positions(rng, n, spacing, lo, jitter=0.0):
    """Particles on a cubic lattice with the given spacing from `lo` (row-major), optional jitter."""
    m = int(math.ceil(n ** (1.0 / 3.0)))
    idx = np.arange(n)
    ijk = np.stack([idx % m, (idx // m) % m, idx // (m * m)], 1).astype(np.float64)
    p = np.asarray(lo) + (ijk + 0.5) * spacing
    if jitter:
        p += rng.uniform(-jitter, jitter, size=p.shape)
    return p


# ---------------------------------------------------------------------------
# Scenes


def seed_for(config_id: int, base: int = 12345) -> int:
    """SplitMix64(base + config id)."""
    z = (base + config_id + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return int((z ^ (z >> 31)) & 0x7FFFFFFF)


def ellipsoid_falling(n=2000, axes=(5e-3, 4e-3, 3e-3), n_grid=32, n_nodes=1000, box=(0.2, 0.2, 0.4), seed=None,
                      kn=1e5, kt_ratio=0.8, mu=0.5, e=0.6, density=2500.0, dt=1e-6, fraction_z=1.0,
                      packing="rsa", vel_sigma=0.0):
    """Identical ellipsoids at seeded non-overlapping positions above a floor wall (gravity -z).

    Defaults are the small plain-method workload: 2,000 ellipsoids (5, 4, 3 mm), 32^3 FP64 SDF from the
    exact ellipsoid distance, 1,000 Fibonacci surface nodes, 0.2 x 0.2 x 0.4 m box, kn = 1e5 N/m,
    kt = 0.8 kn, mu = 0.5, e = 0.6, 2500 kg/m^3, dt = 1e-6 s."""
    rng = np.random.default_rng(seed_for(0) if seed is None else seed)
    shp = make_ellipsoid(axes, n_grid, n_nodes)
    r = float(np.max(axes))
    box = np.asarray(box, np.float64)
    hi = np.array([box[0], box[1], box[2] * fraction_z])
    if packing == "rsa":
        pos = rsa_positions(rng, n, np.full(n, r), np.zeros(3), hi)
    else:
        pos = cluster_positions(rng, n, packing, np.full(3, r))
    quat = random_quaternions(rng, n)
    vel = rng.normal(0.0, vel_sigma, size=(n, 3)) if vel_sigma else np.zeros((n, 3))
    floor = make_plane_wall(box[:2])
    return {"shape": shp, "pos": pos, "quat": quat, "vel": vel, "kn": kn, "ks": kt_ratio * kn, "mu": mu, "e": e,
            "density": density, "dt": dt, "min": np.zeros(3), "max": box, "gravity": np.array([0.0, 0.0, -9.81]),
            "floor": floor}


def load_into(solver, scene, walls=True):
    """Adds a scene built by ellipsoid_falling() to a Solver through the density path (addLSParticle)."""
    s = scene["shape"]
    n = len(scene["pos"])
    vel = scene.get("vel", np.zeros((n, 3)))
    for i in range(n):
        solver.add_ls_particle(s["nodes"], s["sdf"], s["size"], s["origin"], s["spacing"], scene["pos"][i], vel[i],
                               np.zeros(3), scene["quat"][i], scene["kn"], scene["ks"], scene["mu"], scene["e"],
                               scene["density"])
    if walls and scene.get("floor") is not None:
        f = scene["floor"]
        cx, cy = 0.5 * (scene["min"][0] + scene["max"][0]), 0.5 * (scene["min"][1] + scene["max"][1])
        solver.add_wall(f["verts"], f["sdf"], f["size"], f["origin"], f["spacing"], [cx, cy, scene["min"][2]],
                        [1.0, 0.0, 0.0, 0.0], scene["mu"], scene["e"])


# ---------------------------------------------------------------------------
# Polydisperse multi-template scenes (precision-form workload)


def unit_templates(n_grid=48, n_nodes=2000):
    """The four templates of the precision-form workload, each scaled to a bounding
    diameter of 1 (so a particle of bounding diameter d uses scale d):
    ellipsoid 1:0.8:0.6, superquadric |x|^4+|y|^4+|z|^4 = 1, cube with edge radius
    0.1 of the side, capsule of aspect ratio 2 (length = 2 x diameter)."""
    out = []
    # ellipsoid, exact distance
    ax = np.array([0.5, 0.4, 0.3])
    out.append(make_ellipsoid(ax, n_grid, n_nodes))
    # superquadric exponent 4: max radius at the diagonal, 3^(1/4) * half-size
    hs = 0.5 / 3 ** 0.25
    out.append(make_from_sdf(superquadric_fn((hs, hs, hs), 4.0), np.array([hs, hs, hs]), n_grid, n_nodes,
                             exact=False))
    # rounded cube: side s, edge radius 0.1 s, bounding radius sqrt(3)(s/2 - r) + r = 0.5
    s = 1.0 / (np.sqrt(3.0) * 0.8 + 0.2)
    out.append(make_from_sdf(rounded_box_sdf([s / 2] * 3, 0.1 * s), np.array([s / 2] * 3), n_grid, n_nodes))
    # capsule: radius r, half length of the axis segment r (total length 4r = 2 x diameter), bounding radius 2r = 0.5
    r = 0.25
    out.append(make_from_sdf(capsule_sdf(r, r), np.array([r, r, 2 * r]), n_grid, n_nodes))
    for t in out:
        t["bound"] = float(np.max(np.linalg.norm(t["nodes"], axis=1)))
    return out


def polydisperse_periodic(lsdem, n=100_000, box=0.1, median=2e-3, sigma=0.25, n_grid=48, n_nodes=2000, seed=None,
                          vel_sigma=0.1, kn=1e5, kt_ratio=0.8, mu=0.5, e=0.6, density=2500.0, dt=5e-7, exclusion=0.8,
                          templates=None):
    """Precision-form workload: n particles from the four unit templates, log-normal bounding
    diameters (median 2 mm, sigma 0.25), in a triply periodic cube of side `box`, velocities
    N(0, 0.1 m/s) per component, linear contact as the small workload, dt = 5e-7 s.

    Positions come from random sequential addition of spheres of `exclusion` x the bounding
    radius (largest first): at this count the bounding spheres alone fill more than half of
    the box, beyond any sequential packing, so bounding spheres may overlap by up to 20 %
    while the non-spherical bodies themselves mostly stay apart.

    Returns a dict with the per-template data and per-particle arrays ready for
    Solver.add_shape / Solver.add_particles (frame moved to each template's centroid,
    mass and inertia scaled from the unit-density template integrals)."""
    rng = np.random.default_rng(seed_for(1) if seed is None else seed)
    T = templates or unit_templates(n_grid, n_nodes)
    d = median * np.exp(sigma * rng.standard_normal(n))
    order = np.argsort(-d)
    d = d[order]
    shape = rng.integers(0, len(T), size=n).astype(np.int32)
    pos = lsdem.pack_rsa(0.5 * exclusion * d, np.zeros(3), np.full(3, box), periodic=True,
                         seed=int(rng.integers(1 << 62)))
    quat = random_quaternions(rng, n)
    vel = rng.normal(0.0, vel_sigma, size=(n, 3))
    tm = []
    for t in T:
        mp = lsdem.mass_properties(t["sdf"], t["size"], t["origin"], t["spacing"], 1.0)
        c = mp["centroid"]
        tm.append({"nodes": t["nodes"] - c, "sdf": t["sdf"], "size": t["size"], "origin": t["origin"] - c,
                   "spacing": t["spacing"], "mass": mp["mass"], "inv_inertia": mp["inv_inertia"]})
    m1 = np.array([t["mass"] for t in tm])[shape]
    iI = np.array([t["inv_inertia"] for t in tm])[shape]
    inv_mass = 1.0 / (density * m1 * d ** 3)
    inv_inertia = iI / (density * d[:, None] ** 5)
    return {"templates": tm, "shape": shape, "scale": d, "pos": pos, "quat": quat, "vel": vel,
            "inv_mass": inv_mass, "inv_inertia": inv_inertia, "kn": kn, "ks": kt_ratio * kn, "mu": mu, "e": e,
            "dt": dt, "min": np.zeros(3), "max": np.full(3, box), "gravity": np.zeros(3), "periodic": 7}


def resolve_deep_overlaps(lsdem, sc, threshold=0.02, exclusion=0.8, max_iter=40, device=0, seed=None):
    """Re-places particles whose body overlaps a neighbour by more than `threshold` x the
    smaller bounding radius, until none does (shallow contacts stay).

    The reference's contact law applies the normal stiffness once per surface node inside the
    partner, so a deep initial overlap (many nodes inside) multiplies the contact stiffness and
    can exceed the stability limit of the explicit step. Overlaps are measured by the solver's
    own detection (one step of 1e-12 s from rest); the re-placed particles get new random
    positions (sequential addition around the others, spheres of `exclusion` x the bounding
    radius) and orientations. Updates sc["pos"] and sc["quat"] in place; returns the number of
    iterations."""
    rng = np.random.default_rng(seed_for(7) if seed is None else seed)
    n = len(sc["pos"])
    rest = dict(sc, vel=np.zeros((n, 3)))
    sv = lsdem.Solver(device=device)
    load_polydisperse(sv, rest)
    sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    pp = sv.particle_params()
    radius = pp["radius"]
    nb = np.concatenate([pp["node_base"], [np.iinfo(np.int64).max]])
    zero = np.zeros((n, 3))
    it = 0
    for it in range(1, max_iter + 1):
        sv.set_state(pos=sc["pos"], vel=zero, angvel=zero, quat=sc["quat"])
        sv.step(1e-12, 1)
        bad = set()
        for kind in (lsdem.CONTACT_PARTICLE, lsdem.CONTACT_GHOST):
            c = sv.contacts(kind, geometry=True)
            if len(c["node"]) == 0:
                continue
            owner = np.searchsorted(nb, c["node"], side="right") - 1
            partner = c["partner"]
            rmin = np.minimum(radius[owner], radius[partner])
            deep = c["overlap"] > threshold * rmin
            if kind == lsdem.CONTACT_GHOST:
                deep &= owner != partner
            bad.update(np.maximum(owner[deep], partner[deep]).tolist())
        if not bad:
            break
        bad = np.fromiter(bad, np.int64)
        keep = np.ones(n, np.int32)
        keep[bad] = 0
        if "rsa" in sc:
            # scenes with their own packing spec: re-placed with the same spheres; when no room is
            # left (or in the last pass) the remaining bodies go to the spec's reserve box, where
            # their bounding spheres do not overlap each other or the packing
            rsa = sc["rsa"]
            placed = False
            if it < max_iter:
                try:
                    sc["pos"] = _rsa(lsdem, rng, rsa, keep=keep, pos=sc["pos"])
                    placed = True
                except Exception:
                    placed = False
            if not placed:
                if "reserve_lo" not in rsa:
                    raise RuntimeError("resolve_deep_overlaps: no room to re-place overlapping bodies")
                res = {"radius": rsa["bound"][bad], "lo": rsa["reserve_lo"], "hi": rsa["reserve_hi"], "periodic": False}
                sc["pos"][bad] = _rsa(lsdem, rng, res)
                sc["quat"][bad] = random_quaternions(rng, len(bad))
                sc["reserve_placed"] = int(len(bad))
                break
        else:
            # re-placed spheres may come a little closer than the first packing (0.75 x radius)
            rad = 0.5 * exclusion * sc["scale"]
            rad = np.where(keep == 0, rad * (0.75 / exclusion), rad)
            sc["pos"] = lsdem.pack_rsa(rad, sc["min"], sc["max"], periodic=bool(sc["periodic"]),
                                       seed=int(rng.integers(1 << 62)), max_tries=20000, keep=keep, pos=sc["pos"])
        sc["quat"][bad] = random_quaternions(rng, len(bad))
    sv.close()
    return it


def load_polydisperse(solver, sc):
    """Adds a multi-template scene (this module's scene dicts) to a Solver: shapes, particles,
    walls with their prescribed motion, bonds and the periodic axes."""
    ids = [solver.add_shape(t["nodes"], t["sdf"], t["size"], t["origin"], t["spacing"]) for t in sc["templates"]]
    shape = np.asarray(ids, np.int32)[sc["shape"]]
    solver.add_particles(shape, sc["pos"], sc["quat"], sc["inv_mass"], sc["inv_inertia"], sc["kn"], sc["ks"],
                         sc["mu"], sc["e"], vel=sc["vel"], angvel=sc.get("angvel"), scale=sc["scale"])
    for w in sc.get("walls", ()):
        k = solver.add_wall(w["verts"], w["sdf"], w["size"], w["origin"], w["spacing"], w["pos"], w["quat"], w["mu"],
                            w["e"])
        if w.get("vel") is not None:
            solver.set_wall_velocity(k, w["vel"])
        if w.get("angvel") is not None:
            solver.set_wall_angular_velocity(k, w["angvel"])
    b = sc.get("bonds")
    if b is not None:
        for k in range(len(b["master"])):
            solver.add_bond(int(b["master"][k]), int(b["slave"][k]), b["point"][k], b["normal"][k], b["radius"][k],
                            b["length"][k], b["youngs"], b["poisson"], b["tensile"][k], b["cohesion"][k], b["mu"])
    solver.set_periodic(sc["periodic"])


# ---------------------------------------------------------------------------
# Bonded, drum and large-scale workloads


def _unit_density_templates(lsdem, T, gpu=False):
    """Mass (= volume at density 1), inverse inertia and the frame moved to the centroid, from
    each template's grid by the reference's smoothed-Heaviside integration (LSSolver.h:66-135),
    on the host or (gpu=True, for the large template sets) on the GPU."""
    out = []
    mp_fn = lsdem.mass_properties_gpu if gpu else lsdem.mass_properties
    for t in T:
        mp = mp_fn(t["sdf"], t["size"], t["origin"], t["spacing"], 1.0)
        c = mp["centroid"]
        out.append({"nodes": t["nodes"] - c, "sdf": t["sdf"], "size": t["size"], "origin": t["origin"] - c,
                    "spacing": t["spacing"], "mass": mp["mass"], "inv_inertia": mp["inv_inertia"],
                    "bound": float(np.max(np.linalg.norm(t["nodes"] - c, axis=1)))})
    return out


def _rsa(lsdem, rng, rsa, keep=None, pos=None, max_tries=20000):
    """Random sequential addition of the spheres of an "rsa" spec (radius per particle, box lo/hi,
    periodic flag), largest first."""
    r = np.asarray(rsa["radius"], np.float64)
    order = np.argsort(-r, kind="stable")
    out = np.empty((len(r), 3))
    kp = None if keep is None else np.asarray(keep)[order]
    p0 = None if pos is None else np.asarray(pos)[order]
    out[order] = lsdem.pack_rsa(r[order], rsa["lo"], rsa["hi"], periodic=rsa["periodic"],
                                seed=int(rng.integers(1 << 62)), max_tries=max_tries, keep=kp, pos=p0)
    return out


def _body_arrays(tm, shape, scale, density):
    m1 = np.array([t["mass"] for t in tm])[shape]
    iI = np.array([t["inv_inertia"] for t in tm])[shape]
    return 1.0 / (density * m1 * scale ** 3), iI / (density * scale[:, None] ** 5)


def plane_wall(extent, pos, up=True, mu=0.5, e=0.6, h=2e-3):
    """Flat wall at `pos` covering a square of side 2 x extent around it, free side above
    (up=True) or below (turned by a half turn about x). phi = z on a grid of spacing `h`
    (2 mm) five nodes deep (|z| <= 2h): phi is linear, so the grid is exact at any spacing,
    and a fine spacing keeps the 16-bit copy of phi / h precise in absolute terms (its
    certified error band is a fixed fraction of a spacing)."""
    m = int(math.ceil(extent / h))
    size = np.array([2 * m + 1, 2 * m + 1, 5], np.int32)
    origin = np.array([-m * h, -m * h, -2 * h])
    sdf = grid_points(size, origin, h)[:, 2].copy()
    verts = np.array([[-extent, -extent, 0.0], [extent, -extent, 0.0], [extent, extent, 0.0], [-extent, extent, 0.0]])
    return {"verts": verts, "sdf": sdf, "size": size, "origin": origin, "spacing": h,
            "pos": np.asarray(pos, np.float64), "quat": np.array([1.0, 0, 0, 0]) if up else np.array([0.0, 1, 0, 0]),
            "mu": mu, "e": e}


def drum_wall(radius, length, h, mu=0.5, e=0.6, pad=2):
    """Closed rotating-drum wall: the cavity of a cylinder of `radius` and `length` around the
    local x axis, centred at the local origin; phi is the exact distance to the cavity boundary,
    positive inside the cavity (the free side) and negative in the wall."""
    n = [int(math.ceil((0.5 * length) / h)) + pad, int(math.ceil(radius / h)) + pad, int(math.ceil(radius / h)) + pad]
    size = np.array([2 * n[0] + 1, 2 * n[1] + 1, 2 * n[2] + 1], np.int32)
    origin = -h * np.array(n, np.float64)
    p = grid_points(size, origin, h)
    rho = np.sqrt(p[:, 1] ** 2 + p[:, 2] ** 2)
    ax = np.abs(p[:, 0])
    inside = (rho < radius) & (ax < 0.5 * length)
    out = np.sqrt(np.maximum(rho - radius, 0.0) ** 2 + np.maximum(ax - 0.5 * length, 0.0) ** 2)
    sdf = np.where(inside, np.minimum(radius - rho, 0.5 * length - ax), -out)
    a = 2 * math.pi * np.arange(32) / 32
    ring = np.stack([np.zeros(32), radius * np.cos(a), radius * np.sin(a)], 1)
    verts = np.concatenate([ring + [-0.5 * length, 0, 0], ring + [0.5 * length, 0, 0]])
    return {"verts": verts, "sdf": sdf, "size": size, "origin": origin, "spacing": h, "mu": mu, "e": e}


def superquadric_templates(lsdem, rng, count, exponents, semi_axes, n_grid, n_nodes, level=5, pad=2, device=0):
    """`count` superquadrics |x/a|^p + |y/b|^p + |z/c|^p = 1 with p uniform in `exponents` and
    a, b, c uniform in `semi_axes`. Each grid is the mesh distance of the shape's subdivided
    icosphere mesh (superellipsoid_mesh, `level` subdivisions: 20 x 4^level triangles), computed
    on the GPU by the reference's buildGrid rule with a spacing that puts about n_grid nodes
    along the longest axis; the surface nodes are Fibonacci directions scaled onto the surface."""
    T = []
    for p, ax in superquadric_specs(rng, count, exponents, semi_axes):
        ee = en = 2.0 / p
        v, f = superellipsoid_mesh(ax, ee, en, level)
        h = 2.0 * float(ax.max()) / (n_grid - 1 - 2 * pad)
        sdf, size, origin = lsdem.mesh_grid(v, f, h, pad=pad, device=device)
        T.append({"nodes": superellipsoid_nodes(ax, ee, en, n_nodes), "sdf": sdf, "size": size, "origin": origin,
                  "spacing": h, "exponent": p, "semi_axes": ax})
    return T


def superquadric_specs(rng, count, exponents, semi_axes):
    """Exponent and semi-axes of each of `count` seeded superquadrics (the draws of
    superquadric_templates, in its order)."""
    out = []
    for _ in range(count):
        p = float(rng.uniform(*exponents))
        ax = rng.uniform(*semi_axes, size=3)
        out.append((p, ax))
    return out


def mesh_grid_box_np(verts, spacing, pad=2):
    """Grid box of buildGrid around a mesh (LevelSetObjectGenerator.h:122-170): the vertices'
    bounding box grown by max(1, pad) spacings, snapped outward to multiples of the spacing
    (the same operations as the library's lsdem_mesh_grid_box, so the same bits)."""
    v = np.asarray(verts, np.float64).reshape(-1, 3)
    mn, mx = v.min(axis=0), v.max(axis=0)
    padding = float(max(1, pad)) * spacing
    lo = spacing * np.floor((mn - padding) / spacing)
    hi = spacing * np.ceil((mx + padding) / spacing)
    size = (np.floor((hi - lo) / spacing + 0.5) + 1).astype(np.int32)
    return lo, size


def superquadric_templates_host(grid_fn, rng, count, exponents, semi_axes, n_grid, n_nodes, level=5, pad=2):
    """superquadric_templates without the library: the same shapes (same draws of `rng`), with
    each grid from grid_fn(verts, tris, origin, size, spacing) (a host mesh-grid routine that
    computes the reference's buildGrid values, e.g. the oracle's)."""
    T = []
    for p, ax in superquadric_specs(rng, count, exponents, semi_axes):
        ee = en = 2.0 / p
        v, f = superellipsoid_mesh(ax, ee, en, level)
        h = 2.0 * float(ax.max()) / (n_grid - 1 - 2 * pad)
        origin, size = mesh_grid_box_np(v, h, pad)
        T.append({"nodes": superellipsoid_nodes(ax, ee, en, n_nodes), "sdf": grid_fn(v, f, origin, size, h),
                  "size": size, "origin": origin, "spacing": h, "exponent": p, "semi_axes": ax})
    return T


def settling_sample(mass_fn, T, n, seed, solid_fraction=0.25, kn=1e5, kt_ratio=0.8, mu=0.5, e=0.6, density=2500.0,
                    dt=5e-7, exclusion=0.85):
    """A bounded sample of the large-scale workload for host-side timing: n particles of the
    templates T (as drawn for that workload) in a box periodic in x and y with a floor and a
    ceiling, at the same solid fraction, placed by random sequential addition of spheres of
    `exclusion` x the bounding radius (this module's host RSA), random orientations, at rest.
    mass_fn(sdf, size, origin, spacing) -> (mass, centroid, inv_inertia) at density 1 (the
    reference's smoothed-Heaviside integration, LSSolver.h:66-135). Deep initial overlaps are
    not re-placed (no device is used)."""
    rng = np.random.default_rng(seed)
    tm = []
    for t in T:
        mass, c, iI = mass_fn(t["sdf"], t["size"], t["origin"], t["spacing"])
        tm.append({"nodes": t["nodes"] - c, "sdf": t["sdf"], "size": t["size"], "origin": t["origin"] - c,
                   "spacing": t["spacing"], "mass": mass, "inv_inertia": iI,
                   "bound": float(np.max(np.linalg.norm(t["nodes"] - c, axis=1)))})
    shape = rng.integers(0, len(tm), size=n).astype(np.int32)
    vol = np.array([t["mass"] for t in tm])[shape].sum()
    L = (vol / solid_fraction) ** (1.0 / 3.0)
    bound = np.array([t["bound"] for t in tm])[shape]
    b = float(bound.max())
    order = np.argsort(-bound, kind="stable")
    pos = np.empty((n, 3))
    placed = np.zeros(n, bool)
    pos[order] = rsa_positions(rng, n, exclusion * bound[order], np.array([0.0, 0.0, b]), np.array([L, L, L - b]),
                               max_tries=300, periodic=True, placed_out=placed)
    ok = np.empty(n, bool)
    ok[order] = placed
    H = L + b
    if not ok.all():
        # as the full workload: bodies that find no room go to a reserve slab above the
        # packing (bounding spheres at 20 % fraction, no overlaps)
        left = np.nonzero(~ok)[0]
        slab = len(left) * (4.0 / 3.0) * math.pi * float(np.mean(bound[left] ** 3)) / 0.2 / (L * L) + 2 * b
        pos[left] = rsa_positions(rng, len(left), bound[left], np.array([0.0, 0.0, L + b]),
                                  np.array([L, L, L + b + slab]), max_tries=20000, periodic=True)
        H = L + b + slab
    scale = np.ones(n)
    inv_mass, inv_inertia = _body_arrays(tm, shape, scale, density)
    walls = [plane_wall(L, [0.5 * L, 0.5 * L, 0.0], True, mu, e), plane_wall(L, [0.5 * L, 0.5 * L, H], False, mu, e)]
    return {"templates": tm, "shape": shape, "scale": scale, "pos": pos, "quat": random_quaternions(rng, n),
            "vel": np.zeros((n, 3)), "inv_mass": inv_mass, "inv_inertia": inv_inertia, "kn": kn, "ks": kt_ratio * kn,
            "mu": mu, "e": e, "dt": dt, "min": np.zeros(3), "max": np.array([L, L, H]),
            "gravity": np.array([0.0, 0.0, -9.81]), "periodic": 3, "walls": walls, "solid_fraction": solid_fraction}


def bonded_hcp(lsdem, n=50_000, axes=(2e-3, 1.6e-3, 1.2e-3), n_grid=32, n_nodes=1000, gap=0.05, jitter=0.02,
               bond_reach=1.1, youngs=1e8, poisson=0.3, strength_median=1e6, strength_sigma=0.3,
               wall_speed=0.1, kn=1e5, kt_ratio=0.8, mu=0.5, e=0.6, density=2500.0, dt=2e-7, seed=None):
    """Bonded workload: n identical ellipsoids (semi-axes 2, 1.6, 1.2 mm) on a jittered HCP
    lattice, bonded to every lattice neighbour, compressed by a top wall at 0.1 m/s.

    The lattice is the reference's hexagonal close packing (SpherePackingGenerator.h:486-555:
    rows shifted by r, layers by (r, r/sqrt(3))) of unit-diameter spheres at a spacing of
    (1 + gap), mapped by diag(2a, 2b, 2c): the map sends touching spheres to touching aligned
    ellipsoids, so the gap is 5 % of the contact distance along every lattice direction. Every
    centre then moves by a random vector of length up to jitter x spacing (2 %, less than the
    gap: no initial overlaps). Bonds join lattice neighbours whose centre distance in the unit
    lattice is within bond_reach (1.1) of the contact distance: bond point at the midpoint,
    normal from slave to master, length = centre distance (the reference's convention,
    tutorial3-bondedLSParticleBeam.cpp:78-86), radius = 1 x the radius of the sphere of equal
    volume (abc)^(1/3); tensile strength and cohesion log-normal (median 1e6 Pa, sigma 0.3),
    bond friction 0. Floor at z = 0, top wall above the top layer moving down at wall_speed.
    Contact law as the small workload; gravity -z."""
    rng = np.random.default_rng(seed_for(2) if seed is None else seed)
    ax = np.asarray(axes, np.float64)
    r = 0.5 * (1.0 + gap)
    m = int(round(n ** (1.0 / 3.0))) + 2
    dx, dy, dz = 2 * r, math.sqrt(3.0) * r, math.sqrt(8.0 / 3.0) * r
    pts = []
    for k in range(2 * m):
        for j in range(2 * m):
            for i in range(2 * m):
                x = i * dx + (r if j % 2 else 0.0) + (r if k % 2 else 0.0)
                y = j * dy + (r / math.sqrt(3.0) if k % 2 else 0.0)
                pts.append((x, y, k * dz))
                if len(pts) >= 8 * m ** 3:
                    break
    pts = np.array(pts)
    # a block of nx x ny x nz sites, as close to a cube in the mapped frame as n allows
    span = 2 * ax * np.array([dx, dy, dz])
    per = (n / np.prod(1.0 / span)) ** (1.0 / 3.0) / span
    nx, ny = max(2, int(round(per[0]))), max(2, int(round(per[1])))
    nz = int(math.ceil(n / (nx * ny)))
    ii = np.round((pts[:, 0] - np.where(np.round(pts[:, 1] / dy) % 2 == 1, r, 0.0)) / dx)
    jj = np.round(pts[:, 1] / dy)
    kk = np.round(pts[:, 2] / dz)
    sel = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny) & (kk >= 0) & (kk < nz)
    u = pts[sel]
    u = u[np.lexsort((u[:, 0], u[:, 1], u[:, 2]))][:n]
    d = rng.normal(size=(len(u), 3))
    d *= (rng.random(len(u)) ** (1.0 / 3.0) / np.linalg.norm(d, axis=1))[:, None]
    u = u + jitter * 2 * r * d
    from scipy.spatial import cKDTree

    pairs = cKDTree(u).query_pairs(bond_reach, output_type="ndarray")
    pos = u * (2 * ax)
    pos -= pos.min(0)
    pos += ax + 0.5 * gap * 2 * ax
    shp = make_ellipsoid(ax, n_grid, n_nodes)
    tm = _unit_density_templates(lsdem, [shp])
    nb = len(pos)
    shape = np.zeros(nb, np.int32)
    scale = np.ones(nb)
    inv_mass, inv_inertia = _body_arrays(tm, shape, scale, density)
    master, slave = pairs[:, 0], pairs[:, 1]
    dv = pos[master] - pos[slave]
    L0 = np.linalg.norm(dv, axis=1)
    nb_bonds = len(master)
    lo = np.zeros(3)
    hi = pos.max(0) + ax + 0.5 * gap * 2 * ax
    extent = float(max(hi[0], hi[1]))
    walls = [plane_wall(extent, [0.5 * hi[0], 0.5 * hi[1], 0.0], True, mu, e),
             dict(plane_wall(extent, [0.5 * hi[0], 0.5 * hi[1], hi[2]], False, mu, e),
                  vel=np.array([0.0, 0.0, -wall_speed]))]
    bonds = {"master": master.astype(np.int32), "slave": slave.astype(np.int32), "point": 0.5 * (pos[master] + pos[slave]),
             "normal": dv / L0[:, None], "length": L0, "radius": np.full(nb_bonds, float(np.prod(ax) ** (1.0 / 3.0))),
             "youngs": youngs, "poisson": poisson,
             "tensile": strength_median * np.exp(strength_sigma * rng.standard_normal(nb_bonds)),
             "cohesion": strength_median * np.exp(strength_sigma * rng.standard_normal(nb_bonds)), "mu": 0.0}
    margin = 4 * float(ax.max())
    return {"templates": tm, "shape": shape, "scale": scale, "pos": pos, "quat": np.tile([1.0, 0, 0, 0], (nb, 1)),
            "vel": np.zeros((nb, 3)), "inv_mass": inv_mass, "inv_inertia": inv_inertia, "kn": kn, "ks": kt_ratio * kn,
            "mu": mu, "e": e, "dt": dt, "min": lo - margin * np.array([1, 1, 0]),
            "max": hi + margin * np.array([1, 1, 1]), "gravity": np.array([0.0, 0.0, -9.81]), "periodic": 0,
            "walls": walls, "bonds": bonds}


def drum(lsdem, n=500_000, shapes=64, exponents=(2.0, 8.0), semi_axes=(1e-3, 3e-3), n_grid=64, n_nodes=1500,
         radius=0.15, length=0.1, rpm=30.0, fill_fraction=0.22, wall_spacing=1e-3, kn=1e5, kt_ratio=0.8, mu=0.5,
         e=0.6, density=2500.0, dt=5e-7, exclusion=0.85, seed=None, device=0, templates=None):
    """Rotating-drum workload: n particles drawn uniformly from `shapes` seeded superquadrics
    (exponents uniform 2-8, semi-axes uniform 1-3 mm, 64^3 grids from their meshes, 1500
    nodes) in a closed drum of radius 0.15 m and length 0.1 m turning at 30 rpm about its
    horizontal axis (x), gravity -z.

    The stated counts and sizes do not fit the stated drum: 500,000 such bodies hold ~0.024 m^3
    of solid, 3.4 x the drum's 7.1e-3 m^3. The drum, the count and the shape family are kept
    and every shape is scaled by one common factor so that the bodies fill the loading box (the
    part of the drum below z = 0.3 R, |y| <= 0.7 R, 5 mm clear of the end caps) at a solid
    fraction of `fill_fraction`; the factor is returned as "size_factor". Positions by random
    sequential addition of spheres of `exclusion` x the bounding radius (bounding spheres of
    these shapes hold ~2.2 x their volume, so 0.22 with exclusion 0.85 is close to the densest
    random placement without mass interpenetration), random orientations, at rest; deep overlaps
    are removed afterwards by resolve_deep_overlaps, which puts the bodies it cannot fit into
    the empty upper part of the drum."""
    rng = np.random.default_rng(seed_for(3) if seed is None else seed)
    T = templates or superquadric_templates(lsdem, rng, shapes, exponents, semi_axes, n_grid, n_nodes, device=device)
    tm = _unit_density_templates(lsdem, T, gpu=True)
    shape = rng.integers(0, len(tm), size=n).astype(np.int32)
    vol = np.array([t["mass"] for t in tm])[shape].sum()
    lo = np.array([-0.5 * length + 5e-3, -0.7 * radius, -math.sqrt(radius ** 2 - (0.7 * radius) ** 2)])
    hi = np.array([0.5 * length - 5e-3, 0.7 * radius, 0.3 * radius])
    box_vol = float(np.prod(hi - lo))
    s = (fill_fraction * box_vol / vol) ** (1.0 / 3.0)
    scale = np.full(n, s)
    bound = np.array([t["bound"] for t in tm])[shape] * s
    bm = float(bound.max())
    rsa = {"radius": exclusion * bound, "lo": lo + bm, "hi": hi - bm, "periodic": False, "bound": bound,
           "reserve_lo": np.array([lo[0] + bm, -0.5 * radius, hi[2] + bm]),
           "reserve_hi": np.array([hi[0] - bm, 0.5 * radius, 0.8 * radius])}
    pos = _rsa(lsdem, rng, rsa)
    inv_mass, inv_inertia = _body_arrays(tm, shape, scale, density)
    w = drum_wall(radius, length, wall_spacing, mu, e)
    w.update(pos=np.zeros(3), quat=np.array([1.0, 0, 0, 0]), angvel=np.array([2 * math.pi * rpm / 60.0, 0, 0]))
    ext = np.array([0.5 * length, radius, radius])
    return {"templates": tm, "shape": shape, "scale": scale, "pos": pos, "quat": random_quaternions(rng, n),
            "vel": np.zeros((n, 3)), "inv_mass": inv_mass, "inv_inertia": inv_inertia, "kn": kn, "ks": kt_ratio * kn,
            "mu": mu, "e": e, "dt": dt, "min": -ext, "max": ext, "gravity": np.array([0.0, 0.0, -9.81]),
            "periodic": 0, "walls": [w], "size_factor": s, "rsa": rsa}


def settling_geometry(vol, solid_fraction, n, sphere_volume, b, reserve):
    """Side L of the cubic domain of the large-scale workload and the height of its reserve slab:
    the packing fills [0, L)^2 x [0, L - slab) at solid_fraction (L^2 (L - slab) = vol /
    solid_fraction), the slab on top holds reserve x n bounding spheres (mean volume
    sphere_volume) at 20 % fraction plus a gap of two largest bounding radii b."""
    L = (vol / solid_fraction) ** (1.0 / 3.0)
    for _ in range(60):  # a contraction (factor about 1/2): converged to rounding
        slab = reserve * n * sphere_volume / 0.2 / (L * L) + 2 * b
        L = math.sqrt(vol / solid_fraction / (L - slab))
    return L, reserve * n * sphere_volume / 0.2 / (L * L) + 2 * b


def settling_box(lsdem, n=2_000_000, shapes=16, exponents=(2.0, 6.0), semi_axes=(1e-3, 2.5e-3), n_grid=48,
                 n_nodes=1500, solid_fraction=0.25, kn=1e5, kt_ratio=0.8, mu=0.5, e=0.6, density=2500.0, dt=5e-7,
                 exclusion=0.85, reserve=0.02, seed=None, device=0, templates=None):
    """Large-scale workload: n particles from `shapes` seeded superquadrics (exponents uniform
    2-6, semi-axes uniform 1-2.5 mm, 1500 nodes, 48^3 grids from their meshes), periodic in x
    and y, floor and ceiling walls in z, settling under gravity from a random loose packing at
    solid fraction (cube box; random sequential addition of spheres of `exclusion` x the bounding
    radius, periodic in x and y and kept one bounding radius clear of the walls; random
    orientations, at rest; deep overlaps removed afterwards by resolve_deep_overlaps).

    Random placement of these shapes cannot reach the stated 0.3 without deep overlaps: their
    bounding spheres hold ~1.9 x their volume, so at 0.3 the spheres must overlap (exclusion
    <= 0.8) and a third or more of the bodies then start deeply interpenetrated, which
    re-placement cannot resolve. The default is 0.25 with exclusion 0.85 (~14 % of bodies in
    deep overlap before re-placement, a few per thousand after it); the bodies re-placement
    cannot fit go to a reserve slab above the packing (`reserve` x n bounding spheres at 20 %
    fraction, no overlaps). The domain is a cube: the packing fills its lower part at the stated
    fraction and the slab its top, so no body starts above the domain's y extent (the
    reference's image keys test z against the y bound, which would image such a body in place
    onto itself)."""
    rng = np.random.default_rng(seed_for(4) if seed is None else seed)
    T = templates or superquadric_templates(lsdem, rng, shapes, exponents, semi_axes, n_grid, n_nodes, device=device)
    tm = _unit_density_templates(lsdem, T, gpu=True)
    shape = rng.integers(0, len(tm), size=n).astype(np.int32)
    vol = np.array([t["mass"] for t in tm])[shape].sum()
    scale = np.ones(n)
    bound = np.array([t["bound"] for t in tm])[shape]
    b = float(bound.max())
    # A cube of side L holds the packing (height L - slab, at the stated solid fraction) and
    # the reserve slab above it. The domain is kept no taller than it is wide: the images'
    # cell keys test z against the y bound (the reference's rule, kept), so a body above
    # the y extent would be imaged in place onto itself.
    L, slab = settling_geometry(vol, solid_fraction, n, (4.0 / 3.0) * math.pi * float(np.mean(bound ** 3)), b,
                                reserve)
    H = L
    rsa = {"radius": exclusion * bound, "lo": np.array([0.0, 0.0, b]), "hi": np.array([L, L, L - slab - b]),
           "periodic": True, "bound": bound, "reserve_lo": np.array([0.0, 0.0, L - slab + b]),
           "reserve_hi": np.array([L, L, H])}
    pos = _rsa(lsdem, rng, rsa)
    inv_mass, inv_inertia = _body_arrays(tm, shape, scale, density)
    walls = [plane_wall(L, [0.5 * L, 0.5 * L, 0.0], True, mu, e), plane_wall(L, [0.5 * L, 0.5 * L, H], False, mu, e)]
    return {"templates": tm, "shape": shape, "scale": scale, "pos": pos, "quat": random_quaternions(rng, n),
            "vel": np.zeros((n, 3)), "inv_mass": inv_mass, "inv_inertia": inv_inertia, "kn": kn, "ks": kt_ratio * kn,
            "mu": mu, "e": e, "dt": dt, "min": np.zeros(3), "max": np.array([L, L, H]),
            "gravity": np.array([0.0, 0.0, -9.81]), "periodic": 3, "walls": walls, "rsa": rsa,
            "solid_fraction": solid_fraction, "raw_templates": T}


def write_c0_app_scene(path, sc, nsteps, k0, k1, nsteps2=0, floor_wz=0.0):
    """Scene file of the config-0 app (tests/apps/c0_bench.cpp, written against the LSSolver
    API only, so the same source builds against the reference and against the drop-in):
    magic "LSDEMC0", shape (node count, grid size, spacing, origin, nodes, SDF), particles
    (count, positions, quaternions, velocities), material (kn, ks, mu, e, density), the floor
    wall (grid, spacing, origin, SDF, position, quaternion, mu, e, vertices, two triangles),
    dt, domain, gravity, and the step count with the timed window (k0, k1], counted in
    hook calls; optionally a second phase of nsteps2 steps after the floor's angular velocity
    about z is set to floor_wz."""
    s, f = sc["shape"], sc["floor"]
    n = len(sc["pos"])
    d = lambda a: np.ascontiguousarray(a, np.float64).tobytes()
    i32 = lambda *v: struct.pack(f"<{len(v)}i", *v)
    cx, cy = 0.5 * (sc["min"][0] + sc["max"][0]), 0.5 * (sc["min"][1] + sc["max"][1])
    tris = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    with open(path, "wb") as fh:
        fh.write(b"LSDEMC0\0")
        fh.write(i32(len(s["nodes"]), *[int(v) for v in s["size"]], n))
        fh.write(d([s["spacing"]]) + d(s["origin"]) + d(s["nodes"]) + d(s["sdf"]))
        fh.write(d(sc["pos"]) + d(sc["quat"]) + d(sc["vel"]))
        fh.write(d([sc["kn"], sc["ks"], sc["mu"], sc["e"], sc["density"]]))
        fh.write(i32(*[int(v) for v in f["size"]]) + d([f["spacing"]]) + d(f["origin"]) + d(f["sdf"]))
        fh.write(d([cx, cy, sc["min"][2]]) + d([1.0, 0.0, 0.0, 0.0]) + d([sc["mu"], sc["e"]]))
        fh.write(i32(len(f["verts"]), len(tris)) + d(f["verts"]) + tris.tobytes())
        fh.write(d([sc["dt"]]) + d(sc["min"]) + d(sc["max"]) + d(sc["gravity"]))
        fh.write(i32(nsteps, k0, k1))
        if nsteps2 > 0:
            fh.write(i32(nsteps2) + d([floor_wz]))


def read_c0_app_result(path):
    """(steps run, window length, window device time in ms, velocities at the window's end)
    from the result file of the config-0 app."""
    raw = open(path, "rb").read()
    steps, window, nvel = struct.unpack("<3i", raw[:12])
    ms = struct.unpack("<d", raw[12:20])[0]
    vel = np.frombuffer(raw[20:20 + 24 * nvel], np.float64).reshape(nvel, 3)
    return steps, window, ms, vel

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


def rsa_positions(rng, n, radii, lo, hi, max_tries=200, periodic=False):
    """Random sequential addition of non-overlapping spheres (radii per particle) in the box [lo, hi]."""
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
                break
        else:
            raise RuntimeError(f"RSA could not place particle {i} (fraction too high)")
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
        # re-placed spheres may come a little closer than the first packing (0.75 x radius)
        rad = 0.5 * exclusion * sc["scale"]
        rad = np.where(keep == 0, rad * (0.75 / exclusion), rad)
        sc["pos"] = lsdem.pack_rsa(rad, sc["min"], sc["max"], periodic=bool(sc["periodic"]),
                                   seed=int(rng.integers(1 << 62)), max_tries=20000, keep=keep, pos=sc["pos"])
        sc["quat"][bad] = random_quaternions(rng, len(bad))
    sv.close()
    return it


def load_polydisperse(solver, sc):
    ids = [solver.add_shape(t["nodes"], t["sdf"], t["size"], t["origin"], t["spacing"]) for t in sc["templates"]]
    shape = np.asarray(ids, np.int32)[sc["shape"]]
    solver.add_particles(shape, sc["pos"], sc["quat"], sc["inv_mass"], sc["inv_inertia"], sc["kn"], sc["ks"],
                         sc["mu"], sc["e"], vel=sc["vel"], scale=sc["scale"])
    solver.set_periodic(sc["periodic"])

"""Numpy restatement of the support tables of the candidate separation test.

Mirrors the host construction of the solid's bounding points (runtime.cu, the grid refined by
two: sub-cell corners with phi <= tolerance, dilated by one refined point, boundary points
kept), the vertex tables of k_support_vertices / k_support_pack (largest projection at every
cube-map vertex direction (+-1, p, q), rounded up to FP32) and the FP32 lookup sup_bound_f
(face, gnomonic cell, linear interpolation on the cell's lower or upper triangle), each FP32
operation rounded as the kernel rounds it.
"""
import numpy as np

f32 = np.float32
M = 24


def fma32(a, b, c):
    return f32(np.float64(a) * np.float64(b) + np.float64(c))


def refined_solid_mask(t):
    """Mask (z, y, x) of the lattice at half spacings: the corners of every sub-cell with a
    corner phi <= tolerance, before the boundary reduction."""
    gx, gy, gz = (int(v) for v in t["size"])
    phi = np.asarray(t["sdf"], np.float64).reshape(gz, gy, gx)
    nx, ny, nz = 2 * gx - 1, 2 * gy - 1, 2 * gz - 1
    m = np.zeros((nz, ny, nx), bool)
    c = [phi[z0:gz - 1 + z0, y0:gy - 1 + y0, x0:gx - 1 + x0] for z0 in (0, 1) for y0 in (0, 1) for x0 in (0, 1)]
    c = np.stack(c, -1)  # (cz, cy, cx, 8), corner k = dx + 2 dy + 4 dz
    lo, hi = c.min(-1), c.max(-1)
    tol = 1e-12 * np.abs(c).max(-1)
    for k in range(27):
        i, j, l = k % 3, (k // 3) % 3, k // 9
        fx, fy, fz = 0.5 * i, 0.5 * j, 0.5 * l
        c00 = c[..., 0] * (1 - fx) + c[..., 1] * fx
        c10 = c[..., 2] * (1 - fx) + c[..., 3] * fx
        c01 = c[..., 4] * (1 - fx) + c[..., 5] * fx
        c11 = c[..., 6] * (1 - fx) + c[..., 7] * fx
        v = (c00 * (1 - fy) + c10 * fy) * (1 - fz) + (c01 * (1 - fy) + c11 * fy) * fz
        v = np.where(hi <= tol, lo, v)
        mark = (lo <= tol) & (v <= tol)
        zz, yy, xx = np.nonzero(mark)
        m[2 * zz + l, 2 * yy + j, 2 * xx + i] = True
    for ax in range(3):  # dilation by one point along each axis: the 27-neighbourhood
        d = m.copy()
        a, b = [slice(None)] * 3, [slice(None)] * 3
        a[ax], b[ax] = slice(1, None), slice(None, -1)
        d[tuple(a)] |= m[tuple(b)]
        d[tuple(b)] |= m[tuple(a)]
        m = d
    return m


def boundary(m):
    pad = np.pad(m, 1)
    interior = m & pad[2:, 1:-1, 1:-1] & pad[:-2, 1:-1, 1:-1] & pad[1:-1, 2:, 1:-1] & pad[1:-1, :-2, 1:-1] \
        & pad[1:-1, 1:-1, 2:] & pad[1:-1, 1:-1, :-2]
    interior[[0, -1], :, :] = False
    interior[:, [0, -1], :] = False
    interior[:, :, [0, -1]] = False
    return m & ~interior


def lattice_points(t, mask):
    z, y, x = np.nonzero(mask)
    o, h = np.asarray(t["origin"], np.float64), 0.5 * float(t["spacing"])
    return np.stack([o[0] + h * x, o[1] + h * y, o[2] + h * z], 1)


def solid_points(t):
    """The points the host uploads for the solid's table (boundary of the refined set)."""
    return lattice_points(t, boundary(refined_solid_mask(t)))


def vertex_dirs():
    """(6, M + 1, M + 1, 3): vertex (i, j) of face f as (+-1, p, q) in the face's axes."""
    V = np.zeros((6, M + 1, M + 1, 3))
    for f in range(6):
        sg = -1.0 if f & 1 else 1.0
        for j in range(M + 1):
            for i in range(M + 1):
                p, q = -1.0 + 2.0 * i / M, -1.0 + 2.0 * j / M
                V[f, j, i] = [sg, p, q] if f < 2 else ([q, sg, p] if f < 4 else [p, q, sg])
    return V


def round_up32(v):
    v = np.asarray(v, np.float64)
    v = v + 1e-9 * np.abs(v) + 1e-30
    r = v.astype(np.float32)
    low = r.astype(np.float64) < v
    r[low] = np.nextafter(r[low], np.float32(np.inf))
    return r


def vertex_table(points):
    """(6, M + 1, M + 1) FP32 vertex values of the largest projection of `points`."""
    V = vertex_dirs().reshape(-1, 3)
    return round_up32((V @ np.asarray(points).T).max(1)).reshape(6, M + 1, M + 1)


def face_coords(u):
    a = [abs(x) for x in u]
    if a[0] >= a[1] and a[0] >= a[2]:
        return (0 if u[0] >= 0 else 1), a[0], u[1], u[2]
    if a[1] >= a[2]:
        return (2 if u[1] >= 0 else 3), a[1], u[2], u[0]
    return (4 if u[2] >= 0 else 5), a[2], u[0], u[1]


def sup_bound_f(tab, u):
    """(bound of h(u / m), m) as sup_bound_f computes them (u in FP32)."""
    u = [f32(x) for x in u]
    f, m, p, q = face_coords(u)
    m = f32(m)
    if not m > 0:
        return f32(0.0), f32(0.0)
    r = f32(f32(1.0) / m)
    x = f32(fma32(p, r, f32(1.0)) * f32(0.5 * M))
    y = f32(fma32(q, r, f32(1.0)) * f32(0.5 * M))
    i = min(max(int(np.floor(x)), 0), M - 1)
    j = min(max(int(np.floor(y)), 0), M - 1)
    s = f32(min(max(f32(x - f32(i)), f32(0.0)), f32(1.0)))
    t = f32(min(max(f32(y - f32(j)), f32(0.0)), f32(1.0)))
    c0, c1, c2, c3 = tab[f, j, i], tab[f, j, i + 1], tab[f, j + 1, i], tab[f, j + 1, i + 1]
    if f32(s + t) <= f32(1.0):
        return fma32(s, f32(c1 - c0), fma32(t, f32(c2 - c0), c0)), m
    return fma32(f32(f32(1.0) - s), f32(c2 - c3), fma32(f32(f32(1.0) - t), f32(c1 - c3), c3)), m


def sup_bound_exact(tab, u):
    """The same bound in FP64 arithmetic (exact interpolation point): h(u / m) <= value."""
    f, m, p, q = face_coords(np.asarray(u, np.float64))
    x, y = (p / m + 1.0) * 0.5 * M, (q / m + 1.0) * 0.5 * M
    i, j = min(max(int(np.floor(x)), 0), M - 1), min(max(int(np.floor(y)), 0), M - 1)
    s, t = x - i, y - j
    c0, c1, c2, c3 = (np.float64(v) for v in (tab[f, j, i], tab[f, j, i + 1], tab[f, j + 1, i], tab[f, j + 1, i + 1]))
    if s + t <= 1.0:
        return c0 + s * (c1 - c0) + t * (c2 - c0), m
    return c3 + (1.0 - s) * (c2 - c3) + (1.0 - t) * (c1 - c3), m

"""The separation test's tables and FP32 margins against exact supports (CPU).

pair_separated drops a pair when scale_A sup_n + scale_B sup_s, looked up at the cube-map
cells of the FP32-rotated centre difference, plus its slack, falls short of the FP32
centre distance. Here the tables are built as k_support_tables builds them and the test is
restated in numpy float32 (each operation rounded to FP32, fused multiply-adds rounded
once); for random pairs of the four templates near their touching distance, in domains at
the origin and 3 m from it, every pair the FP32 test drops is separated in exact FP64
arithmetic: the largest projection of A's nodes onto the line of centres plus that of B's
solid cells (the grid points of the cells with a corner phi <= 0) falls short of the
distance. And the test does drop pairs.
"""
import numpy as np

f32 = np.float32
M = 24


def _fma(a, b, c):
    return f32(np.float64(a) * np.float64(b) + np.float64(c))


def _sup_dir(f, p, q):
    sg = -1.0 if f & 1 else 1.0
    v = np.array([sg, p, q]) if f < 2 else (np.array([q, sg, p]) if f < 4 else np.array([p, q, sg]))
    return v / np.linalg.norm(v)


def _cells():
    C, D = [], []
    h = 2.0 / M
    for f in range(6):
        for j in range(M):
            for i in range(M):
                p0, q0 = -1.0 + h * i, -1.0 + h * j
                c = _sup_dir(f, p0 + 0.5 * h, q0 + 0.5 * h)
                d = max(np.linalg.norm(_sup_dir(f, p0 + h * (k & 1), q0 + h * (k >> 1)) - c) for k in range(4))
                C.append(c)
                D.append(d * (1.0 + 1e-9) + 1e-5)
    return np.array(C), np.array(D)


def _solid_points(t):
    nx, ny, nz = t["size"]
    m = np.asarray(t["sdf"]).reshape(nz, ny, nx) <= 0
    for ax in range(3):
        d = m.copy()
        a, b = [slice(None)] * 3, [slice(None)] * 3
        a[ax], b[ax] = slice(1, None), slice(None, -1)
        d[tuple(a)] |= m[tuple(b)]
        d[tuple(b)] |= m[tuple(a)]
        m = d
    z, y, x = np.nonzero(m)
    o, h = np.asarray(t["origin"]), t["spacing"]
    return np.stack([o[0] + h * x, o[1] + h * y, o[2] + h * z], 1)


def _tables(templates):
    C, Dl = _cells()
    out = []
    for t in templates:
        nd, sp = np.asarray(t["nodes"]), _solid_points(t)
        hn = (C @ nd.T + Dl[:, None] * np.linalg.norm(nd, axis=1)[None]).max(1)
        hs = (C @ sp.T + Dl[:, None] * np.linalg.norm(sp, axis=1)[None]).max(1)
        up = lambda v: np.nextafter(f32(v), f32(np.inf)) if f32(v) < v else f32(v)
        out.append({"n": [up(v * (1 + 1e-9)) for v in hn], "s": [up(v * (1 + 1e-9)) for v in hs],
                    "r": up(np.linalg.norm(sp, axis=1).max() * (1 + 1e-9)), "nodes": nd, "solid": sp})
    return out


def _rot_inv_f(v, q):
    w, a, b, c = f32(q[0]), -f32(q[1]), -f32(q[2]), -f32(q[3])
    two = f32(2.0)
    tx = two * _fma(b, v[2], -(c * v[1]))
    ty = two * _fma(c, v[0], -(a * v[2]))
    tz = two * _fma(a, v[1], -(b * v[0]))
    return (f32(_fma(w, tx, v[0]) + _fma(b, tz, -(c * ty))), f32(_fma(w, ty, v[1]) + _fma(c, tx, -(a * tz))),
            f32(_fma(w, tz, v[2]) + _fma(a, ty, -(b * tx))))


def _cell_f(u):
    a = [abs(x) for x in u]
    if a[0] >= a[1] and a[0] >= a[2]:
        f, m, p, q = (0 if u[0] >= 0 else 1), a[0], u[1], u[2]
    elif a[1] >= a[2]:
        f, m, p, q = (2 if u[1] >= 0 else 3), a[1], u[2], u[0]
    else:
        f, m, p, q = (4 if u[2] >= 0 else 5), a[2], u[0], u[1]
    r = f32(1.0) / m
    i = min(max(int(np.floor(f32(_fma(p, r, f32(1.0)) * f32(0.5 * M)))), 0), M - 1)
    j = min(max(int(np.floor(f32(_fma(q, r, f32(1.0)) * f32(0.5 * M)))), 0), M - 1)
    return (f * M + j) * M + i


def _separated_f(tab, pa, qa, sa, ka, pb, qb, sb, kb):
    d = [f32(pb[k] - pa[k]) for k in range(3)]
    D2 = _fma(d[0], d[0], _fma(d[1], d[1], f32(d[2] * d[2])))
    ua, ub = _rot_inv_f(d, qa), _rot_inv_f([-x for x in d], qb)
    hA, hB = tab[ka]["n"][_cell_f(ua)], tab[kb]["s"][_cell_f(ub)]
    reach = _fma(sa, hA, f32(sb * hB))
    D = f32(np.sqrt(np.float64(D2)))
    n1a = f32(f32(abs(pa[0]) + abs(pa[1])) + abs(pa[2]))
    n1 = f32(n1a + f32(f32(abs(pb[0]) + abs(pb[1])) + abs(pb[2])))
    eps = f32(f32(f32(f32(4e-7) * f32(n1 + D)) / D) + f32(4e-6))
    rho = f32(pa[3] + f32(sb * tab[kb]["r"]))
    slack = _fma(eps, rho, _fma(f32(1e-6), n1, f32(f32(1e-5) * D)))
    return f32(f32(reach + slack) * f32(1.0 + 1e-5)) < D


def _rot(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _run(offset, pairs=1500, seed=0):
    from conftest import load_package
    lsdem = load_package()
    from lsdem_b200 import scenes
    T = scenes.unit_templates(n_grid=16, n_nodes=200)
    tab = _tables(T)
    rng = np.random.default_rng(seed)
    dropped = wrong = 0
    for _ in range(pairs):
        ka, kb = rng.integers(0, 4, size=2)
        qa, qb = (q / np.linalg.norm(q) for q in rng.normal(size=(2, 4)))
        sa, sb = 2e-3 * np.exp(0.25 * rng.standard_normal(2))
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        Ra, Rb = _rot(qa), _rot(qb)
        exact = sa * (tab[ka]["nodes"] @ (Ra.T @ u)).max() + sb * (tab[kb]["solid"] @ (Rb.T @ -u)).max()
        D = exact * rng.uniform(0.98, 1.3)
        xa = offset + rng.uniform(0.0, 0.05, size=3)
        xb = xa + D * u
        ra = sa * np.linalg.norm(tab[ka]["nodes"], axis=1).max()
        pa = [f32(v) for v in xa] + [f32(ra)]
        pb = [f32(v) for v in xb] + [f32(0.0)]
        if _separated_f(tab, pa, qa, f32(sa), ka, pb, qb, f32(sb), kb):
            dropped += 1
            wrong += not (exact < np.linalg.norm(xb - xa))
    return dropped, wrong


def test_dropped_pairs_are_separated_near_origin():
    dropped, wrong = _run(np.zeros(3))
    assert wrong == 0
    assert dropped > 100


def test_dropped_pairs_are_separated_far_from_origin():
    dropped, wrong = _run(np.full(3, 3.0), seed=1)
    assert wrong == 0
    assert dropped > 100

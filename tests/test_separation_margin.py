"""The separation test's tables and FP32 margins against exact supports (CPU).

pair_separated drops a pair when scale_A h_n + scale_B h_s, interpolated from the vertex
tables at the FP32-rotated centre difference, plus its slack, falls short of the FP32 centre
distance. Here the tables are built as the library builds them (support_restate.py) and the
test is restated in numpy float32 (each operation rounded to FP32, fused multiply-adds rounded
once); for random pairs of the four templates near their touching distance, in domains at the
origin and 3 m from it, every pair the FP32 test drops is separated in exact FP64 arithmetic:
the largest projection of A's nodes onto the line of centres plus that of B's solid point set
(whose hull holds every point with phi <= 0) falls short of the distance. And the test drops
most pairs beyond 1.05 times that distance.
"""
import numpy as np

import support_restate as sr
from support_restate import f32, fma32 as _fma


def _tables(templates):
    out = []
    for t in templates:
        nd, sp = np.asarray(t["nodes"]), sr.solid_points(t)
        out.append({"n": sr.vertex_table(nd), "s": sr.vertex_table(sp),
                    "r": sr.round_up32([np.linalg.norm(sp, axis=1).max()])[0], "nodes": nd, "solid": sp})
    return out


def _rot_inv_f(v, q):
    w, a, b, c = f32(q[0]), -f32(q[1]), -f32(q[2]), -f32(q[3])
    two = f32(2.0)
    tx = two * _fma(b, v[2], -(c * v[1]))
    ty = two * _fma(c, v[0], -(a * v[2]))
    tz = two * _fma(a, v[1], -(b * v[0]))
    return (f32(_fma(w, tx, v[0]) + _fma(b, tz, -(c * ty))), f32(_fma(w, ty, v[1]) + _fma(c, tx, -(a * tz))),
            f32(_fma(w, tz, v[2]) + _fma(a, ty, -(b * tx))))


def _separated_f(tab, pa, qa, sa, ka, pb, qb, sb, kb):
    d = [f32(pb[k] - pa[k]) for k in range(3)]
    D2 = _fma(d[0], d[0], _fma(d[1], d[1], f32(d[2] * d[2])))
    if not D2 > 0:
        return False
    ua, ub = _rot_inv_f(d, qa), _rot_inv_f([-x for x in d], qb)
    hA, ma = sr.sup_bound_f(tab[ka]["n"], ua)
    hB, mb = sr.sup_bound_f(tab[kb]["s"], ub)
    D = f32(np.sqrt(np.float64(D2)))
    reach = f32(_fma(f32(sa * ma), hA, f32(f32(sb * mb) * hB)) / D)
    n1a = f32(f32(abs(pa[0]) + abs(pa[1])) + abs(pa[2]))
    n1 = f32(n1a + f32(f32(abs(pb[0]) + abs(pb[1])) + abs(pb[2])))
    eps = f32(f32(f32(f32(4e-7) * f32(n1 + D)) / D) + f32(8e-6))
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
    dropped = wrong = far = far_dropped = 0
    for _ in range(pairs):
        ka, kb = rng.integers(0, 4, size=2)
        qa, qb = (q / np.linalg.norm(q) for q in rng.normal(size=(2, 4)))
        sa, sb = 2e-3 * np.exp(0.25 * rng.standard_normal(2))
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        Ra, Rb = _rot(qa), _rot(qb)
        exact = sa * (tab[ka]["nodes"] @ (Ra.T @ u)).max() + sb * (tab[kb]["solid"] @ (Rb.T @ -u)).max()
        D = exact * rng.uniform(0.98, 1.3)
        far += D > 1.05 * exact
        xa = offset + rng.uniform(0.0, 0.05, size=3)
        xb = xa + D * u
        ra = sa * np.linalg.norm(tab[ka]["nodes"], axis=1).max()
        pa = [f32(v) for v in xa] + [f32(ra)]
        pb = [f32(v) for v in xb] + [f32(0.0)]
        if _separated_f(tab, pa, qa, f32(sa), ka, pb, qb, f32(sb), kb):
            dropped += 1
            wrong += not (exact < np.linalg.norm(xb - xa))
            far_dropped += D > 1.05 * exact
    return dropped, wrong, far_dropped / far


def test_dropped_pairs_are_separated_near_origin():
    dropped, wrong, far = _run(np.zeros(3))
    assert wrong == 0
    assert dropped > 100
    assert far > 0.9


def test_dropped_pairs_are_separated_far_from_origin():
    dropped, wrong, far = _run(np.full(3, 3.0), seed=1)
    assert wrong == 0
    assert dropped > 100
    assert far > 0.9

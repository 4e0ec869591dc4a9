"""The margin argument of the neighbour lists, on a restatement of the FP32 tests (CPU).

k_candidates keeps in a particle's list the bodies that pass the bounding-sphere test
with the reach enlarged by the margin (skin, plus 1e-5 of the coordinate sum, times
1 + 1e-4), and rebuilds the lists once any particle has moved sqrt(move2) = 0.4 skin,
skin = a tenth of the largest bounding radius. Between rebuilds a listed body is a
candidate when it passes the plain test. The lists are exact when every pair that passes
the plain test after such moves was listed. Checked here with the kernel's operations
restated in numpy float32 (each add and multiply rounded to FP32; fused multiply-adds
rounded once), on random polydisperse packings placed near the origin and far from it,
with every pair moved towards each other by the full rebuild distance each, and the
margin shown to be needed: without the skin, pairs are missed.
"""
import numpy as np

f32 = np.float32


def _fma(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(f32)


def _n1(p):
    return (np.abs(p[:, 0]) + np.abs(p[:, 1])).astype(f32) + np.abs(p[:, 2])


def _reach(pa, pb):
    n1 = (_n1(pa) + _n1(pb)).astype(f32)
    return _fma(np.full_like(n1, f32(1e-6)), n1, ((pa[:, 3] + pb[:, 3]) * f32(1.0 + 1e-5)).astype(f32)), n1


def _dist2(pa, pb):
    d = (pb[:, :3] - pa[:, :3]).astype(f32)
    return _fma(d[:, 0], d[:, 0], _fma(d[:, 1], d[:, 1], (d[:, 2] * d[:, 2]).astype(f32)))


def _packed(x, r):
    return np.concatenate([x.astype(f32), r.astype(f32)[:, None]], axis=1)


def _pairs(rng, n, offset):
    r = 1e-3 * np.exp(0.25 * rng.standard_normal(n))
    x = offset + rng.uniform(0.0, 0.02, size=(n, 3))
    i, j = np.triu_indices(n, 1)
    near = np.linalg.norm(x[i] - x[j], axis=1) < (r[i] + r[j]) * 1.3
    return x, r, i[near], j[near]


def _check(offset, skin_scale=1.0, seed=0):
    rng = np.random.default_rng(seed)
    x, r, i, j = _pairs(rng, 1500, offset)
    sr = 0.1 * r.max()
    skin = f32(sr * skin_scale)
    move = 0.4 * sr
    # build: list the pairs within reach + margin
    pa, pb = _packed(x[i], r[i]), _packed(x[j], r[j])
    R, n1 = _reach(pa, pb)
    Rs = (_fma(np.full_like(n1, f32(1e-5)), n1, (R + skin).astype(f32)) * f32(1.0 + 1e-4)).astype(f32)
    listed = _dist2(pa, pb) <= (Rs * Rs).astype(f32)
    # every pair moves towards each other by the full rebuild distance, each (in FP64)
    u = x[j] - x[i]
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    xa, xb = x[i] + move * u, x[j] - move * u
    qa, qb = _packed(xa, r[i]), _packed(xb, r[j])
    R1, _ = _reach(qa, qb)
    passes = _dist2(qa, qb) <= (R1 * R1).astype(f32)
    return passes, listed


def test_lists_hold_every_pair_after_moves_near_origin():
    passes, listed = _check(np.zeros(3))
    assert passes.sum() > 100
    assert not (passes & ~listed).any()


def test_lists_hold_every_pair_after_moves_far_from_origin():
    # coordinates of 3 m: FP32 spacing 2.4e-7 m; the coordinate part of the margin, 1e-5 of
    # the coordinate sum (0.18 mm), is then about the size of the skin (0.1 mm here)
    passes, listed = _check(np.full(3, 3.0), seed=1)
    assert passes.sum() > 100
    assert not (passes & ~listed).any()


def test_the_margin_is_needed():
    passes, listed = _check(np.zeros(3), skin_scale=0.0, seed=2)
    assert (passes & ~listed).any()

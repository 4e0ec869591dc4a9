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

The rebuild also has to reach the listed bodies: cells are only 2 rmax wide and reach +
skin is up to 2.1 rmax, so a listed partner can lie two cells away. The rebuild walk's
cell range (the 27 cells widened to the ball of reach + skin) is restated and checked on
near-largest bodies: every pair found after the moves was listed, while a walk of the
27 cells alone would miss some.
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


def _walk_window(xa, ra, rmax, skin, mn, w, size):
    """Cells the rebuild walks for owners at xa (k_candidates): the 27 cells around the
    clamped cell, widened to every cell the ball of reach + skin overlaps."""
    c = np.clip(np.floor((xa - mn) / w).astype(np.int64), 0, size - 1)
    R = ra + rmax + skin
    ext = 1.001 * R + 1e-4 * (np.abs(xa).sum(axis=1) + 4.0 * R)
    e0 = np.clip(np.floor((xa - ext[:, None] - mn) / w), 0, size - 1).astype(np.int64)
    e1 = np.clip(np.floor((xa + ext[:, None] - mn) / w), 0, size - 1).astype(np.int64)
    lo = np.minimum(np.clip(c - 1, 0, size - 1), e0)
    hi = np.maximum(np.clip(c + 1, 0, size - 1), e1)
    return c, lo, hi


def _window_check(offset, seed):
    """Pairs of near-largest bodies at 1.9-2.1 bounding radii along random directions,
    owners anywhere in their cells (cell = 2 rmax, the narrowest grid). Returns, per
    pair, whether it passes the plain test and lies in the 27-cell window after both
    bodies moved the rebuild distance towards each other, whether the rebuild walk
    listed it, and whether a walk of the 27 cells alone would have."""
    rng = np.random.default_rng(seed)
    n = 200_000
    rmax = 1e-3
    ra, rb = rmax * rng.uniform(0.9, 1.0, n), rmax * rng.uniform(0.9, 1.0, n)
    w = 2.0 * rmax
    mn = offset - 0.5
    size = np.full(3, int(1.0 / w))
    xa = offset + rng.uniform(-0.2, 0.2, size=(n, 3))
    u = rng.standard_normal((n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    xb = xa + (rng.uniform(1.9, 2.1, n) * rmax)[:, None] * u
    sr = 0.1 * rmax
    skin = f32(sr)
    pa, pb = _packed(xa, ra), _packed(xb, rb)
    R, n1 = _reach(pa, pb)
    Rs = (_fma(np.full_like(n1, f32(1e-5)), n1, (R + skin).astype(f32)) * f32(1.0 + 1e-4)).astype(f32)
    within = _dist2(pa, pb) <= (Rs * Rs).astype(f32)
    c, lo, hi = _walk_window(xa, ra, rmax, sr, mn, w, size)
    cb = np.floor((xb - mn) / w).astype(np.int64)
    walked = ((cb >= lo) & (cb <= hi)).all(axis=1)
    in27 = (np.abs(cb - c) <= 1).all(axis=1)
    move = 0.4 * sr
    xa1, xb1 = xa + move * u, xb - move * u
    qa, qb = _packed(xa1, ra), _packed(xb1, rb)
    R1, _ = _reach(qa, qb)
    c1 = np.clip(np.floor((xa1 - mn) / w).astype(np.int64), 0, size - 1)
    cb1 = np.floor((xb1 - mn) / w).astype(np.int64)
    found = (_dist2(qa, qb) <= (R1 * R1).astype(f32)) & (np.abs(cb1 - c1) <= 1).all(axis=1)
    return found, within & walked, within & in27


def test_rebuild_walk_lists_partners_beyond_the_27_cells():
    for offset, seed in ((np.zeros(3), 3), (np.full(3, 3.0), 4)):
        found, listed, listed27 = _window_check(offset, seed)
        assert found.sum() > 1000
        assert not (found & ~listed).any()
        # a walk of the 27 cells alone misses pairs that later pass
        assert (found & ~listed27).any()

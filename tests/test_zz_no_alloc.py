"""The allocation-free cell sort (lsdem_cell_sort_static) against the oracle.

Callers that cannot allocate device memory when they call the library (loops
where an allocation could block or synchronise the device, host applications
whose device memory belongs to their own pool or fixed budget) get a cell sort
whose scratch is a fixed device array inside the library. These tests call it
through the C ABI and compare its cell keys, stable sorted order, sorted keys and
cell ranges with the FP64 oracle's (ora_hash + ora_sort_ranges, restating
mySpatialGrid.cu:4-26 and buildHashStartEnd.cu:18-137): exact match, on two calls
in a row each, since every call shares the array and must clear what it needs.

* the particle positions of a running solver (125 bodies, three below the domain),
  also checked against the solver's own sort;
* synthetic positions at the scratch's limits, 2^18 bodies and 2^18 cells, with one
  cell of 300 bodies (the block-ranked large-bucket path), 150 bodies outside the
  domain (key -1) and, through an inverse cell size a little above the grid's,
  bodies whose key lies past the last cell (both placed in index order by the
  special-bucket path);
* sizes beyond the limits, an overflowing cell-count product included, rejected.

Kept in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import dense_ellipsoid_scene, load_scene

pytestmark = pytest.mark.gpu

LIMIT = 1 << 18


def _call(lsdem, pos_ptr, n, g, out, sorted_key=True):
    d = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(lsdem.DP)
    size = np.ascontiguousarray(g["size"], np.int32)
    sk = C.c_void_p(out["sorted_key"].data_ptr()) if sorted_key else None
    return lsdem.lib.lsdem_cell_sort_static(
        C.c_void_p(pos_ptr), int(n), d(g["min"]), d(g["max"]), d(g["inv"]), size.ctypes.data_as(lsdem.IP),
        C.c_void_p(out["key"].data_ptr()), C.c_void_p(out["sorted_idx"].data_ptr()), sk,
        C.c_void_p(out["start"].data_ptr()), C.c_void_p(out["end"].data_ptr()), None)


def _outputs(n, nc):
    import torch
    dev = torch.device("cuda", 0)
    out = {k: torch.full((max(n, 1),), -7, dtype=torch.int32, device=dev) for k in ("key", "sorted_idx", "sorted_key")}
    out.update({k: torch.full((nc,), -7, dtype=torch.int32, device=dev) for k in ("start", "end")})
    return out


def _oracle(ora, pos, g):
    key = ora.hash_keys(pos, g)
    r = ora.sort_ranges(key, int(np.prod(g["size"])))
    return {"key": key, "sorted_idx": r["sorted_idx"], "sorted_key": r["sorted_key"], "start": r["start"],
            "end": r["end"]}


def _check(got, ref, what, keys=("key", "sorted_idx", "sorted_key", "start", "end")):
    for k in keys:
        assert np.array_equal(got[k], ref[k]), f"{what}: {k} differs"


def test_static_cell_sort_matches_oracle_and_solver(lsdem, ora):
    import torch
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=125, seed=13)
    sc["pos"][:3, 2] = -0.05  # three bodies below the domain: key -1
    sv = load_scene(lsdem, scenes, sc)
    n = sv.n_particles
    g = sv.grid()
    nc = int(np.prod(g["size"]))
    out = _outputs(n, nc)
    for call in range(2):
        sv.step(1e-6, 1)
        ref = sv.hash()
        pos_host = sv.state()["pos"]
        torch.cuda.synchronize()
        rc = _call(lsdem, sv.device_pointers()["pos"], n, g, out)
        torch.cuda.synchronize()
        assert rc == 0, f"call {call}: status {rc}"
        got = {k: v.cpu().numpy()[: len(ref[k])] for k, v in out.items()}
        assert (got["key"] == -1).sum() == 3
        _check(got, _oracle(ora, pos_host, g), f"call {call} vs oracle")
        _check(got, ref, f"call {call} vs solver")
    # beyond the fixed scratch: rejected before any device work
    pos = sv.device_pointers()["pos"]
    assert _call(lsdem, pos, LIMIT + 1, g, out) == 1  # LSDEM_ERR_ARG
    assert _call(lsdem, pos, n, dict(g, size=np.array([1 << 7, 1 << 7, 1 << 5], np.int32)), out) == 1  # 2^19 cells
    # a product that wraps a 64-bit integer to a small value is rejected too
    assert _call(lsdem, pos, n, dict(g, size=np.array([1 << 21, 1 << 21, 1 << 21], np.int32)), out) == 1
    assert _call(lsdem, pos, n, dict(g, size=np.array([1 << 30, 1, 1], np.int32)), out) == 1
    sv.close()


def _limit_scene(seed):
    """2^18 positions in a 64^3 grid of the unit cube: uniform, one cell crowded with
    300 bodies, 150 bodies outside the domain, and the z inverse cell size 0.2 %
    above the grid's, so that bodies in the top 0.2 % of the box get keys past the
    last cell."""
    rng = np.random.default_rng(seed)
    n = LIMIT
    pos = rng.uniform(0.0, 1.0, size=(n, 3))
    crowd = rng.choice(n, 300, replace=False)
    pos[crowd] = (np.array([17, 40, 5]) + rng.uniform(0.05, 0.95, size=(300, 3))) / 64.0
    rest = np.setdiff1d(np.arange(n), crowd)
    out = rng.choice(rest, 150, replace=False)
    pos[out] = rng.uniform(1.1, 2.0, size=(150, 3)) * rng.choice([-1.0, 1.0], size=(150, 3))
    g = {"min": np.zeros(3), "max": np.ones(3), "inv": np.array([64.0, 64.0, 64.0 * 1.002]),
         "size": np.array([64, 64, 64], np.int32)}
    return pos, g


def test_static_cell_sort_at_the_scratch_limits(lsdem, ora):
    import torch
    n, nc = LIMIT, LIMIT
    out = _outputs(n, nc)
    for call, seed in enumerate((101, 102)):
        pos, g = _limit_scene(seed)
        ref = _oracle(ora, pos, g)
        # the paths this case is meant to reach
        assert np.bincount(ref["key"][(ref["key"] >= 0) & (ref["key"] < nc)]).max() >= 300
        assert (ref["key"] == -1).sum() >= 150 and (ref["key"] >= nc).sum() > 64
        dpos = torch.from_numpy(pos).to("cuda:0")
        torch.cuda.synchronize()
        rc = _call(lsdem, dpos.data_ptr(), n, g, out, sorted_key=(call == 0))
        torch.cuda.synchronize()
        assert rc == 0, f"call {call}: status {rc}"
        got = {k: v.cpu().numpy() for k, v in out.items()}
        keys = ("key", "sorted_idx", "sorted_key", "start", "end") if call == 0 else ("key", "sorted_idx", "start", "end")
        _check(got, ref, f"call {call}", keys)

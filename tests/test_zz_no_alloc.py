"""The allocation-free cell sort (lsdem_cell_sort_static) against the solver's own.

Callers that cannot allocate device memory when they call the library get a
cell sort whose scratch is a fixed device array inside the library. This test
calls it through the C ABI on the particle positions of a running solver and
checks that its cell keys, stable sorted order, sorted keys and cell ranges are
identical to those the solver's step produced (lsdem_get_hash), on two calls in a
row (after two consecutive steps), and that sizes beyond its fixed limit are
rejected. Integer outputs: exact match. Kept in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import dense_ellipsoid_scene, load_scene

pytestmark = pytest.mark.gpu

LIMIT = 1 << 18


def _call(lsdem, pos_ptr, n, g, out, stream=None):
    d = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(lsdem.DP)
    size = np.ascontiguousarray(g["size"], np.int32)
    return lsdem.lib.lsdem_cell_sort_static(
        C.c_void_p(pos_ptr), int(n), d(g["min"]), d(g["max"]), d(g["inv"]), size.ctypes.data_as(lsdem.IP),
        C.c_void_p(out["key"].data_ptr()), C.c_void_p(out["sorted_idx"].data_ptr()),
        C.c_void_p(out["sorted_key"].data_ptr()), C.c_void_p(out["start"].data_ptr()),
        C.c_void_p(out["end"].data_ptr()), stream)


def test_static_cell_sort_matches_solver(lsdem):
    import torch
    from lsdem_b200 import scenes
    sc = dense_ellipsoid_scene(scenes, n=125, seed=13)
    sc["pos"][:3, 2] = -0.05  # three bodies below the domain: key -1
    sv = load_scene(lsdem, scenes, sc)
    n = sv.n_particles
    g = sv.grid()
    nc = int(np.prod(g["size"]))
    dev = torch.device("cuda", 0)
    out = {k: torch.full((n,), -7, dtype=torch.int32, device=dev) for k in ("key", "sorted_idx", "sorted_key")}
    out.update({k: torch.full((nc,), -7, dtype=torch.int32, device=dev) for k in ("start", "end")})
    for call in range(2):
        sv.step(1e-6, 1)
        ref = sv.hash()
        pos = sv.device_pointers()["pos"]
        torch.cuda.synchronize()
        rc = _call(lsdem, pos, n, g, out)
        torch.cuda.synchronize()
        assert rc == 0, f"call {call}: status {rc}"
        got = {k: v.cpu().numpy() for k, v in out.items()}
        assert (got["key"] == -1).sum() == 3
        for k in ("key", "sorted_idx", "sorted_key", "start", "end"):
            assert np.array_equal(got[k], ref[k]), f"call {call}: {k} differs"
    # beyond the fixed scratch: rejected before any device work
    assert _call(lsdem, sv.device_pointers()["pos"], LIMIT + 1, g, out) == 1  # LSDEM_ERR_ARG
    big = dict(g, size=np.array([1 << 7, 1 << 7, 1 << 5], np.int32))  # 2^19 cells
    assert _call(lsdem, sv.device_pointers()["pos"], n, big, out) == 1  # LSDEM_ERR_ARG
    sv.close()

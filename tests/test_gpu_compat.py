"""The reference's separable launchers (include/lsdem_compat.h) against the golden vectors
the reference's own kernels produced (tests/golden/, made by tests/golden/make_golden.py
from oracle/_ref/libfundem_ref.so): launchUpdateSpatialGridHashStartEnd
(mySpatialGrid.h:33-49; sorted keys, sorted order and cell ranges bit-exact, twice, the
second call on other positions), the two integration launchers (particleIntegrationKernel.cuh:4-30;
velocities and angular velocities within 1e-14 / 1e-13 relative, positions and quaternions
within 1e-15, the tolerances the oracle meets on the same vectors: FMA contraction), and
the periodic wraps along x and y (mySpatialGrid.h:51-65; bit-exact). Called through ctypes
with the reference's by-value vector arguments.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


class D3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class I3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


def gold(name):
    return np.load(ROOT / "tests" / "golden" / name)


def _d3(v):
    return D3(*[float(x) for x in v])


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def _p(t):
    return C.c_void_p(t.data_ptr())


def _close(a, b, rtol, scale=None):
    s = scale if scale is not None else max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) <= rtol * s


def test_hash_start_end_launcher(lsdem):
    import torch
    L = lsdem.lib
    f = L.launchUpdateSpatialGridHashStartEnd
    f.restype = None
    f.argtypes = [C.c_void_p] * 5 + [D3, D3, D3, I3, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p]
    g = gold("hash_sort.npz")
    nc = int(np.prod(g["size"]))
    n = len(g["pos"])
    for call, pos in enumerate((g["pos"], g["pos"][::-1].copy())):
        idx = torch.full((n,), -7, dtype=torch.int32, device="cuda:0")
        key = torch.full((n,), -7, dtype=torch.int32, device="cuda:0")
        st = torch.full((nc,), -7, dtype=torch.int32, device="cuda:0")
        en = torch.full((nc,), -7, dtype=torch.int32, device="cuda:0")
        dpos = _dev(pos)
        f(_p(idx), _p(key), _p(dpos), _p(st), _p(en), _d3(g["min"]), _d3(g["max"]), _d3(g["inv"]),
          I3(*[int(v) for v in g["size"]]), nc, n, 1, 256, None)
        torch.cuda.synchronize()
        if call == 0:
            assert np.array_equal(key.cpu().numpy(), g["key"])
            assert np.array_equal(idx.cpu().numpy(), g["idx"])
            assert np.array_equal(st.cpu().numpy(), g["start"])
            assert np.array_equal(en.cpu().numpy(), g["end"])
        else:  # reversed input: the same keys, the object order reversed within each cell's stable order
            k = key.cpu().numpy()
            assert np.array_equal(k, g["key"])
            orig = n - 1 - idx.cpu().numpy()  # indices into the original order
            assert np.array_equal(np.sort(orig), np.arange(n))
            assert np.array_equal(g["pos"][orig], pos[idx.cpu().numpy()])
            for c in np.unique(k):
                sel = k == c
                assert np.all(np.diff(idx.cpu().numpy()[sel]) > 0)  # stable: ascending index in each cell
            assert np.array_equal(st.cpu().numpy(), g["start"]) and np.array_equal(en.cpu().numpy(), g["end"])


def test_integration_launchers(lsdem):
    import torch
    L = lsdem.lib
    kick = L.launchParticleVelocityAngularVelocityIntegration
    kick.restype = None
    kick.argtypes = [C.c_void_p] * 7 + [D3, C.c_double, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p]
    drift = L.launchParticlePositionOrientationIntegration
    drift.restype = None
    drift.argtypes = [C.c_void_p] * 4 + [C.c_double, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p]
    g = gold("integration.npz")
    n = len(g["vel"])
    v, w = _dev(g["vel"]), _dev(g["angvel"])
    keep = {k: _dev(g[k]) for k in ("force", "torque", "invm", "quat", "invI")}  # alive until the kernel ran
    kick(_p(v), _p(w), _p(keep["force"]), _p(keep["torque"]), _p(keep["invm"]), _p(keep["quat"]), _p(keep["invI"]),
         _d3(g["g"]), float(g["h"]), n, 1, 64, None)
    torch.cuda.synchronize()
    assert _close(v.cpu().numpy(), g["vel_out"], 1e-14)
    assert _close(w.cpu().numpy(), g["angvel_out"], 1e-13)
    p, q = _dev(g["pos"]), _dev(g["quat"])
    vo, wo = _dev(g["vel_out"]), _dev(g["angvel_out"])
    drift(_p(p), _p(q), _p(vo), _p(wo), float(g["dt"]), n, 1, 64, None)
    torch.cuda.synchronize()
    assert _close(p.cpu().numpy(), g["pos_out"], 1e-15)
    assert _close(q.cpu().numpy(), g["quat_out"], 1e-15, scale=1.0)


def test_wrap_launchers(lsdem):
    import torch
    L = lsdem.lib
    fx, fy = L.launchUpdatePositionOutOfBoundaryXD, L.launchUpdatePositionOutOfBoundaryYD
    for f in (fx, fy):
        f.restype = None
        f.argtypes = [C.c_void_p, D3, D3, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p]
    g = gold("periodic.npz")
    n = len(g["pos"])
    p = _dev(g["pos"])
    fx(_p(p), _d3(g["min"]), _d3(g["max"]), n, 1, 256, None)
    torch.cuda.synchronize()
    assert np.array_equal(p.cpu().numpy(), g["wrap_x"])
    fy(_p(p), _d3(g["min"]), _d3(g["max"]), n, 1, 256, None)
    torch.cuda.synchronize()
    assert np.array_equal(p.cpu().numpy(), g["wrap_xy"])

"""Mass properties on the GPU (lsdem_mass_properties_gpu) against the host routine that
restates LSSolver.h:66-135 loop for loop (lsdem_mass_properties) and against the FP64 oracle:
mass, centroid, inertia and inverse inertia within 1e-12 of their scale (the parallel sums
are ordered differently from the triple loop), and the same bits on a second call."""
import numpy as np
import pytest

from conftest import load_oracle

pytestmark = pytest.mark.gpu


def _templates(lsdem):
    from lsdem_b200 import scenes
    out = [scenes.make_ellipsoid((5e-3, 4e-3, 3e-3), 32, 200)]
    rng = np.random.default_rng(4)
    out += scenes.superquadric_templates(lsdem, rng, 2, (2.0, 8.0), (1e-3, 3e-3), 64, 200, level=4)
    return out


def test_gpu_mass_properties_match_host_and_oracle(lsdem):
    ora = load_oracle()
    for t in _templates(lsdem):
        args = (t["sdf"], t["size"], t["origin"], t["spacing"], 2500.0)
        g = lsdem.mass_properties_gpu(*args)
        h = lsdem.mass_properties(*args)
        o = ora.mass_props(*args)
        assert g["mass"] > 0
        ref = {"mass": o[0], "centroid": o[1:4], "inertia": o[4:10], "inv_inertia": o[10:16]}
        for k in ("mass", "centroid", "inertia", "inv_inertia"):
            gv, hv, rv = np.atleast_1d(g[k]), np.atleast_1d(h[k]), np.atleast_1d(ref[k])
            scale = {"centroid": float(np.max(np.asarray(t["size"]) * t["spacing"]))}.get(k, np.abs(rv).max())
            assert np.abs(gv - hv).max() <= 1e-12 * scale, (k, np.abs(gv - hv).max() / scale)
            assert np.abs(gv - rv).max() <= 1e-12 * scale, k
        again = lsdem.mass_properties_gpu(*args)
        for k in g:
            assert np.array_equal(np.atleast_1d(g[k]), np.atleast_1d(again[k])), k

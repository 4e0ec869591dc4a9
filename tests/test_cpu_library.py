"""CPU-only checks of the C-ABI library: exported symbols, host-side model
building and its reference semantics (no device work)."""
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_oracle

HEADER = ROOT / "include" / "lsdem_b200.h"


def declared_symbols():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(lsdem_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol(lsdem):
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lsdem.lib, n), f"{n} declared in include/lsdem_b200.h but not exported"
    assert sorted(lsdem.EXPORTED) == names, "python binding out of sync with the header"


def test_mass_properties_match_oracle(lsdem):
    ora = load_oracle()
    from lsdem_b200 import scenes
    shp = scenes.make_ellipsoid((5e-3, 4e-3, 3e-3), n_grid=20, n_nodes=100)
    mp = lsdem.mass_properties(shp["sdf"], shp["size"], shp["origin"], shp["spacing"], 2500.0)
    ref = ora.mass_props(shp["sdf"], shp["size"], shp["origin"], shp["spacing"], 2500.0)
    got = np.concatenate([[mp["mass"]], mp["centroid"], mp["inertia"], mp["inv_inertia"]])
    assert np.array_equal(got, ref)  # same IEEE operation order, bit-exact
    vol = 4.0 / 3.0 * np.pi * 5e-3 * 4e-3 * 3e-3
    assert abs(mp["mass"] / (2500.0 * vol) - 1.0) < 0.03


def test_add_ls_particle_reference_semantics(lsdem):
    """LSSolver::addLSParticle: frame moved to the centroid, position shifted by the rotated
    centroid, quaternion normalised twice, stiffness/friction clamped at 0, restitution
    outside (0, 1] set to 1 (LSSolver.h:137-162, LSParticle.h:188-202)."""
    from lsdem_b200 import scenes
    shp = scenes.make_ellipsoid((5e-3, 4e-3, 3e-3), n_grid=16, n_nodes=64)
    nodes = shp["nodes"] + np.array([1e-3, -2e-3, 0.5e-3])      # off-centre frame
    origin = shp["origin"] + np.array([1e-3, -2e-3, 0.5e-3])
    sv = lsdem.Solver()
    q = np.array([2.0, 0.2, -0.4, 0.1])
    i0 = sv.add_ls_particle(nodes, shp["sdf"], shp["size"], origin, shp["spacing"], [0.1, 0.2, 0.3], [0, 0, 0],
                            [0, 0, 0], q, -5.0, 3.0, -1.0, 1.7, 2500.0)
    i1 = sv.add_ls_particle(nodes, shp["sdf"], shp["size"], origin, shp["spacing"], [0.2, 0.2, 0.3], [0, 0, 0],
                            [0, 0, 0], q, 1e5, 8e4, 0.5, 0.0, 2500.0)
    assert (i0, i1) == (0, 1)
    assert sv.num(4) == 1, "identical templates are stored once"
    pp = sv.particle_params()
    assert pp["kn"][0] == 0.0 and pp["ks"][0] == 3.0 and pp["mu"][0] == 0.0 and pp["e"][0] == 1.0
    assert pp["e"][1] == 1.0
    mp = lsdem.mass_properties(shp["sdf"], shp["size"], origin, shp["spacing"], 2500.0)
    st = sv.state()
    qn = q / np.sqrt(q @ q)
    assert np.allclose(st["quat"][0], qn, rtol=0, atol=1e-15)
    c = mp["centroid"]
    t = 2.0 * np.cross(qn[1:], c)
    rc = c + qn[0] * t + np.cross(qn[1:], t)
    assert np.allclose(st["pos"][0], np.array([0.1, 0.2, 0.3]) + rc, rtol=0, atol=1e-15)
    s = sv.shape(0)
    assert np.allclose(s["nodes"], nodes - c, rtol=0, atol=1e-18)
    assert np.allclose(s["origin"], origin - c, rtol=0, atol=1e-18)
    assert pp["radius"][0] == np.max(np.linalg.norm(s["nodes"], axis=1))
    assert pp["inv_mass"][0] == 1.0 / mp["mass"]


def test_invalid_input_errors(lsdem):
    sv = lsdem.Solver()
    with pytest.raises(lsdem.LSDEMError) as e:
        sv.add_shape(np.zeros((4, 3)), np.zeros(8), [1, 2, 2], [0, 0, 0], 1.0)
    assert e.value.code == 1 and "grid size" in str(e.value)
    with pytest.raises(lsdem.LSDEMError) as e:
        sv.add_shape(np.zeros((4, 3)), np.zeros(8), [2, 2, 2], [0, 0, 0], 0.0)
    assert e.value.code == 1
    with pytest.raises(lsdem.LSDEMError) as e:
        sv.step(1e-6, 1)
    assert e.value.code == 4
    with pytest.raises(lsdem.LSDEMError) as e:
        sv.initialize([0, 0, 0], [1, 0, 1])
    assert e.value.code == 1 and "domain" in str(e.value)
    # training options of the learned SDF: the trust band must lie inside the clip range
    sv.set_learned_training(-0.1, 0.3, 0.8)
    for bad in ((-0.01, 0.5, 0.5), (-0.25, 0.05, 0.5), (-0.25, 0.5, 1.5)):
        with pytest.raises(lsdem.LSDEMError) as e:
            sv.set_learned_training(*bad)
        assert e.value.code == 1 and "clip_lo" in str(e.value)


def test_bond_stiffness_from_beam_theory(lsdem):
    """VBondedInteraction::add: B1 = EA/L, B2 = L^2 Ks, B4 = GJ/L, B3 = EI/L - B2/4 - B4/2
    (VBondedInteraction.h:133-148); local frames normalised."""
    sv = lsdem.Solver()
    shp = {"nodes": np.array([[1e-3, 0, 0], [-1e-3, 0, 0]]), "sdf": np.linspace(-1, 1, 8), "size": [2, 2, 2],
           "origin": [-1e-3] * 3, "spacing": 2e-3}
    sid = sv.add_shape(shp["nodes"], shp["sdf"], shp["size"], shp["origin"], shp["spacing"])
    sv.add_particles([sid, sid], [[0, 0, 0], [3e-3, 0, 0]], [[1, 0, 0, 0], [0.9, 0.1, 0, 0]], 1.0,
                     np.tile([1.0, 1.0, 1.0, 0, 0, 0], (2, 1)), 1e5, 8e4, 0.5, 0.5)
    sv.add_bond(0, 1, [1.5e-3, 0, 0], [-2.0, 0, 0], 1e-3, 1e-3, 1e8, 0.3)
    sv.add_bond(0, 5, [1.5e-3, 0, 0], [-1.0, 0, 0], 1e-3, 1e-3, 1e8, 0.3)  # out of range: ignored
    with pytest.raises(lsdem.LSDEMError):
        sv.add_bond(0, 1, [1.5e-3, 0, 0], [-1.0, 0, 0], 1e-3, 1e-3, 1e8, 0.5)  # Poisson ratio >= 0.5
    assert sv.num(2) == 1
    b = sv.bonds()
    assert b["ids"].tolist() == [[0, 1]] and b["bonded"].tolist() == [1]


def test_compat_launchers_exported(lsdem):
    """Every launcher include/lsdem_compat.h declares (the reference's extern "C" names) is
    exported by the library."""
    txt = (ROOT / "include" / "lsdem_compat.h").read_text()
    names = sorted(set(re.findall(r"^void\s+(launch\w+)\s*\(", txt, flags=re.M)))
    assert len(names) == 5
    for n in names:
        assert hasattr(lsdem.lib, n), f"{n} declared in include/lsdem_compat.h but not exported"


def test_host_model_of_a_scene_equals_the_solvers(lsdem):
    """The oracle model built on the host from a scene dict (model_from_scene: the reference
    arm of the benchmark prepares its sample without the CUDA library) holds the same
    per-particle constants as the solver's set-up (lsdem_add_particles, LSParticle.h:115-212)."""
    from lsdem_b200 import scenes
    ora = load_oracle()
    T = scenes.unit_templates(n_grid=12, n_nodes=60)
    rng = np.random.default_rng(3)
    n = 40
    tm = []
    for t in T:
        mp = lsdem.mass_properties(t["sdf"], t["size"], t["origin"], t["spacing"], 1.0)
        tm.append(dict(t, nodes=t["nodes"] - mp["centroid"], origin=t["origin"] - mp["centroid"]))
    sc = {"templates": tm, "shape": rng.integers(0, 4, n).astype(np.int32), "scale": rng.uniform(1e-3, 3e-3, n),
          "pos": rng.uniform(0, 0.05, (n, 3)), "quat": scenes.random_quaternions(rng, n), "vel": np.zeros((n, 3)),
          "inv_mass": rng.uniform(1, 2, n), "inv_inertia": rng.uniform(1, 2, (n, 6)), "kn": 1e5, "ks": 8e4,
          "mu": 0.5, "e": 0.6, "min": np.zeros(3), "max": np.full(3, 0.05), "gravity": np.zeros(3), "periodic": 0,
          "walls": [scenes.plane_wall(0.05, [0.025, 0.025, 0.0])]}
    sv = lsdem.Solver()
    scenes.load_polydisperse(sv, sc)
    pp = sv.particle_params()
    m = ora.model_from_scene(sc)["particles"]
    for k in ("radius", "origin", "invh", "scale", "kn", "ks", "mu", "e"):
        assert np.array_equal(np.asarray(m[k]), pp[k]), k
    assert np.allclose(m["quat"], sv.state()["quat"], rtol=0, atol=1e-15)
    sv.close()


def test_settling_domain_is_a_cube_with_the_packing_at_its_fraction(lsdem):
    """The large-scale workload's domain: a cube whose lower part holds the packing at the
    stated solid fraction and whose top holds the reserve slab, so that no body starts above
    the domain's y extent (the image-key rule tests z against the y bound)."""
    import math
    from lsdem_b200 import scenes
    for n, b, sph in ((2_000_000, 2.9e-3, 4.0e-8), (200_000, 2.9e-3, 4.0e-8), (4000, 2.5e-3, 3.0e-8)):
        vol = n * sph / 1.9  # bounding spheres hold ~1.9 x the body volume
        L, slab = scenes.settling_geometry(vol, 0.25, n, sph, b, 0.02)
        assert abs(L * L * (L - slab) * 0.25 / vol - 1.0) < 1e-9
        assert slab == pytest.approx(0.02 * n * sph / 0.2 / (L * L) + 2 * b, rel=1e-12)
        assert 2 * b < slab < 0.5 * L
        assert L > (vol / 0.25) ** (1.0 / 3.0)

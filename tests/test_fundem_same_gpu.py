"""Configs 0 and 2 on the reference solver's own CUDA build and on this solver, same GPU, same app.

tests/apps/c0_bench.cpp is written against the LSSolver API only. oracle/build_ref.sh builds
it against the reference (FunDEM/kernel/LSSolver.h and its kernel sources, Release flags,
sm_100a) into oracle/_ref/c0_bench_fundem; this test builds the same source against the
drop-in include/kernel/LSSolver.h (FP64 form, the reference's arithmetic). Both run the
config-0 scene (2,000 identical ellipsoids, 32^3 grids, 1,000 nodes, floor wall) from one
scene file; each reports the device time of a fixed window of steps, measured with CUDA
events recorded from the external-force hook (called by both solvers every step between
the forces and the second half kick), and the particle velocities at the window's end.

Checked: the velocities agree to FP64 round-off (same algorithm, same inputs), and the output
frames the two solvers write (the reference's VTU files: surface-node mesh, particles, contacts,
bonds, walls, wall contacts) are the same files with the same XML structure and equal arrays
(float32 values to 1e-5 of the scale, integers exact, contacts as sets). The two timings are
printed (they are reported, not asserted).

Config 2 (tests/apps/c2_bench.cpp, oracle/_ref/c2_bench_fundem): aligned ellipsoids (2, 1.6,
1.2 mm, 32^3 grids, 1,000 nodes) on the jittered HCP lattice with a V-bond to every lattice
neighbour, a floor and a top wall moving down at 0.1 m/s, added through addLSParticle (density),
addWall, setFixedVelocityToWall and addBondedInteraction, at a reduced count of 8,000
particles by default: the reference keeps a full SDF copy per particle in host and device
memory (Q14), 2.1 GB here, 13 GB at the configuration's 50,000 (LSDEM_C2_PARTICLES=50000 runs
that size).
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

FUNDEM = ROOT / "oracle" / "_ref" / "c0_bench_fundem"
OURS = ROOT / "lsdem2.0_b200" / "_build" / "c0_bench_b200"
APP = ROOT / "tests" / "apps" / "c0_bench.cpp"
FUNDEM2 = ROOT / "oracle" / "_ref" / "c2_bench_fundem"
OURS2 = ROOT / "lsdem2.0_b200" / "_build" / "c2_bench_b200"
APP2 = ROOT / "tests" / "apps" / "c2_bench.cpp"


def build_ours(app=APP, out=OURS) -> None:
    if out.exists() and out.stat().st_mtime >= max(app.stat().st_mtime,
                                                    (ROOT / "include" / "kernel" / "LSSolver.h").stat().st_mtime):
        return
    cmd = ["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include"), "-I", str(ROOT / "include" / "kernel"), str(app),
           "-L", str(ROOT / "lsdem2.0_b200"), "-llsdem_b200", "-Xlinker", "-rpath", "-Xlinker",
           str(ROOT / "lsdem2.0_b200"), "-o", str(out)]
    out.parent.mkdir(exist_ok=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def write_scene(path, sc, nsteps, k0, k1):
    from lsdem_b200 import scenes
    scenes.write_c0_app_scene(path, sc, nsteps, k0, k1)


def _structure(path):
    """Element tags and attributes of a VTU file, array payloads left out."""
    import xml.etree.ElementTree as ET
    out = []
    for el in ET.parse(path).getroot().iter():
        attrs = dict(el.attrib)
        if el.tag == "DataArray" and attrs.get("format") == "ascii":
            attrs["value"] = (el.text or "").strip()
        out.append((el.tag, tuple(sorted(attrs.items()))))
    return out


def compare_frames(dir_ref, dir_ours, scale):
    """The last frame's files of both solvers: the same files, the same XML structure, equal
    arrays (float32 casts of FP64 values that agree to round-off), contacts as sets."""
    from helpers import read_vtu
    ref = {p.relative_to(dir_ref): p for p in dir_ref.rglob("*.vtu")}
    ours = {p.relative_to(dir_ours): p for p in dir_ours.rglob("*.vtu")}
    assert sorted(ref) == sorted(ours), (sorted(ref), sorted(ours))
    last = max(int(p.stem.split("_")[-1]) for p in ref)
    checked = []
    for rel in sorted(ref):
        if int(rel.stem.split("_")[-1]) != last:
            continue
        assert _structure(ref[rel]) == _structure(ours[rel]), rel
        a, b = read_vtu(ref[rel]), read_vtu(ours[rel])
        assert a["n_points"] == b["n_points"] and a["n_cells"] == b["n_cells"], rel
        if rel.name.startswith("LSInteraction"):
            oa, ob = np.lexsort(a["points"].T[::-1]), np.lexsort(b["points"].T[::-1])
        else:
            oa = ob = slice(None)
        for k, v in a.items():
            if k in ("n_points", "n_cells", "connectivity", "offsets", "types") and rel.name.startswith("LSInteraction"):
                continue
            va, vb = np.asarray(v), np.asarray(b[k])
            if va.ndim and len(va) == a["n_points"] and va.size:
                va, vb = va[oa], vb[ob]
            if va.dtype.kind == "f":
                s = scale if k in ("points",) else max(float(np.abs(va).max(initial=0.0)), 1e-30)
                assert np.abs(va.astype(np.float64) - vb).max(initial=0.0) <= 1e-5 * s, (rel, k)
            else:
                assert np.array_equal(va, vb), (rel, k)
        checked.append(str(rel))
    return checked


def run(binary, scene, outdir, result):
    r = subprocess.run([str(binary), str(scene), str(outdir), str(result)], capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    from lsdem_b200 import scenes
    return scenes.read_c0_app_result(result)


@pytest.mark.skipif(not FUNDEM.exists(), reason="oracle/_ref/c0_bench_fundem not built (needs the reference tree)")
@pytest.mark.skipif(shutil.which("nvcc") is None and not OURS.exists(), reason="nvcc not available")
def test_config0_same_gpu(lsdem, tmp_path):
    from lsdem_b200 import scenes
    build_ours()
    sc = scenes.ellipsoid_falling()
    nsteps, k0, k1 = 2000, 200, 1900
    scene = tmp_path / "c0.bin"
    write_scene(scene, sc, nsteps, k0, k1)
    res = {}
    for name, binary in (("fundem", FUNDEM), ("b200", OURS)):
        out = tmp_path / name
        out.mkdir()
        res[name] = run(binary, scene, out, tmp_path / f"{name}.res")
    (s0, w0, ms0, v0), (s1, w1, ms1, v1) = res["fundem"], res["b200"]
    assert s0 >= k1 and s1 >= k1 and w0 == w1 == k1 - k0
    assert v0.shape == v1.shape == (len(sc["pos"]), 3)
    vmax = np.abs(v0).max()
    assert np.abs(v1 - v0).max() <= 1e-9 * vmax, np.abs(v1 - v0).max() / vmax
    files = compare_frames(tmp_path / "fundem_phase1", tmp_path / "b200_phase1", float(np.abs(sc["max"]).max()))
    print("frame files equal to the reference build's:", ", ".join(files))
    print(f"config 0, {len(sc['pos'])} ellipsoids, steps {k0}..{k1}: reference build {ms0 / w0:.4f} ms/step, "
          f"this solver (FP64) {ms1 / w1:.4f} ms/step, ratio {ms0 / ms1:.2f}x")


def write_scene_c2(path, sc, nsteps, k0, k1):
    t = sc["templates"][0]
    n = len(sc["pos"])
    d = lambda a: np.ascontiguousarray(a, np.float64).tobytes()
    i32 = lambda *v: struct.pack(f"<{len(v)}i", *v)
    tris = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    b = sc["bonds"]
    with open(path, "wb") as fh:
        fh.write(b"LSDEMC2\0")
        fh.write(i32(len(t["nodes"]), *[int(v) for v in t["size"]]) + d([t["spacing"]]) + d(t["origin"]))
        fh.write(d(t["nodes"]) + d(t["sdf"]))
        fh.write(i32(n) + d(sc["pos"]) + d(sc["quat"]) + d(sc["vel"]))
        fh.write(d([sc["kn"], sc["ks"], sc["mu"], sc["e"], 2500.0]))
        fh.write(i32(len(sc["walls"])))
        for w in sc["walls"]:
            fh.write(i32(*[int(v) for v in w["size"]]) + d([w["spacing"]]) + d(w["origin"]) + d(w["sdf"]))
            fh.write(d(w["pos"]) + d(w["quat"]) + d([w["mu"], w["e"]]))
            fh.write(d(w["vel"] if w.get("vel") is not None else np.zeros(3)))
            fh.write(i32(len(w["verts"]), len(tris)) + d(w["verts"]) + tris.tobytes())
        nb = len(b["master"])
        ids = np.stack([b["master"], b["slave"]], 1).astype(np.int32)
        fh.write(i32(nb) + ids.tobytes() + d(b["point"]) + d(b["normal"]) + d(b["radius"]) + d(b["length"]))
        fh.write(d(b["tensile"]) + d(b["cohesion"]) + d([b["youngs"], b["poisson"], b["mu"]]))
        fh.write(d([sc["dt"]]) + d(sc["min"]) + d(sc["max"]) + d(sc["gravity"]))
        fh.write(i32(nsteps, k0, k1))


@pytest.mark.skipif(not FUNDEM2.exists(), reason="oracle/_ref/c2_bench_fundem not built (needs the reference tree)")
@pytest.mark.skipif(shutil.which("nvcc") is None and not OURS2.exists(), reason="nvcc not available")
def test_config2_bonded_same_gpu(lsdem, tmp_path):
    from lsdem_b200 import scenes
    build_ours(APP2, OURS2)
    sc = scenes.bonded_hcp(lsdem, n=int(os.environ.get("LSDEM_C2_PARTICLES", "8000")))
    # frames are written at steps 0, 119 and 120: the window (20, 110] times steps only
    nsteps, k0, k1 = 120, 20, 110
    scene = tmp_path / "c2.bin"
    write_scene_c2(scene, sc, nsteps, k0, k1)
    res = {}
    for name, binary in (("fundem", FUNDEM2), ("b200", OURS2)):
        out = tmp_path / name
        out.mkdir()
        res[name] = run(binary, scene, out, tmp_path / f"{name}.res")
    (s0, w0, ms0, v0), (s1, w1, ms1, v1) = res["fundem"], res["b200"]
    assert s0 >= k1 and s1 >= k1 and w0 == w1 == k1 - k0
    assert v0.shape == v1.shape == (len(sc["pos"]), 3)
    vmax = np.abs(v0).max()
    err = np.abs(v1 - v0).max() / vmax
    assert err <= 1e-6, err
    files = compare_frames(tmp_path / "fundem_phase1", tmp_path / "b200_phase1", float(np.abs(sc["max"]).max()))
    print("frame files equal to the reference build's:", ", ".join(files))
    print(f"config 2 (bonded, {len(sc['pos'])} ellipsoids, {len(sc['bonds']['master'])} bonds), steps {k0}..{k1}: "
          f"reference build {ms0 / w0:.4f} ms/step, this solver (FP64) {ms1 / w1:.4f} ms/step, "
          f"ratio {ms0 / ms1:.2f}x, velocity difference {err:.2e} of the largest")


@pytest.mark.skipif(not FUNDEM.exists(), reason="oracle/_ref/c0_bench_fundem not built (needs the reference tree)")
@pytest.mark.skipif(shutil.which("nvcc") is None and not OURS.exists(), reason="nvcc not available")
def test_two_phases_same_gpu(lsdem, tmp_path):
    """Two solve() phases, the floor's angular velocity set between them (as tutorial 2
    does), on a dense scene whose contacts persist across the phase boundary: the
    reference keeps its state, forces and contact history between phases; the velocities
    after 30 steps of the second phase agree with the reference build's to FP64 round-off."""
    from helpers import dense_ellipsoid_scene
    from lsdem_b200 import scenes
    build_ours()
    sc = dense_ellipsoid_scene(scenes, n=64, seed=23, vel_sigma=0.2)
    n1, n2 = 40, 40
    k0, k1 = 5, n1 + 30
    scene = tmp_path / "c0p.bin"
    scenes.write_c0_app_scene(scene, sc, n1, k0, k1, nsteps2=n2, floor_wz=20.0)
    res = {}
    for name, binary in (("fundem", FUNDEM), ("b200", OURS)):
        out = tmp_path / name
        out.mkdir()
        res[name] = run(binary, scene, out, tmp_path / f"{name}.res")
    (s0, w0, ms0, v0), (s1, w1, ms1, v1) = res["fundem"], res["b200"]
    assert s0 == s1 == n1 + n2 and w0 == w1 == k1 - k0
    vmax = np.abs(v0).max()
    err = np.abs(v1 - v0).max() / vmax
    assert err <= 1e-9, err
    print(f"two phases: velocity difference {err:.2e} of the largest")

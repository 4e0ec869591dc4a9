"""Benchmark of the level-set DEM time step (particle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload scale|polydisperse|small|bonded|drum]
                    [--form fp32-bf16-learned|fp32-bf16|fp32-fp16|fp64]

Workload (default "scale", the largest configuration that fits one GPU and the one the
"plain grid vs FP32 + learned SDF" comparison is stated for): 2,000,000 particles from 16
seeded superquadrics (exponents uniform 2-6, semi-axes uniform 1-2.5 mm, 1,500 surface
nodes, 48-node grids along the longest axis from the mesh distance of each shape's
20,480-triangle mesh), periodic in x and y with a floor and a ceiling, settling under
gravity from a random loose packing (solid fraction 0.25), linear contact (kn 1e5,
kt 0.8 kn, mu 0.5, e 0.6), dt 5e-7 s. Synthetic, seeded (no dataset).

The headline form is FP32 + learned SDF: one 3-64-64-1 SiLU network per shape, trained on
the GPU, screens nodes before the FP32 screen on BF16 grid templates; both only reject
nodes that measured or proven error bounds show the FP64 test rejects, and the remaining
nodes and all contacts are evaluated in FP64 (positions, integration, spring history stay
FP64). The same run times the plain grid form (FP64, the reference's arithmetic, bit-exact
pair lists) and the FP32 grid screen without the network, and states each FP32 form's force,
torque and energy error against the FP64 path from the same state.

Other workloads (--workload; each a stated configuration of the method, synthetic and seeded):
"polydisperse" 100,000 particles from 4 templates (48^3 grids, 2,000 nodes), log-normal sizes,
0.1 m triply periodic cube, velocities N(0, 0.1 m/s); "small" 2,000 ellipsoids (5, 4, 3 mm)
falling on a floor, 32^3 grids, 1,000 nodes, dt 1e-6 s; "bonded" 50,000 aligned ellipsoids (2,
1.6, 1.2 mm) on a jittered HCP lattice with ~286,000 V-bonds, floor and a top wall moving down
at 0.1 m/s, dt 2e-7 s; "drum" 500,000 particles from 64 superquadrics (64^3 grids, 1,500
nodes) in a drum of radius 0.15 m and length 0.1 m turning at 30 rpm (all shapes scaled by one
factor so that they fit the drum).

One step = one full time step (half kick, drift, cell sort, candidates,
narrowphase + contact forces, periodic images, half kick) of the whole scene. The
cell sort and the 27-cell candidate walk run in the steps that rebuild the
neighbour lists (when a particle moved 0.04 of the largest bounding radius since
the last rebuild; a periodic wrap counts); the other steps test each particle's
list and find the same candidate pairs in the same order (lsdem_set_neighbour_lists,
tests/test_gpu_neighbour_lists.py). Every step runs the narrowphase and the
contact forces of every candidate pair.
Multi-GPU: independent replicas (the step has no data-parallel split in this
build), one process per GPU, timing = max over ranks, value = total over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent

FORMS = {"fp32-bf16": 2, "fp32-fp16": 1, "fp64": 0, "fp32-bf16-learned": 2}
DTYPE = {"fp32-bf16": "f32 screen on bf16 SDF, f64 contacts", "fp32-fp16": "f32 screen on fp16 SDF, f64 contacts",
         "fp64": "f64", "fp32-bf16-learned": "bf16 network + f32 screen on bf16 SDF, f64 contacts"}
LEARN = {"iterations": 12000, "batch": 4096, "samples": 1 << 17, "lr": 1e-2}
# training target clipped to [-0.1, 0.3] R, 80 % of the samples near the surface (the smallest
# one-sided error of the settings compared on the large-scale workload's 16 shapes)
LEARN_OPTS = {"clip_lo": -0.1, "clip_hi": 0.3, "near_fraction": 0.8}


def _package():
    pkg = ROOT / "lsdem2.0_b200"
    spec = importlib.util.spec_from_file_location("lsdem_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lsdem_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _bf16_peak():
    """Dense BF16 tensor throughput (TFLOP/s): the measured burst figure (the network pass
    is timed on its own launches), else the fallback."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


# FLOP per network evaluation: layer 1 (3 x 64 multiply-adds + bias), the layer-2 MMA
# (64 x 64 multiply-adds), the output layer (64 multiply-adds): 2 x (192 + 4096 + 64) = 8704.
NET_FLOP = 8704


# Algorithmic bytes of the narrowphase kernel of each form.
# FP64 form, k_narrowphase (detection and forces fused): per owner particle (pose,
# velocities, slot counts, force/torque write: 208 B), per candidate pair (partner id,
# pose, velocities, shape and material scalars, segment bookkeeping, reaction atomics:
# 236 B) and per contact (node id, FP64 spring read and write, history lookup: 56 B).
# Precision forms, k_screen_f (the screen; contacts are evaluated by the separate
# FP64 contact pass): per owner particle (pose, scale, shape, slot count: 72 B) and
# per candidate pair (partner id, pose, radius, grid origin and spacing, shape,
# segment words: 120 B).
B_PARTICLE = 208
B_PAIR = 236
B_CONTACT = 56
B_PARTICLE_SCREEN = 72
B_PAIR_SCREEN = 120
# whole-step algorithmic bytes per particle (state, keys, sort, candidates)
B_STEP_PARTICLE = 448
# What bounds the screen: an ncu full-set capture of k_screen_f<1, 2, 0> (particle pairs,
# FP32/BF16 form) on the settling configuration at 200,000 particles (two launches alike).
SCREEN_CAPTURE = {
    "case": "settling configuration at 200,000 particles, FP32/BF16 form, particle-pair screen, steps 2-3",
    "dram_bytes_per_launch": 38.35e6,
    # 72 B x 200,000 owners + 120 B x ~51,500 particle pairs (of 55,400 pairs of all kinds)
    "algorithmic_bytes_per_launch": 72 * 200_000 + 120 * 51_500,
    "issue_active": 0.616, "warps_active": 0.447, "warps_active_limit": 0.50,
    "leading_stall": "long_scoreboard (5.5 warps per issue): dependent L2 loads",
    "dram_throughput": 0.039,
}


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def mark(self, start: bool):
        """Brackets the timed region (host clock, after a device synchronize)."""
        if start:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
        rows = [r for t, r in self.rows if t0 <= t <= t1]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if len(r) > 3 + k and r[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_scene(lsdem, workload: str, rank: int, particles: int = 100_000, device: int = 0):
    from lsdem_b200 import scenes
    if workload == "small":
        sc = scenes.ellipsoid_falling(seed=scenes.seed_for(0) + rank)
        return sc, {"workload": "ellipsoids-2000-floor", "particles": 2000, "nodes_per_particle": 1000,
                    "sdf_grid": "32^3", "box_m": [0.2, 0.2, 0.4], "dt_s": 1e-6}
    if workload == "bonded":
        sc = scenes.bonded_hcp(lsdem, seed=scenes.seed_for(2) + rank)
        return sc, {"workload": "bonded-hcp-50k-ellipsoids", "particles": len(sc["pos"]),
                    "bonds": len(sc["bonds"]["master"]), "nodes_per_particle": 1000, "sdf_grid": "32^3",
                    "lattice": "HCP mapped to aligned ellipsoids (2, 1.6, 1.2 mm), 5% gap, 2% jitter",
                    "walls": "floor + top wall at -0.1 m/s", "dt_s": sc["dt"]}
    if workload in ("drum", "scale"):
        t0 = time.perf_counter()
        if workload == "drum":
            sc = scenes.drum(lsdem, n=particles if particles != 100_000 else 500_000,
                             seed=scenes.seed_for(3) + rank, device=device)
        else:
            sc = scenes.settling_box(lsdem, n=particles if particles != 100_000 else 2_000_000,
                                     seed=scenes.seed_for(4) + rank, device=device)
        t_gen = time.perf_counter() - t0
        iters = scenes.resolve_deep_overlaps(lsdem, sc, device=device)
        n = len(sc["pos"])
        T = sc["templates"]
        cfg = {"workload": (f"drum-{n}-superquadrics-64" if workload == "drum" else f"settling-{n}-superquadrics-16"),
               "particles": n, "templates": len(T), "nodes_per_particle": len(T[0]["nodes"]),
               "sdf_grid": "x".join(str(int(v)) for v in np.max([t["size"] for t in T], axis=0)) + " (largest)",
               "sdf_from": "mesh distance of 20480-triangle superquadric meshes, built on the GPU",
               "setup_s": round(t_gen, 1), "dt_s": sc["dt"],
               "initial_state": (f"random sequential addition, deep overlaps re-placed ({iters} passes, "
                                 f"{sc.get('reserve_placed', 0)} bodies to the reserve box)")}
        if workload == "drum":
            cfg.update(drum="R 0.15 m, L 0.1 m, 30 rpm about x", size_factor=round(float(sc["size_factor"]), 4),
                       fill="solid fraction 0.22 of the loading box")
        else:
            cfg.update(box_m=[round(float(v), 4) for v in sc["max"]], periodic="xy", walls="z",
                       solid_fraction=sc["solid_fraction"])
        return sc, cfg
    cache = ROOT / "_build" / "templates_48_2000.npz"
    if cache.exists():
        T = list(np.load(cache, allow_pickle=True)["T"])
    else:
        T = scenes.unit_templates(48, 2000)
        cache.parent.mkdir(exist_ok=True)
        np.savez(cache, T=np.array(T, dtype=object))
    box = 0.1 * (particles / 1e5) ** (1.0 / 3.0)
    sc = scenes.polydisperse_periodic(lsdem, n=particles, box=box, seed=scenes.seed_for(1) + rank, templates=T)
    # deep initial overlaps (many surface nodes inside a neighbour) would exceed the stability
    # limit of the explicit step; re-place those particles, keep shallow contacts
    iters = scenes.resolve_deep_overlaps(lsdem, sc, device=device)
    name = ("polydisperse-100k-4templates-periodic" if particles == 100_000
            else f"polydisperse-{particles}-4templates-periodic")
    return sc, {"workload": name, "particles": particles, "nodes_per_particle": 2000, "sdf_grid": "48^3",
                "templates": 4, "size": "lognormal(median 2 mm, sigma 0.25)", "box_m": round(box, 6),
                "periodic": "xyz", "dt_s": 5e-7,
                "initial_state": f"random sequential addition, deep overlaps re-placed ({iters} passes)"}


def load(lsdem, sc, workload, device, prec, learned=False, info=None, record=False):
    """A solver of the scene in the given form; started from the settled state when the
    scene carries one (sc["snapshot"], written by settle())."""
    from lsdem_b200 import scenes
    sv = lsdem.Solver(device=device)
    if workload == "small":
        scenes.load_into(sv, sc)
    else:
        scenes.load_polydisperse(sv, sc)
    sv.set_precision(prec)
    if record:
        sv.set_record_contacts(True)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    if learned:
        t0 = time.perf_counter()
        sv.set_learned_training(**LEARN_OPTS)
        loss, err = sv.train_learned_sdf(**LEARN)
        sv.set_learned_sdf(True)
        if info is not None:
            info["training"] = dict(LEARN, **LEARN_OPTS, seconds=round(time.perf_counter() - t0, 3), loss=loss.tolist(),
                                    err_over_R=[sv.learned_sdf(k)[1]["err"] / sv.learned_sdf(k)[1]["R"]
                                                for k in range(len(loss))],
                                    err_in_over_R=[sv.learned_sdf(k)[1]["err_in"] / sv.learned_sdf(k)[1]["R"]
                                                   for k in range(len(loss))],
                                    threshold_h=[sv.learned_sdf(k)[1]["threshold_h"] for k in range(len(loss))])
    if sc.get("snapshot"):
        sv.snapshot_load(sc["snapshot"])
    return sv


def settle(lsdem, sc, workload, device, steps, gravity_factor=1.0, relax=2000, chunk=2000):
    """Steps the scene `steps` times in the FP32/BF16 form (untimed) under gravity_factor
    times its gravity, then `relax` steps under its own gravity (from the state reached),
    and saves the state and contact history as the common starting state of every timed
    form (a compacted, contact-dense packing instead of the random placement). Returns
    node contacts per particle."""
    import tempfile
    g = np.asarray(sc["gravity"], np.float64)
    sv = load(lsdem, dict(sc, gravity=g * gravity_factor), workload, device, 2)
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        sv.step(sc["dt"], k)
        done += k
    path = Path(tempfile.mkdtemp(prefix="lsdem_settled_")) / "state.snp"
    if relax > 0 and gravity_factor != 1.0:
        sv.snapshot_save(path)
        sv.close()
        sv = load(lsdem, dict(sc, snapshot=str(path)), workload, device, 2)
        done = 0
        while done < relax:
            k = min(chunk, relax - done)
            sv.step(sc["dt"], k)
            done += k
    contacts = sv.step_stats()["contacts"]
    sv.snapshot_save(path)
    n = sv.n_particles
    sv.close()
    sc["snapshot"] = str(path)
    return contacts / n


def _energies(lsdem, sv):
    """Kinetic energy (translation + rotation) of the state and elastic energy stored in the
    contacts (normal + tangential terms of every particle, wall and image contact)."""
    st = sv.state()
    pp = sv.particle_params()
    im = pp["inv_mass"]
    live = im > 0
    ke = 0.5 * float(np.sum((st["vel"] ** 2).sum(1)[live] / im[live]))
    q = st["quat"]
    w0, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w0 * z), 2 * (x * z + w0 * y)], 1),
                  np.stack([2 * (x * y + w0 * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w0 * x)], 1),
                  np.stack([2 * (x * z - w0 * y), 2 * (y * z + w0 * x), 1 - 2 * (x * x + y * y)], 1)], 1)
    wb = np.einsum("nji,nj->ni", R, st["angvel"])  # body-frame angular velocity
    ii = pp["inv_inertia"]
    inv = np.stack([np.stack([ii[:, 0], ii[:, 3], ii[:, 4]], 1), np.stack([ii[:, 3], ii[:, 1], ii[:, 5]], 1),
                    np.stack([ii[:, 4], ii[:, 5], ii[:, 2]], 1)], 1)
    ok = live & (np.abs(np.linalg.det(inv)) > 0)
    Lb = np.linalg.solve(inv[ok], wb[ok][:, :, None])[:, :, 0]
    ke += 0.5 * float(np.sum((wb[ok] * Lb).sum(1)))
    ec = 0.0
    for kind in (lsdem.CONTACT_PARTICLE, lsdem.CONTACT_WALL, lsdem.CONTACT_GHOST):
        c = sv.contacts(kind, geometry=True)
        ec += float(np.sum(c["en_n"]) + np.sum(c["en_s"]))
    return ke, ec


def force_error(lsdem, sc, workload, device, prec, warm=20, learned=False):
    """Force / torque / energy error of an FP32 form against the FP64 path, from the same
    state: both run `warm` FP64 steps, then one step each; forces are captured in the external
    hook, kinetic and contact energies read after the step."""
    import torch
    out = {}
    sv = load(lsdem, sc, workload, device, 0)
    sv.step(sc["dt"], warm)
    st = sv.state()
    sv.close()
    for p in (0, prec):
        sv = load(lsdem, sc, workload, device, p, learned=learned and p != 0, record=True)
        sv.set_state(pos=st["pos"], vel=st["vel"], angvel=st["angvel"], quat=st["quat"])
        box = {}
        sv.step(sc["dt"], 1, hook=lambda t, sv=sv: box.update(sv.state()))
        torch.cuda.synchronize()
        box["energy"] = _energies(lsdem, sv)
        out[p] = box
        sv.close()
    F64, T64 = out[0]["force"], out[0]["torque"]
    (k64, e64), (kp, ep) = out[0]["energy"], out[prec]["energy"]
    return {"force_l2": float(np.linalg.norm(out[prec]["force"] - F64) / np.linalg.norm(F64)),
            "torque_l2": float(np.linalg.norm(out[prec]["torque"] - T64) / np.linalg.norm(T64)),
            "force_max": float(np.abs(out[prec]["force"] - F64).max() / np.abs(F64).max()),
            "kinetic_energy_rel": abs(kp - k64) / k64 if k64 > 0 else None,
            "contact_energy_rel": abs(ep - e64) / e64 if e64 > 0 else None}


SAMPLE_PARTICLES = 4000  # host sample of the large-scale workload (CPU baseline, reference arm)


ORACLE_BUILD = {"flags": "-O3 -fopenmp -ffp-contract=off (portable x86-64 build)"}


def _oracle():
    """The FP64 oracle for the CPU timing, built here with -march=native for this host's cores
    (the checker's portable build when that fails)."""
    if "oracle" not in sys.modules and not os.environ.get("LSDEM_ORACLE_LIB"):
        import tempfile
        out = Path(tempfile.mkdtemp(prefix="lsdem_oracle_")) / "liboracle_native.so"
        r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "native", f"NATIVE_OUT={out}"],
                           capture_output=True, text=True)
        if r.returncode == 0 and out.exists():
            os.environ["LSDEM_ORACLE_LIB"] = str(out)
            ORACLE_BUILD["flags"] = "-O3 -march=native -fopenmp -ffp-contract=off (built on this host)"
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as ora  # the checker, timed as the CPU baseline / reference arm only
    return ora


def _scenes_host():
    """The scenes module loaded on its own (it imports nothing of the package), so that the
    reference arm prepares its sample without loading the CUDA library."""
    spec = importlib.util.spec_from_file_location("lsdem_scenes_host", ROOT / "lsdem2.0_b200" / "scenes.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def scale_sample(ora, scenes, T):
    """The bounded host sample of the large-scale workload: SAMPLE_PARTICLES bodies of its 16
    superquadrics (grids T), periodic in x and y, floor and ceiling, the same solid fraction
    (scenes.settling_sample), as an oracle model."""
    def mass_fn(sdf, size, origin, h):
        o = ora.mass_props(sdf, size, origin, h, 1.0)
        return o[0], o[1:4].copy(), o[10:16].copy()
    smp = scenes.settling_sample(mass_fn, T, SAMPLE_PARTICLES, seed=scenes.seed_for(4) + 7919)
    return ora.model_from_scene(smp), smp


def time_oracle(ora, model, dt, steps, min_seconds, max_steps):
    """Steps of the FP64 oracle on all host threads: one untimed (history), then at least
    `steps`, and more until `min_seconds` (at most `max_steps`). Returns (steps, seconds, threads)."""
    threads = os.cpu_count() or 1
    ora.set_threads(threads)
    sim = ora.OracleSim(model, nthreads=threads)
    sim.step(dt)
    t0 = time.perf_counter()
    done = 0
    while done < steps or (time.perf_counter() - t0 < min_seconds and done < max_steps):
        sim.step(dt)
        done += 1
    return done, time.perf_counter() - t0, threads


def cpu_baseline(lsdem, sc, workload, target_particles=3000, steps=2, min_seconds=10.0, max_steps=200):
    """FP64 oracle step (the reference algorithm restated on the CPU, all host threads) on a
    bounded sample. Large-scale workload: a smaller box of the same configuration
    (scale_sample, the same templates). Others: the particles inside a corner sub-box of the
    same scene (for the bonded and drum workloads the cluster of particles nearest the median
    position). At least `steps` steps are timed, and more until `min_seconds` of CPU work (at
    most `max_steps`)."""
    ora = _oracle()
    if workload == "scale" and "raw_templates" in sc:
        from lsdem_b200 import scenes
        model, smp = scale_sample(ora, scenes, sc["raw_templates"])
        done, t, threads = time_oracle(ora, model, sc["dt"], steps, min_seconds, max_steps)
        m = len(smp["pos"])
        return {"value": m * done / t, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                "build": ORACLE_BUILD["flags"], "sample": (f"{m} particles of the same 16 superquadrics in a box periodic in x and y with floor and "
                           f"ceiling at the same solid fraction ({smp['max'][0]:.4f} m side), random sequential "
                           f"addition, {done} steps of the FP64 oracle (reference per-node 27-cell algorithm)")}

    n = len(sc["pos"])
    pos = np.asarray(sc["pos"])
    lo, hi = np.asarray(sc["min"]), np.asarray(sc["max"])
    frac = min(1.0, (target_particles / n) ** (1.0 / 3.0))
    sub_hi = lo + (hi - lo) * frac
    idx = np.nonzero(np.all((pos >= lo) & (pos < sub_hi), axis=1))[0]
    if workload in ("bonded", "drum", "scale"):
        # a compact cluster of the particles nearest to the one closest to the median position
        from scipy.spatial import cKDTree
        tree = cKDTree(pos)
        c = pos[tree.query(np.median(pos, axis=0))[1]]
        idx = np.sort(tree.query(c, k=min(n, target_particles))[1])
        r = float(np.max([t["bound"] for t in sc["templates"]]) * np.max(sc["scale"]))
        lo, sub_hi = pos[idx].min(0) - 2 * r, pos[idx].max(0) + 2 * r
        frac = len(idx) / n
    sv = lsdem.Solver()
    from lsdem_b200 import scenes
    if workload == "small":
        sub = dict(sc)
        sub["pos"], sub["quat"] = pos[idx], np.asarray(sc["quat"])[idx]
        sub["vel"] = np.asarray(sc.get("vel", np.zeros((n, 3))))[idx]
        scenes.load_into(sv, sub)
        dmin, dmax = sc["min"], sc["max"]
    else:
        sub = dict(sc)
        for k in ("shape", "scale", "pos", "quat", "vel", "inv_mass", "inv_inertia"):
            sub[k] = np.asarray(sc[k])[idx]
        ids = [sv.add_shape(t["nodes"], t["sdf"], t["size"], t["origin"], t["spacing"]) for t in sub["templates"]]
        sv.add_particles(np.asarray(ids, np.int32)[sub["shape"]], sub["pos"], sub["quat"], sub["inv_mass"],
                         sub["inv_inertia"], sub["kn"], sub["ks"], sub["mu"], sub["e"], vel=sub["vel"],
                         scale=sub["scale"])
        b = sc.get("bonds")
        if b is not None:
            # the bonds among the sampled particles
            where = np.full(n, -1)
            where[idx] = np.arange(len(idx))
            for k in np.nonzero((where[b["master"]] >= 0) & (where[b["slave"]] >= 0))[0]:
                sv.add_bond(int(where[b["master"][k]]), int(where[b["slave"][k]]), b["point"][k], b["normal"][k],
                            b["radius"][k], b["length"][k], b["youngs"], b["poisson"], b["tensile"][k],
                            b["cohesion"][k], b["mu"])
        dmin, dmax = lo, sub_hi
    model = ora.model_from_solver(sv)
    model.update(domain=(dmin, dmax), gravity=sc["gravity"], periodic=0)
    steps, t, threads = time_oracle(ora, model, sc["dt"], steps, min_seconds, max_steps)
    m = len(idx)
    return {"value": m * steps / t, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "build": ORACLE_BUILD["flags"], "sample": (f"{m} particles of the same scene in a {frac:.3f}-scaled corner sub-box, {steps} steps "
                       f"of the FP64 oracle (reference per-node 27-cell algorithm)") if workload in ("small", "polydisperse")
            else (f"{m} particles of the same scene (the cluster nearest its median position, with the bonds among "
                  f"them), {steps} steps of the FP64 oracle (reference per-node 27-cell algorithm)")}


def fundem_config0(binary, scenes, workdir):
    """Config 0 (2,000 ellipsoids on a floor, 32^3 grids, 1,000 nodes) through an LSSolver app
    built from tests/apps/c0_bench.cpp: device time of steps 200-1900 from CUDA events
    recorded in the app's external-force hook. Returns ms per step, or None."""
    if not Path(binary).exists():
        return None
    workdir.mkdir(parents=True, exist_ok=True)
    sc = scenes.ellipsoid_falling()
    nsteps, k0, k1 = 2000, 200, 1900
    scene, res = workdir / "c0.bin", workdir / "c0.res"
    scenes.write_c0_app_scene(scene, sc, nsteps, k0, k1)
    r = subprocess.run([str(binary), str(scene), str(workdir / "out"), str(res)], capture_output=True, text=True,
                       timeout=900)
    if r.returncode != 0:
        return None
    steps, window, ms, _ = scenes.read_c0_app_result(res)
    return {"ms_per_step": ms / window, "window_steps": window, "particles": len(sc["pos"])}


def run_reference(args, rank, world):
    """--impl reference: the reference algorithm's CPU implementation (the FP64 oracle port;
    the reference has no CPU path of its own) on the host cores, same metric and workload.
    For the large-scale workload everything is prepared on the host (the CUDA library is not
    loaded): the same 16 templates from the oracle's host grid generator, a smaller box of
    the same configuration, the oracle's own mass properties. Beside it, the reference's own
    CUDA build runs the config-0 app on this box's GPU (when it was built)."""
    if rank != 0:
        return
    ora = _oracle()
    scenes = _scenes_host()
    if args.workload == "scale":
        rng = np.random.default_rng(scenes.seed_for(4))
        t0 = time.perf_counter()
        T = scenes.superquadric_templates_host(lambda v, f, o, size, h: ora.mesh_grid(v, f, o, size, h), rng, 16,
                                               (2.0, 6.0), (1e-3, 2.5e-3), 48, 1500)
        t_prep = time.perf_counter() - t0
        model, smp = scale_sample(ora, scenes, T)
        steps, t, threads = time_oracle(ora, model, 5e-7, max(1, args.steps), 0.0, max(1, args.steps))
        m = len(smp["pos"])
        cfg = {"workload": "settling-2000000-superquadrics-16", "particles": 2_000_000, "templates": 16,
               "nodes_per_particle": 1500, "sdf_grid": "48 nodes on the longest axis", "periodic": "xy",
               "walls": "z", "solid_fraction": 0.25, "dt_s": 5e-7}
        cb = {"value": m * steps / t, "unit": "particle-steps/s", "cores": threads, "kind": "port",
              "build": ORACLE_BUILD["flags"], "sample": (f"{m} particles of the same 16 superquadrics (grids from the oracle's host generator, "
                         f"{t_prep:.0f} s) in a box periodic in x and y with floor and ceiling at the same solid "
                         f"fraction ({smp['max'][0]:.4f} m side), {steps} steps of the FP64 oracle "
                         f"(reference per-node 27-cell algorithm)")}
    else:
        lsdem = _package()
        import torch  # noqa: F401  (device 0 hosts the scene preparation)
        sc, cfg = build_scene(lsdem, args.workload, 0, args.particles)
        cb = cpu_baseline(lsdem, sc, args.workload, steps=max(1, min(args.steps, 3)))
    line = {"metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference", "config": cfg, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if not args.no_fundem:
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            fd = fundem_config0(ROOT / "oracle" / "_ref" / "c0_bench_fundem", scenes, Path(d))
        if fd is not None:
            line["fundem_gpu_config0"] = dict(fd, build="the reference's own CUDA kernels and LSSolver.h (sm_100a), "
                                                        "app tests/apps/c0_bench.cpp")
    print(json.dumps(line), flush=True)


L2_FLUSH_BYTES = 256 << 20  # > the 126 MB L2


def tensor_roofline(head, scr):
    """The learned form's network pass (k_net_screen, tcgen05): network evaluations per step
    x NET_FLOP over the pass's per-step time (its own profile phase), against the dense BF16
    peak."""
    ms, calls = head["profile"].get("network", (0.0, 0))
    rows = (scr or {}).get("net_evals", 0.0)
    if not calls or not rows:
        return None
    t = ms / head["profile_steps"] * 1e-3
    achieved = rows * NET_FLOP / t / 1e12
    peak, kind = _bf16_peak()
    return {"bound": "tensor", "kernel": "k_net_screen", "achieved": achieved, "peak": peak, "peak_kind": kind,
            "unit": "TFLOP/s", "frac": achieved / peak, "rows_per_step": rows, "flop_per_row": NET_FLOP,
            "ms_per_step": t * 1e3}


def build_c0_app():
    """Builds tests/apps/c0_bench.cpp against the drop-in LSSolver header and this library
    (nvcc, sm_100a) under the package's build folder; returns the executable or None."""
    import shutil
    app = ROOT / "tests" / "apps" / "c0_bench.cpp"
    out = ROOT / "lsdem2.0_b200" / "_build" / "c0_bench_b200"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if out.exists() and out.stat().st_mtime >= app.stat().st_mtime:
        return out
    if not Path(nvcc).exists():
        return None
    out.parent.mkdir(exist_ok=True)
    r = subprocess.run([nvcc, "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", str(ROOT / "include"), "-I", str(ROOT / "include" / "kernel"), str(app),
                        "-L", str(ROOT / "lsdem2.0_b200"), "-llsdem_b200", "-Xlinker", "-rpath", "-Xlinker",
                        str(ROOT / "lsdem2.0_b200"), "-o", str(out)], capture_output=True, text=True)
    return out if r.returncode == 0 else None


def max_over_ranks(dist, value, device):
    """Largest value over the ranks of the process group (identity without one)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_form(lsdem, torch, sc, args, local, prec, dist, barrier, clocks, learned=False):
    """W warm-up steps, then exactly K timed steps, each bracketed by CUDA events on the
    solver's stream with a 256 MB scratch write before it (outside the events) so that no
    step starts from data the previous one left in L2; the state backup of each batch of
    steps is timed with the batch's first step. Max over ranks. A second run of K steps
    timed as a whole, L2 not flushed, is reported beside it (`warm_l2`)."""
    info = {}
    sv = load(lsdem, sc, args.workload, local, prec, learned=learned, info=info)
    dt = float(sc["dt"])
    if clocks is not None:
        clocks.__enter__()  # the sampler starts up during the warm-up
    sv.step(dt, max(3, args.warmup))
    launches0 = sv.num(8)
    reruns0 = sv.num(7)
    builds0 = sv.num(9)
    sv.set_step_timing(True, L2_FLUSH_BYTES)
    barrier()
    if clocks is not None:
        clocks.mark(True)
    sv.step(dt, args.steps)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark(False)
        clocks.__exit__()
    step_ms, step_calls = sv.profile()["step"]
    assert step_calls == args.steps, (step_calls, args.steps)
    sv.set_step_timing(False)
    res = {"ms": step_ms, "launches": sv.num(8) - launches0, "reruns": sv.num(7) - reruns0,
           "builds": sv.num(9) - builds0, "stats": sv.step_stats(), **info}
    # the same number of steps timed as one region, L2 not flushed
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    sv.step(dt, args.steps)
    ev1.record()
    torch.cuda.synchronize()
    res["warm_ms"] = ev0.elapsed_time(ev1)
    # per-phase device times (CUDA events between phases) from a separate, shorter run
    res["profile_steps"] = min(args.steps, 20)
    sv.set_profiling(True)
    if prec != 0:
        sv.set_screen_stats(True)
    sv.step(dt, res["profile_steps"])
    res["profile"] = sv.profile()
    sv.set_profiling(False)
    if prec != 0:
        res["screen"] = {k: v / res["profile_steps"] for k, v in sv.screen_stats().items()}
        sv.set_screen_stats(False)
    for key in ("ms", "warm_ms"):
        res[key] = max_over_ranks(dist, res[key], "cuda")
    return sv, res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="scale", choices=["polydisperse", "small", "bonded", "drum", "scale"])
    ap.add_argument("--form", default="fp32-bf16-learned", choices=list(FORMS))
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fundem", action="store_true", help="skip the config-0 app leg")
    ap.add_argument("--all-forms", action="store_true", help="also time the FP16-template form")
    ap.add_argument("--headline-only", action="store_true", help="skip the other forms and the error check")
    ap.add_argument("--settle-steps", type=int, default=0,
                    help="untimed steps before the measurement (a settled, contact-dense state shared by all forms)")
    ap.add_argument("--settle-gravity", type=float, default=1.0,
                    help="gravity multiplier during the settling steps (then 2000 steps under the scene's gravity)")
    ap.add_argument("--particles", type=int, default=100_000, help="polydisperse workload size (profiling cases)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        run_reference(args, rank, world)
        if world > 1:
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    lsdem = _package()
    sc, cfg = build_scene(lsdem, args.workload, rank, args.particles, local)
    if args.settle_steps > 0:
        t0 = time.perf_counter()
        cpp = settle(lsdem, sc, args.workload, local, args.settle_steps, args.settle_gravity)
        how = (f"{args.settle_steps} untimed steps under {args.settle_gravity:g} x gravity and 2000 under gravity"
               if args.settle_gravity != 1.0 else f"{args.settle_steps} untimed steps")
        cfg["initial_state"] = (f"{cfg.get('initial_state', 'seeded placement')}, then {how} "
                                f"({time.perf_counter() - t0:.0f} s): {cpp:.3f} node contacts per particle")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    prec = FORMS[args.form]
    clk = Clocks(local)
    sv, head = time_form(lsdem, torch, sc, args, local, prec, dist, barrier, clk, learned="learned" in args.form)
    n = sv.n_particles
    value = n * world * args.steps / (head["ms"] * 1e-3)

    # end-to-end through the C ABI: per step, pinned host state -> device, one step,
    # state + forces back to pinned host memory
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    h = {k: pin((n, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
    h["quat"] = pin((n, 4))
    st = sv.state()
    for k in h:
        h[k][:] = st[k]
    dp = lambda a: a.ctypes.data_as(lsdem.DP)
    dt = float(sc["dt"])
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        assert lsdem.lib.lsdem_set_state(sv.h, dp(h["pos"]), dp(h["vel"]), dp(h["angvel"]), dp(h["quat"])) == 0
        sv.step(dt, 1)
        assert lsdem.lib.lsdem_get_state(sv.h, dp(h["pos"]), dp(h["vel"]), dp(h["angvel"]), dp(h["quat"]),
                                         dp(h["force"]), dp(h["torque"])) == 0
    barrier()
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0, "cuda")
    e2e = n * world * args.e2e_steps / e2e_s
    sv.close()

    forms = {}
    if not args.headline_only:
        for name, p in FORMS.items():
            if name == args.form or (name == "fp32-fp16" and not args.all_forms):
                continue
            svf, r = time_form(lsdem, torch, sc, args, local, p, dist, barrier, None, learned="learned" in name)
            svf.close()
            forms[name] = {"value": n * world * args.steps / (r["ms"] * 1e-3), "ms_per_step": r["ms"] / args.steps,
                           "warm_l2": {"value": n * world * args.steps / (r["warm_ms"] * 1e-3),
                                       "ms_per_step": r["warm_ms"] / args.steps}}
            if "training" in r:
                forms[name]["training"] = r["training"]
                forms[name]["screen_per_step"] = r.get("screen")
        for name, p in FORMS.items():
            if p != 0 and (name != "fp32-fp16" or args.all_forms):
                err = force_error(lsdem, sc, args.workload, local, p, learned="learned" in name)
                forms.setdefault(name, {})["error_vs_fp64"] = err

    # the config-0 app through the drop-in LSSolver header (same source as the reference
    # arm's build of the reference), built here against this library
    dropin0 = None
    if rank == 0 and not args.no_fundem:
        import tempfile
        from lsdem_b200 import scenes
        exe = build_c0_app()
        if exe is not None:
            with tempfile.TemporaryDirectory() as d:
                dropin0 = fundem_config0(exe, scenes, Path(d))

    if rank == 0:
        peak, peak_kind = _peaks()
        prof, stats = head["profile"], head["stats"]
        np_ms, np_calls = prof["narrowphase"]
        g_ms, g_calls = prof["ghost_narrowphase"]
        pairs = stats["pairs_particle"] + stats["pairs_wall"] + stats["pairs_ghost"]
        avg_ms = (np_ms + g_ms) / max(1, np_calls + g_calls)
        # a step runs the particle/wall launch and the image launch: per-launch bytes = per-step / 2
        launches_per_step = 2 if g_calls else 1
        if prec == 0:
            kernel = "k_narrowphase"
            bytes_launch = (B_PARTICLE * n * launches_per_step + B_PAIR * pairs + B_CONTACT * stats["contacts"]) / \
                launches_per_step
        else:
            kernel = "k_screen_f"
            bytes_launch = (B_PARTICLE_SCREEN * n * launches_per_step + B_PAIR_SCREEN * pairs) / launches_per_step
        # DRAM bytes per launch: the capture's measured traffic scaled by algorithmic bytes
        # (its excess over them is the 16-bit template store read once per step after the
        # L2 flush, so the scaling overstates it for larger cases: an upper estimate)
        traffic = (SCREEN_CAPTURE["dram_bytes_per_launch"] / SCREEN_CAPTURE["algorithmic_bytes_per_launch"] *
                   bytes_launch) if prec != 0 else None
        achieved = bytes_launch / (avg_ms * 1e-3) / 1e9
        b_step = B_STEP_PARTICLE * n + B_CONTACT * stats["contacts"] + 16 * pairs
        ms_step = head["ms"] / args.steps
        forms[args.form] = dict(forms.get(args.form, {}), value=value, ms_per_step=ms_step,
                                warm_l2={"value": n * world * args.steps / (head["warm_ms"] * 1e-3),
                                         "ms_per_step": head["warm_ms"] / args.steps})
        if "training" in head:
            forms[args.form]["training"] = head["training"]
        per_s = world * args.steps / (head["ms"] * 1e-3)  # steps per second, all ranks
        scr = head.get("screen") or {}
        plain = forms.get("fp64", {}).get("value")
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPE[args.form],
            "data": "synthetic (seeded)",
            "config": dict(cfg, form=args.form, parallelism=f"replicas x{world}",
                           l2=f"flushed: {L2_FLUSH_BYTES >> 20} MB written before every timed step, outside "
                              f"its events (per-step algorithmic traffic {b_step / 1e6:.0f} MB)",
                           contacts_per_step=stats["contacts"], candidate_pairs_per_step=pairs,
                           pairs_per_step={"particle": stats["pairs_particle"], "wall": stats["pairs_wall"],
                                           "image": stats["pairs_ghost"]},
                           contacts_per_particle=stats["contacts"] / n),
            "forms": forms,
            "headline_over_plain_grid": (value / plain) if plain else None,
            "contacts_per_s": stats["contacts"] * per_s,
            "node_tests_per_s": scr.get("node_tests", 0.0) * per_s if scr else None,
            # The screen is bound by load latency and instruction issue, not by DRAM: its
            # algorithmic bytes over its launch time are a few percent of HBM bandwidth
            # (reported as such), the issue and warp figures come from ncu.
            "roofline": {"bound": "latency/issue", "kernel": kernel, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": avg_ms,
                         "traffic_kind": "scaled from a 200,000-particle ncu capture" if prec != 0 else None,
                         "hbm_is_limiter": False,
                         "limiter": ({"bound": "L2 load latency / issue", "issue_active": SCREEN_CAPTURE["issue_active"],
                                      "warps_active": SCREEN_CAPTURE["warps_active"],
                                      "warps_active_limit": SCREEN_CAPTURE["warps_active_limit"],
                                      "leading_stall": SCREEN_CAPTURE["leading_stall"],
                                      "case": SCREEN_CAPTURE["case"]} if prec != 0 else None),
                         "node_tests_per_s_in_screen": (scr.get("node_tests", 0.0) * head["profile_steps"] /
                                                        ((np_ms + g_ms) * 1e-3)) if scr else None},
            "step_roofline": {"bytes_per_step": b_step, "achieved_gbs": b_step / (ms_step * 1e-3) / 1e9},
            "tensor_roofline": tensor_roofline(head, scr),
            "phases_ms_per_step": {k: v[0] / head["profile_steps"] for k, v in prof.items()},
            "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": n * (3 * 24 + 32),
                    "d2h_bytes_per_step": n * (5 * 24 + 32)},
            "screen_per_step": head.get("screen"),
            "gpu_launches": head["launches"],
            "overflow_reruns": head["reruns"],
            # timed steps that sorted the cells and rebuilt the neighbour lists
            "neighbour_list_rebuilds": head["builds"],
            "clocks": clk.summary(),
        }
        if dropin0 is not None:
            line["dropin_gpu_config0"] = dict(dropin0, build="tests/apps/c0_bench.cpp against include/kernel/LSSolver.h "
                                                              "and this library (FP64 form)")
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(lsdem, sc, args.workload)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

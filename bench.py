"""Benchmark of the level-set DEM time step (particle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload polydisperse|small]

Workload (default "polydisperse", the precision-form configuration that fits one
GPU): 100,000 particles from 4 templates (ellipsoid 1:0.8:0.6, superquadric
exponent 4, rounded cube, capsule of aspect 2) with log-normal bounding
diameters (median 2 mm, sigma 0.25), 48^3 SDF grids, 2,000 surface nodes each,
0.1 m triply periodic cube, velocities N(0, 0.1 m/s), linear contact (kn 1e5,
kt 0.8 kn, mu 0.5, e 0.6), dt 5e-7 s. Synthetic, seeded (no dataset).

One step = one full time step (half kick, drift, cell sort, candidates,
narrowphase + contact forces, periodic images, half kick) of the whole scene.
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


# Algorithmic bytes of the fused narrowphase + contact-force kernel (k_narrowphase):
# per owner particle, per candidate pair and per contact ("roofline").
B_PARTICLE = 208
B_PAIR = 236
B_CONTACT = 56
# whole-step algorithmic bytes per particle for the other phases (state read+write,
# keys, sort, candidates): see DESIGN.md
B_STEP_PARTICLE = 448


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
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 3 + k and r[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def build_scene(lsdem, workload: str, rank: int, particles: int = 100_000):
    from lsdem_b200 import scenes
    if workload == "small":
        sc = scenes.ellipsoid_falling(seed=scenes.seed_for(0) + rank)
        return sc, {"workload": "ellipsoids-2000-floor", "particles": 2000, "nodes_per_particle": 1000,
                    "sdf_grid": "32^3 fp64", "box_m": [0.2, 0.2, 0.4], "dt_s": 1e-6}
    cache = ROOT / "_build" / "templates_48_2000.npz"
    T = None
    if cache.exists():
        z = np.load(cache, allow_pickle=True)
        T = list(z["T"])
    else:
        T = scenes.unit_templates(48, 2000)
        cache.parent.mkdir(exist_ok=True)
        np.savez(cache, T=np.array(T, dtype=object))
    box = 0.1 * (particles / 1e5) ** (1.0 / 3.0)
    sc = scenes.polydisperse_periodic(lsdem, n=particles, box=box, seed=scenes.seed_for(1) + rank, templates=T)
    # deep initial overlaps (many surface nodes inside a neighbour) would exceed the stability
    # limit of the explicit step; re-place those particles, keep shallow contacts
    iters = scenes.resolve_deep_overlaps(lsdem, sc, device=int(os.environ.get("LOCAL_RANK", "0")))
    sc["resolve_iterations"] = iters
    name = "polydisperse-100k-4templates-periodic" if particles == 100_000 else f"polydisperse-{particles}-4templates-periodic"
    return sc, {"workload": name, "particles": particles, "nodes_per_particle": 2000,
                "sdf_grid": "48^3 fp64", "templates": 4, "size": "lognormal(median 2 mm, sigma 0.25)",
                "box_m": round(box, 6), "periodic": "xyz", "dt_s": 5e-7}


def load(lsdem, sc, workload, device):
    from lsdem_b200 import scenes
    sv = lsdem.Solver(device=device)
    if workload == "small":
        scenes.load_into(sv, sc)
    else:
        scenes.load_polydisperse(sv, sc)
    sv.initialize(sc["min"], sc["max"], sc["gravity"])
    return sv


def cpu_baseline(lsdem, sc, workload, target_particles=3000, steps=2):
    """FP64 oracle step (the reference algorithm restated on the CPU, all host threads) on a
    bounded sample: the particles inside a sub-box of the same scene holding ~target_particles."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as ora  # the checker, timed here as the CPU baseline

    n = len(sc["pos"])
    pos = np.asarray(sc["pos"])
    lo, hi = np.asarray(sc["min"]), np.asarray(sc["max"])
    frac = min(1.0, (target_particles / n) ** (1.0 / 3.0))
    sub_hi = lo + (hi - lo) * frac
    sel = np.all((pos >= lo) & (pos < sub_hi), axis=1)
    idx = np.nonzero(sel)[0]
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
        dmin, dmax = lo, sub_hi
    model = ora.model_from_solver(sv)
    model.update(domain=(dmin, dmax), gravity=sc["gravity"], periodic=0)
    threads = os.cpu_count() or 1
    ora.set_threads(threads)
    sim = ora.OracleSim(model, nthreads=threads)
    sim.step(sc["dt"])  # untimed first step (history)
    t0 = time.perf_counter()
    for _ in range(steps):
        sim.step(sc["dt"])
    t = time.perf_counter() - t0
    m = len(idx)
    return {"value": m * steps / t, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": f"{m} particles of the same scene in a {frac:.3f}-scaled corner sub-box, {steps} steps "
                      f"of the FP64 oracle (reference per-node 27-cell algorithm)"}


def run_reference(args, rank, world):
    """--impl reference: the reference algorithm's CPU implementation (the FP64 oracle port;
    the reference has no CPU path of its own) on the host cores, same metric and workload."""
    if rank != 0:
        return
    lsdem = _package()
    sc, cfg = build_scene(lsdem, args.workload, 0, args.particles)
    cb = cpu_baseline(lsdem, sc, args.workload, steps=max(1, min(args.steps, 3)))
    line = {"metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference", "config": cfg, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="polydisperse", choices=["polydisperse", "small"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--particles", type=int, default=100_000, help="polydisperse workload size (profiling cases)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=600))
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
    sc, cfg = build_scene(lsdem, args.workload, rank, args.particles)
    sv = load(lsdem, sc, args.workload, local)
    n = sv.n_particles
    dt = float(sc["dt"])
    sv.step(dt, max(3, args.warmup))
    sv.set_profiling(True)
    launches0 = sv.num(8)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record()
        sv.step(dt, args.steps)
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = sv.num(8) - launches0
    prof = sv.profile()
    stats = sv.step_stats()
    sv.set_profiling(False)
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = n * world * args.steps / (ms_max * 1e-3)

    # end-to-end through the C ABI: per step, pinned host state -> device, one step,
    # state + forces back to pinned host memory
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    h = {k: pin((n, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
    h["quat"] = pin((n, 4))
    st = sv.state()
    for k in h:
        h[k][:] = st[k]
    import ctypes as C
    dp = lambda a: a.ctypes.data_as(lsdem.DP)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        rc = lsdem.lib.lsdem_set_state(sv.h, dp(h["pos"]), dp(h["vel"]), dp(h["angvel"]), dp(h["quat"]))
        assert rc == 0
        sv.step(dt, 1)
        rc = lsdem.lib.lsdem_get_state(sv.h, dp(h["pos"]), dp(h["vel"]), dp(h["angvel"]), dp(h["quat"]),
                                       dp(h["force"]), dp(h["torque"]))
        assert rc == 0
    barrier()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = n * world * args.e2e_steps / e2e_s

    if rank == 0:
        peak, peak_kind = _peaks()
        np_ms, np_calls = prof["narrowphase"]
        g_ms, g_calls = prof["ghost_narrowphase"]
        pairs = stats["pairs_particle"] + stats["pairs_wall"] + stats["pairs_ghost"]
        launches_np = np_calls + g_calls
        avg_ms = (np_ms + g_ms) / max(1, launches_np)
        # one step runs the particle/wall launch and the ghost launch: per-launch bytes = per-step / 2
        bytes_step_np = B_PARTICLE * n * 2 + B_PAIR * pairs + B_CONTACT * stats["contacts"]
        bytes_launch = bytes_step_np / 2.0
        achieved = bytes_launch / (avg_ms * 1e-3) / 1e9
        b_step = B_STEP_PARTICLE * n + B_CONTACT * stats["contacts"] + 16 * pairs
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": dict(cfg, form="plain grid (FP64)", parallelism=f"replicas x{world}",
                           l2=f"not flushed: per-step algorithmic traffic {b_step / 1e6:.0f} MB vs 126 MB L2",
                           contacts_per_step=stats["contacts"], candidate_pairs_per_step=pairs),
            "roofline": {"bound": "hbm", "kernel": "k_narrowphase", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": avg_ms},
            "step_roofline": {"bytes_per_step": b_step, "achieved_gbs": b_step / (ms_max / args.steps * 1e-3) / 1e9},
            "phases_ms_per_step": {k: v[0] / max(1, args.steps) for k, v in prof.items()},
            "e2e": {"value": e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": n * (3 * 24 + 32),
                    "d2h_bytes_per_step": n * (5 * 24 + 32)},
            "gpu_launches": launches,
            "overflow_reruns": sv.num(7),
            "clocks": clk.summary(),
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(lsdem, sc, args.workload)
        print(json.dumps(line), flush=True)
    sv.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

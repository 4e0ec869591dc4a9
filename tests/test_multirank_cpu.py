"""The multi-process paths of bench.py on CPU with the gloo backend (world size 2).

bench.py runs one process per GPU (torchrun), times on the device and reports the largest
time over the ranks; on a CPU host the same launch runs the reference arm (the FP64 oracle)
with gloo, where rank 0 alone measures and prints and the other ranks exit 0 without work.
"""
import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench = _bench()
        v = bench.max_over_ranks(dist, 1.5 + rank, "cpu")
        with open(f"{out}.{rank}", "w") as f:
            f.write(repr(v))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    out = str(tmp_path / "r")
    ctx = mp.get_context("spawn")
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert [float(open(f"{out}.{r}").read()) for r in range(2)] == [2.5, 2.5]


@pytest.mark.timeout(600)
def test_reference_arm_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--workload", "small", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"

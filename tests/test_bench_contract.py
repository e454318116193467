"""bench.py's contract on the CPU: the reference arm (the oracle on the host
cores, no GPU) prints one JSON line with the fields the metric needs, on one
process and under torch.distributed.run with two ranks (gloo; rank 0 alone
prints), and the max-over-ranks reduction of the timed figures."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def json_lines(out):
    return [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]


def check_reference_line(d, n_gpus, steps, warmup):
    assert d["impl"] == "reference"
    assert d["unit"] == "ms" and d["higher_is_better"] is False and d["value"] > 0
    assert d["ms_per_step"] == d["value"]
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (n_gpus, steps, warmup)
    assert d["termination"] == "Converged" and d["iterations"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


def test_reference_arm_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--grid", "16", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    check_reference_line(lines[0], 1, 2, 1)


def test_reference_arm_plain_workload():
    """--workload c1: the oracle's Jacobi-PCG on the 2-D 128^2 system."""
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "c1", "--steps", "2",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    d = lines[0]
    check_reference_line(d, 1, 2, 1)
    assert "Jacobi-PCG" in d["metric"] and d["config"]["unknowns"] == 128 * 128
    assert d["iterations"] == 383  # the device solve's count as well (perf configs)


def test_reference_arm_batched_networks():
    """--workload c4: the oracle on every 16th of the 4096 networks, the 1-D
    solve of each (LinearSystemSolver cascade) on worker threads, scaled to the
    whole batch; Jacobi-PCG per network beside it."""
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "c4", "--steps", "1",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0 and d["config"]["systems"] == 4096
    paths = d["paths_in_sample"]
    assert sum(paths.values()) == 256 and "failed" not in paths and "error" not in paths
    assert d["jacobi_pcg_ms"] > 0
    assert d["cpu_baseline"]["value"] == d["value"] and "every 16th" in d["cpu_baseline"]["sample"]


def test_reference_arm_adjoint():
    """--workload c5: the oracle's FP64 adjoint gradient of the 512^2 Darcy loss."""
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "c5", "--steps", "1",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0 and d["loss"] > 0
    assert d["config"]["unknowns"] == 512 * 512 and d["cpu_baseline"]["value"] == d["value"]


def test_reference_arm_two_ranks():
    """Launched with torchrun for N > 1: one rank per process over gloo; rank 0
    alone measures and prints, the other rank exits 0 without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           "bench.py", "--impl", "reference", "--gpus", "2", "--grid", "16", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = json_lines(out.stdout)
    assert len(lines) == 1
    check_reference_line(lines[0], 2, 1, 1)


def _max_worker(rank, port, result):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    sys.path.insert(0, ROOT)
    import bench
    result[rank] = bench.max_over_ranks(1.5 + rank, 2)
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = free_port()
    with ctx.Manager() as m:
        result = m.dict()
        procs = [ctx.Process(target=_max_worker, args=(r, port, result)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(result) == {0: 2.5, 1: 2.5}

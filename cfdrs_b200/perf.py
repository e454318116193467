"""Profiling cases for the solve path (run under ncu or alone).

    python -m cfdrs_b200.perf spmv  --n 128 --reps 5     # FP32 and FP64 SpMV of the n^3 operator
    python -m cfdrs_b200.perf solve --n 256               # one FP32+refinement and one FP64 AMG-PCG solve
    python -m cfdrs_b200.perf levels --n 256              # SpMV bandwidth of every hierarchy operator
    python -m cfdrs_b200.perf batch --systems 4096        # batched network solve, FP64 and FP32+refinement

All cases use the seeded 3-D variable-coefficient Poisson system of bench.py.
"""
from __future__ import annotations

import argparse
import sys


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_spmv(torch, d, n_rows, n_cols, nnz, fp32, reps):
    dt = torch.float32 if fp32 else torch.float64
    vs = 4 if fp32 else 8
    x = torch.rand(n_cols, device="cuda", dtype=dt)
    y = torch.empty(n_rows, device="cuda", dtype=dt)
    for _ in range(3):
        d.spmv(x.data_ptr(), y.data_ptr(), fp32=fp32)
    s = torch.cuda.current_stream()
    e0, e1 = _events(torch)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        d.spmv(x.data_ptr(), y.data_ptr(), fp32=fp32)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nbytes = nnz * (vs + 4) + 4 * (n_rows + 1) + vs * (n_rows + n_cols)
    return ms, nbytes, x, y


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["spmv", "solve", "levels", "batch"])
    p.add_argument("--systems", type=int, default=4096)
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--reps", type=int, default=20)
    a = p.parse_args(argv)
    import torch

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.device import DeviceCsr, context

    if a.case == "batch":
        return batch_case(a)
    A, b, _ = P.poisson_3d_variable(a.n, 8.0, 1.0, seed=0)
    ctx = context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    if a.case == "spmv":
        d = DeviceCsr(A, ctx)
        for fp32 in (True, False):
            ms, nb, x, y = time_spmv(torch, d, A.nrows, A.ncols, A.nnz, fp32, a.reps)
            print(f"{a.n}^3 {'f32' if fp32 else 'f64'}: {ms * 1e3:.1f} us {nb / ms / 1e6:.0f} GB/s", flush=True)
        return 0
    amg = cf.AlgebraicMultigrid(A, cf.AMGConfig.pressure_poisson(), ctx=ctx)
    if a.case == "levels":
        st = amg.statistics()
        for l in range(st.num_levels):
            for which, name in ((0, "A"), (1, "P"), (2, "R")):
                if which and l == st.num_levels - 1:
                    continue
                m = amg.level(l, which)
                d = DeviceCsr(m, ctx)
                for fp32 in (True, False):
                    ms, nb, _, _ = time_spmv(torch, d, m.nrows, m.ncols, m.nnz, fp32, a.reps)
                    print(f"L{l} {name} {m.nrows}x{m.ncols} nnz={m.nnz} ({m.nnz / max(m.nrows, 1):.1f}/row) "
                          f"{'f32' if fp32 else 'f64'}: {ms * 1e3:8.1f} us {nb / ms / 1e6:6.0f} GB/s", flush=True)
        return 0
    bd = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bd)
    cfg = cf.IterativeSolverConfig(0.0, 1e-8, 1000)
    r1 = cf.cg_preconditioned(A, bd, amg, x, cfg, precision=cf.Precision.FP32_REFINE)
    x.zero_()
    r2 = cf.cg_preconditioned(A, bd, amg, x, cfg)
    torch.cuda.synchronize()
    print(r1)
    print(r2)
    print(amg.statistics())
    return 0


def batch_case(a):
    """4096 seeded networks (n uniform in [20, 2000], 10 % loop edges), Jacobi-PCG
    to a 1e-10 equilibrated residual, FP64 and FP32 + FP64 refinement."""
    import time

    import numpy as np

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.batch import NetworkBatch
    t0 = time.perf_counter()
    systems = P.network_batch(a.systems, seed=0)
    mats = [A for A, _ in systems]
    b = np.concatenate([bb for _, bb in systems])
    nb = NetworkBatch(mats)
    print(f"generated {a.systems} systems, {nb.rows} rows, {nb.val.size} nnz in {time.perf_counter() - t0:.1f} s",
          flush=True)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 40000)
    for prec in (cf.Precision.FP64, cf.Precision.FP32_REFINE):
        tc = nb.autotune(prec, sample_iterations=64)
        nb.solve(b, config=cfg, precision=prec)  # warm-up
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            x, rep = nb.solve(b, config=cfg, precision=prec)
            times.append((time.perf_counter() - t0) * 1e3)
        print(f"{prec.name}: device {rep.device_ms:.2f} ms, wall {min(times):.2f} ms, converged "
              f"{rep.converged_systems}/{rep.num_systems}, iterations total {rep.total_iterations} max "
              f"{rep.max_iterations}, max rel residual {rep.max_rel_residual:.2e}, widths {tc}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

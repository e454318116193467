"""Profiling cases for the solve path (run under ncu or alone).

    python -m cfdrs_b200.perf spmv  --n 128 --reps 5     # FP32 and FP64 SpMV of the n^3 operator
    python -m cfdrs_b200.perf solve --n 256               # one FP32+refinement and one FP64 AMG-PCG solve
    python -m cfdrs_b200.perf levels --n 256              # SpMV bandwidth of every hierarchy operator
    python -m cfdrs_b200.perf batch --systems 4096        # batched network solve, FP64 and FP32+refinement
    python -m cfdrs_b200.perf adjoint --n 512             # dL/dtheta of the 2-D Darcy column loss
    python -m cfdrs_b200.perf gmres --n 128               # AMG-GMRES(30), FP64 and FP32+refinement

All cases use the seeded 3-D variable-coefficient Poisson system of bench.py.
"""
from __future__ import annotations

import argparse
import sys


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_spmv(torch, d, n_rows, n_cols, nnz, fp32, reps, path="auto"):
    """Mean time of one SpMV on the given pipeline ("auto": the library's choice)."""
    dt = torch.float32 if fp32 else torch.float64
    vs = 4 if fp32 else 8
    d.set_path(path, fp32)
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
    if path == "diagonal":  # the layout's own bytes: every stored slot, x and y once
        nbytes = d.layout()["diagonals"] * n_rows * vs + vs * (n_rows + n_cols)
    else:  # CSR bytes (values, int32 columns and offsets, x and y once)
        nbytes = nnz * (vs + 4) + 4 * (n_rows + 1) + vs * (n_rows + n_cols)
    return ms, nbytes, x, y


def _paths(d, fp32=False):
    lay = d.layout()
    return ["split"] + (["record"] if lay["all_compressed"] else []) + (["x_staged"] if lay["x_staged"] else []) + \
        (["sliced"] if fp32 and lay["sliced"] else []) + (["diagonal"] if lay["diagonals"] else [])


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=["spmv", "solve", "levels", "batch", "assembly", "simple", "adjoint", "gmres",
                                    "timeline", "configs"])
    p.add_argument("--systems", type=int, default=4096)
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--reps", type=int, default=20)
    p.add_argument("--path", default="auto",
                   help="SpMV pipeline of every operator eligible for it in solve, gmres and timeline")
    a = p.parse_args(argv)
    import torch

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.device import DeviceCsr, context

    if a.case == "batch":
        return batch_case(a)
    if a.case == "assembly":
        return assembly_case(a)
    if a.case == "simple":
        return simple_case(a)
    if a.case == "adjoint":
        return adjoint_case(a)
    if a.case == "configs":
        return configs_case(a)
    A, b, _ = P.poisson_3d_variable(a.n, 8.0, 1.0, seed=0)
    ctx = context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    if a.case == "spmv":
        d = DeviceCsr(A, ctx)
        for fp32 in (True, False):
            for path in _paths(d, fp32):
                ms, nb, x, y = time_spmv(torch, d, A.nrows, A.ncols, A.nnz, fp32, a.reps, path)
                print(f"{a.n}^3 {'f32' if fp32 else 'f64'} {path}: {ms * 1e3:.1f} us {nb / ms / 1e6:.0f} GB/s",
                      flush=True)
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
                    for path in _paths(d, fp32):
                        ms, nb, _, _ = time_spmv(torch, d, m.nrows, m.ncols, m.nnz, fp32, a.reps, path)
                        print(f"L{l} {name} {m.nrows}x{m.ncols} nnz={m.nnz} ({m.nnz / max(m.nrows, 1):.1f}/row) "
                              f"{'f32' if fp32 else 'f64'} {path:8s}: {ms * 1e3:8.1f} us {nb / ms / 1e6:6.0f} GB/s",
                              flush=True)
        return 0
    if a.path != "auto":
        from cfdrs_b200 import _lib
        from cfdrs_b200.device import device_matrix
        for fp32 in (True, False):
            amg.set_path(a.path, fp32)
            try:
                device_matrix(A, ctx).set_path(a.path, fp32)
            except _lib.CfdError:
                pass  # the fine operator is not eligible: it keeps the default rule
    bd = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bd)
    cfg = cf.IterativeSolverConfig(0.0, 1e-8, 1000)
    if a.case == "gmres":
        for prec in (cf.Precision.FP64, cf.Precision.FP32_REFINE):
            for rep_i in range(3):
                x.zero_()
                torch.cuda.synchronize()
                r = cf.gmres_preconditioned(A, bd, amg, x, cfg, restart=30, precision=prec)
            print(f"GMRES(30) {prec.name}: {r.device_ms:.1f} ms device, {r.iterations} iterations, "
                  f"{r.outer_iterations} refinements, final {r.final_residual_norm:.3e} <= {r.threshold:.3e}", flush=True)
        return 0
    if a.case == "timeline":
        return timeline_case(torch, cf, A, bd, amg, x, cfg)
    r1 = cf.cg_preconditioned(A, bd, amg, x, cfg, precision=cf.Precision.FP32_REFINE)
    x.zero_()
    r2 = cf.cg_preconditioned(A, bd, amg, x, cfg)
    torch.cuda.synchronize()
    print(r1)
    print(r2)
    print(amg.statistics())
    return 0


def _short_kernel_name(name):
    """k_spmv_pipe<f,f,true,Jacobi0,true> style names from demangled signatures."""
    import re
    name = re.sub(r"cfd::", "", name)
    m = re.match(r"(?:void )?(?:\(anonymous namespace\)::)?(\w+)<(.*)>\(", name)
    if not m:
        m2 = re.match(r"(?:void )?(?:\(anonymous namespace\)::)?(\w+)", name)
        return m2.group(1) if m2 else name[:40]
    k, t = m.group(1), m.group(2)
    t = re.sub(r"Epi(\w+)<(float|double)(, (\d))?>", lambda mm: mm.group(1) + (mm.group(4) or ""), t)
    return f"{k}<{t.replace('float', 'f').replace('double', 'd').replace(' ', '')}>"


def timeline_case(torch, cf, A, bd, amg, x, cfg):
    """Kernel timeline (CUPTI activity records through torch.profiler) of one
    FP32 + refinement and one FP64 AMG-PCG solve after warm-up: span, busy and
    idle device time, the kernel families by total time, and the kernels of one
    mid-solve PCG iteration in launch order. Durations are those of the plain
    run (no replay, no serialisation)."""
    import collections
    import json
    import os
    import tempfile

    from torch.profiler import ProfilerActivity, profile

    def solve(prec):
        x.zero_()
        return cf.cg_preconditioned(A, bd, amg, x, cfg, precision=prec)

    precs = (("FP32+refinement", cf.Precision.FP32_REFINE), ("FP64", cf.Precision.FP64))
    for _ in range(3):
        for _, p in precs:
            solve(p)
    torch.cuda.synchronize()
    spans = []
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _, p in precs:
            torch.cuda.synchronize()
            spans.append(solve(p))
            torch.cuda.synchronize()
    fd, path = tempfile.mkstemp(suffix=".json")
    os.close(fd)
    try:
        prof.export_chrome_trace(path)
        with open(path) as f:
            events = [e for e in json.load(f)["traceEvents"] if e.get("cat") == "kernel"]
    finally:
        os.unlink(path)
    events.sort(key=lambda e: e["ts"])
    starts = [i for i, e in enumerate(events) if "at::native" in e["name"]]  # x.zero_() opens each solve
    parts = [events[starts[0] + 1:starts[1]], events[starts[1] + 1:]]
    for (name, _), rep, ev in zip(precs, spans, parts):
        t0, t1 = ev[0]["ts"], ev[-1]["ts"] + ev[-1]["dur"]
        busy = sum(e["dur"] for e in ev)
        print(f"== {name}: {rep.iterations} iterations, {rep.outer_iterations} refinements; {len(ev)} kernels, "
              f"span {(t1 - t0) / 1e3:.2f} ms, busy {busy / 1e3:.2f} ms, idle {(t1 - t0 - busy) / 1e3:.2f} ms")
        grp = collections.defaultdict(lambda: [0, 0.0])
        for e in ev:
            g = grp[_short_kernel_name(e["name"])]
            g[0] += 1
            g[1] += e["dur"]
        for k, (c, t) in sorted(grp.items(), key=lambda kv: -kv[1][1])[:16]:
            print(f"   {k:48s} {c:5d} launches {t / 1e3:8.3f} ms  avg {t / c:7.1f} us")
        upd = [i for i, e in enumerate(ev) if "k_p_update" in e["name"]]
        if len(upd) >= 2:
            lo, hi = upd[len(upd) // 2 - 1], upd[len(upd) // 2]
            print(f"   one PCG iteration ({hi - lo} kernels, {(ev[hi]['ts'] - ev[lo]['ts']) / 1e3:.3f} ms):")
            for e in ev[lo:hi]:
                grid = e.get("args", {}).get("grid", ["?"])[0]
                print(f"     {_short_kernel_name(e['name']):48s} {e['dur']:8.1f} us  grid {grid}")
    return 0


def configs_case(a):
    """The two plain-FP64 configurations beside the mixed-precision workload.
    C1: 2-D pressure Poisson on 128^2 cells (homogeneous Dirichlet walls,
    b ~ U[-1, 1]), Jacobi-PCG from zero to relative residual 1e-8. C2: 3-D
    constant-coefficient Poisson on n^3 cells (Dirichlet x = 0, 1, Neumann
    elsewhere), AMG-PCG V(1,1), damped Jacobi w = 2/3, coarsest <= 4096, FP64 to
    1e-8, with the FP32 + FP64 refinement solve beside it. Device time per
    solve (best of 5, events on the solve stream), iterations, the true
    relative residual, and the AMG setup time."""
    import time

    import numpy as np
    import torch

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.device import context

    ctx = context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)

    def best_of(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = _events(torch)
        best, rep = None, None
        for _ in range(reps):
            e0.record(stream)
            rep = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        return best, rep

    A, b = P.poisson_2d_dirichlet(128, seed=0)
    bd = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bd)
    jac = cf.JacobiPreconditioner(A)
    cfg = cf.IterativeSolverConfig(0.0, 1e-8, 20000)

    def c1():
        x.zero_()
        return cf.cg_preconditioned(A, bd, jac, x, cfg)

    ms, rep = best_of(c1)
    rel = np.linalg.norm(b - A.matvec(x.cpu().numpy())) / np.linalg.norm(b)
    print(f"C1 2-D Poisson 128^2 ({A.nrows} unknowns, {A.nnz} nnz), Jacobi-PCG FP64 to 1e-8: {ms:.3f} ms, "
          f"{rep.iterations} iterations, true relative residual {rel:.2e}", flush=True)

    A, b = P.poisson_3d_fv(a.n, None, seed=0)
    t0 = time.perf_counter()
    amg = cf.AlgebraicMultigrid(A, cf.AMGConfig.pressure_poisson(), ctx=ctx)
    setup_s = time.perf_counter() - t0
    st = amg.statistics()
    bd = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bd)
    for name, prec in (("FP64", cf.Precision.FP64), ("FP32+refinement", cf.Precision.FP32_REFINE)):
        def c2():
            x.zero_()
            return cf.cg_preconditioned(A, bd, amg, x, cfg, precision=prec)

        ms, rep = best_of(c2)
        rel = np.linalg.norm(b - A.matvec(x.double().cpu().numpy())) / np.linalg.norm(b)
        print(f"C2 3-D Poisson k = 1, {a.n}^3 ({A.nrows} unknowns, {A.nnz} nnz), AMG-PCG {name} to 1e-8: "
              f"{ms:.2f} ms, {rep.iterations} iterations, {rep.outer_iterations} refinements, "
              f"true relative residual {rel:.2e}", flush=True)
    print(f"   AMG setup {setup_s:.1f} s, {st.num_levels} levels {st.level_sizes}, "
          f"operator complexity {st.operator_complexity:.3f}", flush=True)
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


def network_counts(nets) -> dict:
    """Edges (free-free, free-fixed), fixed nodes and rows of a set of
    networks: the sizes the device assembly's compulsory bytes follow from."""
    import numpy as np
    c = dict(edges=0, ff=0, fd=0, fixed=0, rows=0)
    for n in nets:
        fi, fj = n.fixed[n.edges_i] != 0, n.fixed[n.edges_j] != 0
        c["edges"] += len(n.edges_i)
        c["ff"] += int(np.sum(~fi & ~fj))
        c["fd"] += int(np.sum(fi ^ fj))
        c["fixed"] += int(np.sum(n.fixed != 0))
        c["rows"] += n.n_nodes
    return c


def assembly_case(a):
    """Device assembly of the C4 networks (cfd_batch_assemble) from host and
    from device conductances, its bandwidth on the compulsory bytes, the host
    path of the same code for comparison, and one Picard pass (assemble from
    new device conductances, solve from the last iterate with b resident)."""
    import time

    import numpy as np
    import torch

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.batch import NetworkBatch, network_assemble_host
    t0 = time.perf_counter()
    nets = P.network_batch_edges(a.systems, seed=0)
    nb = NetworkBatch.from_networks(nets)
    pk = nb.packed
    nnz = nb.col.shape[0]
    c = network_counts(nets)
    edges, fd, rows = c["edges"], c["fd"], c["rows"]
    contributions = 4 * c["ff"] + fd + c["fixed"]
    # compulsory bytes: conductances read once; per slot its pointer, its
    # contribution codes and the FP64 + FP32 values written; per row its
    # pointer, fixed flag and pressure, its (edge, node) pairs and b written
    algo = (8 * edges + 4 * (nnz + 1) + 4 * contributions + 12 * nnz + 4 * (rows + 1) + 8 * fd
            + (1 + 8 + 8) * rows)
    print(f"{a.systems} networks: {rows} nodes, {edges} edges, {nnz} entries, {contributions} contributions; "
          f"plan built in {time.perf_counter() - t0:.1f} s; compulsory bytes per assembly {algo / 1e6:.1f} MB",
          flush=True)
    stream = torch.cuda.current_stream()
    gd = torch.tensor(pk.conductance, device="cuda")

    def timed(fn, reps=10):
        fn()
        torch.cuda.synchronize()
        best = None
        for _ in range(reps):
            e0, e1 = _events(torch)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        return best

    ms_dev = timed(lambda: nb.assemble(gd))
    ms_host_in = timed(lambda: nb.assemble(pk.conductance))
    t0 = time.perf_counter()
    network_assemble_host(pk, pk.conductance)
    ms_cpu = (time.perf_counter() - t0) * 1e3
    print(f"assemble, device conductances: {ms_dev * 1e3:.1f} us ({algo / ms_dev / 1e6:.0f} GB/s on compulsory "
          f"bytes, includes the 4-byte status read back); host conductances (+ H2D): {ms_host_in * 1e3:.1f} us; "
          f"the same code on one host core: {ms_cpu:.1f} ms", flush=True)
    cfg = cf.IterativeSolverConfig(0.0, 1e-10, 40000)
    x = torch.zeros(pk.rows, dtype=torch.float64, device="cuda")
    nb.assemble(gd)
    nb.solve(None, x, config=cfg)
    g1 = gd * 1.01
    x_warm = x.clone()

    def picard():
        nb.assemble(g1)
        x.copy_(x_warm)
        return nb.solve(None, x, config=cfg)
    ms_pass = timed(picard, reps=3)
    _, rep = picard()
    print(f"Picard pass (assemble + warm solve, FP64): {ms_pass:.2f} ms, converged {rep.converged_systems}/"
          f"{rep.num_systems}, iterations total {rep.total_iterations}", flush=True)
    return 0


def simple_case(a):
    """GMRES(30) + SIMPLE (the saddle-point tier) on the MAC-grid Stokes system
    of --n cells per side, FP64 and FP32 inside FP64 refinement: device time,
    iterations, time per iteration and the true relative residual."""
    import time

    import numpy as np
    import torch

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    t0 = time.perf_counter()
    A, b, nv = P.stokes_2d_mac(a.n)
    M = cf.SimplePreconditioner(A, nv)
    print(f"Stokes MAC {a.n}^2: {A.shape[0]} unknowns ({nv} velocity), {A.nnz} nonzeros; built and set up in "
          f"{time.perf_counter() - t0:.1f} s", flush=True)
    bd = torch.tensor(b, device="cuda")
    S = A.to_scipy()
    cfg = cf.IterativeSolverConfig(0.0, 1e-8, 200000)
    for prec in (cf.Precision.FP64, cf.Precision.FP32_REFINE):
        best = None
        for _ in range(3):
            x = torch.zeros_like(bd)
            torch.cuda.synchronize()
            r = cf.gmres_preconditioned(A, bd, M, x, cfg, restart=30, precision=prec)
            best = r if best is None or r.device_ms < best.device_ms else best
        xs = x.cpu().numpy()
        res = np.linalg.norm(b - S @ xs) / np.linalg.norm(b)
        print(f"GMRES(30)+SIMPLE {prec.name}: {best.device_ms:.2f} ms device, {best.iterations} iterations "
              f"({best.device_ms / max(best.iterations, 1) * 1e3:.1f} us each), {best.termination.name}, "
              f"true relative residual {res:.2e}", flush=True)
    return 0


def adjoint_case(a):
    """2-D Darcy, n x n cells, k = exp(theta), theta a GRF (l = 16, sigma = 0.5);
    L = sum p^2 over the cell column at x = 0.75; dL/dtheta by the device
    adjoint (forward and adjoint FP32 + FP64 refinement to 1e-10). Times one
    theta update end to end (assembly, forward solve, adjoint solve, chain
    rule) with the Galerkin operators recomputed for the new values and with
    the hierarchy kept. The gradient's accuracy against the FP64 CPU adjoint
    and central differences is asserted by tests/test_gpu_adjoint.py."""
    import time

    import torch

    import cfdrs_b200 as cf
    from cfdrs_b200 import problems as P
    from cfdrs_b200.adjoint import (SparseSolver, column_loss, darcy_2d_pattern, darcy_2d_solve, darcy_2d_torch,
                                    loss_column_index, sparse_solve)

    n = a.n
    theta = P.gaussian_random_field((n, n), 16.0, 0.5, seed=0)
    col = loss_column_index(n)
    pattern, mask = darcy_2d_pattern(n)
    maskd = torch.as_tensor(mask, device="cuda")
    th = torch.as_tensor(theta, device="cuda")

    def generic(t, s, first):  # torch assembly, SparseSolveFunction, autograd through the assembly
        vals, b = darcy_2d_torch(t, maskd)
        return sparse_solve(vals, b, s, first)

    def fused(t, s, first):  # DarcySolveFunction: assembly and chain rule each one kernel
        return darcy_2d_solve(t, s, first)

    for name, fn in (("fused", fused), ("generic", generic)):
        s = SparseSolver(pattern, precision=cf.Precision.FP32_REFINE,
                         config=cf.IterativeSolverConfig(0.0, 1e-10, 500))

        def update(first=False):
            t = th.clone().requires_grad_(True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p = fn(t, s, first)
            fwd = s.last_report
            L = column_loss(p, n, col)
            L.backward()
            torch.cuda.synchronize()
            return (time.perf_counter() - t0) * 1e3, fwd, s.last_report, L.item()

        first_ms = update(True)[0]
        times = []
        for _ in range(3):
            ms, fwd, adj, L = update()
            times.append(ms)
        print(f"{n}^2 {name}: L = {L:.10e}; forward solve {fwd.device_ms:.1f} ms device ({fwd.iterations} inner "
              f"its), adjoint solve {adj.device_ms:.1f} ms device", flush=True)
        s.refresh = "keep"
        keep = [update()[0] for _ in range(3)]
        s.refresh = "recompute"
        print(f"  per theta update end to end: {min(times):.1f} ms with the Galerkin recompute, "
              f"{min(keep):.1f} ms keeping the hierarchy (first call with AMG setup {first_ms:.1f} ms)", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

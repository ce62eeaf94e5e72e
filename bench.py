#!/usr/bin/env python
"""Benchmark: FP64 BiCGSTAB to 1e-8 relative residual on one B200, plus the
H-matvec HBM throughput, on the plain-FP64 workload (configuration C1):

  Laplace single layer 1/(4 pi r), unit icosphere level 5 (20,480 flat
  triangles), piecewise-constant collocation at centroids with the analytic
  flat-triangle integral (self term included), HACApK cluster tree with leaf
  size 32, admissibility eta = 2.0, ACA+ tolerance 1e-5; rhs = 1 + N(0,1e-3^2)
  per element (seed 0); BiCGSTAB from x0 = 0 to ||r||/||b|| < 1e-8.

A step is one complete solve.  `value` is seconds per solve with b resident in
HBM (CUDA events on the launching stream, max over ranks); `e2e` is the same
solve through the host-vector C-ABI call (hbx_bicgstab_host: b and x0 copied
in, the solution copied out, inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank solves its own replica: the solve is one
shared H-matrix per GPU and no data moves between ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hacapk-magma_b200"))
sys.path.insert(0, ROOT)

METRIC = "BiCGSTAB s to 1e-8 rel. residual; H-matvec HBM GB/s (% peak), 1 B200"
WORKLOAD = ("C1 plain FP64: Laplace single layer on a unit icosphere L5 (20,480 triangles), "
            "leaf 32, eta 2.0, ACA+ 1e-5, rhs 1+N(0,1e-3^2) seed 0, BiCGSTAB to 1e-8 from x0=0")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == "C1":
            return float(parts[2])
    return None


class Clocks:
    """nvidia-smi sampler for the timed region.  start() returns once the
    sampler has written its first line (nvidia-smi takes a good part of a
    second to come up, longer than a short timed region), and that line is
    dropped: the samples kept are the ones taken from the start of the timed
    region to stop()."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, index: int, exe: str = "nvidia-smi"):
        self.index = index
        self.exe = exe
        self.proc = None

    def start(self, ready_timeout_s: float = 10.0):
        import select
        try:
            self.proc = subprocess.Popen([self.exe, "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        except OSError:
            self.proc = None
            return
        # the sample taken before the timed region, read from the descriptor
        # itself (communicate() reads the descriptor, not the text buffer)
        fd = self.proc.stdout.fileno()
        deadline = time.monotonic() + ready_timeout_s
        while True:
            left = deadline - time.monotonic()
            if left <= 0 or not select.select([fd], [], [], left)[0]:
                break
            ch = os.read(fd, 1)
            if not ch or ch == b"\n":
                break

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, err = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, err = self.proc.communicate()
        if not out.strip() and err.strip():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi: " + err.strip()[:200]]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl" if os.environ.get("HBX_BENCH_BACKEND", "nccl") == "nccl" else "gloo",
                                timeout=timedelta(seconds=300))
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def vector_bytes_per_iteration(n: int) -> int:
    """HBM bytes of the vector traffic of one iteration launch besides the two
    H-matvecs: p update (r, p, Ap read, p write), rh.Ap, t = r - alpha Ap,
    At.t / At.At, u and r updates with rh.r / r.r."""
    return 8 * n * (4 + 2 + 3 + 2 + 8)


def run_ours(args, world, rank, local):
    import torch
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t0 = time.time()
    H, b = configs.c1(args.level)
    t_build = time.time() - t0
    E = Engine(H.st, H.nd)
    info = E.info
    n = H.nd
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    bd = torch.from_numpy(b).to(dev)
    ud = torch.zeros(n, dtype=torch.float64, device=dev)
    # ---- warm-up solves (untimed)
    for _ in range(max(args.warmup, 3)):
        ud.zero_()
        E.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
    torch.cuda.synchronize(dev)
    # ---- timed region: K device-resident solves
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    infos = []
    for _ in range(args.steps):
        ud.zero_()
        infos.append(E.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter,
                                    stream=s))
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = reduce_max(ms, world)
    iters = infos[-1]["iterations"]
    launches = int(sum(i["launches"] for i in infos))  # kernels of this library only
    # ---- e2e: the same solve through the host-vector C-ABI call
    b_host = torch.from_numpy(b).pin_memory().numpy()
    u_host = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    E.bicgstab_host(b_host, u_host, tol=args.tol, max_iter=args.max_iter)
    barrier(world)
    torch.cuda.synchronize(dev)
    te0 = time.perf_counter()
    for _ in range(args.steps):
        u_host[:] = 0.0
        E.bicgstab_host(b_host, u_host, tol=args.tol, max_iter=args.max_iter, inplace=True)
    torch.cuda.synchronize(dev)
    e2e_s = (time.perf_counter() - te0) / args.steps
    clk = clocks.stop()
    e2e_s = reduce_max(e2e_s, world)
    # ---- iteration-kernel roofline (device time of the iteration launches)
    it_s = sum(i["iter_kernel_seconds"] for i in infos)
    it_n = sum(i["iterations"] for i in infos)
    per_iter_s = it_s / max(1, it_n)
    bytes_iter = 2 * info["alg_bytes"] + vector_bytes_per_iteration(n)
    peak, peak_kind = peaks()
    achieved = bytes_iter / per_iter_s / 1e9
    # ---- standalone H-matvec throughput (secondary metric)
    x = torch.randn(n, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    for _ in range(5):
        E.matvec_dev(x.data_ptr(), y.data_ptr(), stream=s)
    torch.cuda.synchronize(dev)
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 50
    m0.record(stream)
    for _ in range(reps):
        E.matvec_dev(x.data_ptr(), y.data_ptr(), stream=s)
    m1.record(stream)
    torch.cuda.synchronize(dev)
    E.sync(s)
    mv_us = m0.elapsed_time(m1) / reps * 1e3
    mv_gbs = info["alg_bytes"] / (mv_us * 1e-6) / 1e9
    # the forms are a single-GPU report (like cpu_baseline): the scaling runs
    # time the FP64 solve only
    forms = None if (args.no_forms or world > 1) else measure_forms(args, dev, stream)
    out = {
        "metric": METRIC,
        "value": ms / 1e3,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded icosphere mesh and rhs)",
        "config": {
            "workload": WORKLOAD,
            "n": n,
            "iterations": iters,
            "true_relres": infos[-1]["true_relres"],
            "h_alg_bytes": info["alg_bytes"],
            "dense_words": info["dense_words"],
            "lowrank_words": info["lowrank_words"],
            "l2": "inputs larger than L2: the packed H-matrix is %.0f MB > 126 MB" % (info["stream_bytes"] / 1e6),
            "parallelism": "replicas" if world > 1 else "1 GPU",
            "build_seconds": t_build,
            "setup_seconds": info["setup_seconds"],
        },
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n},
        "hmatvec": {"us": mv_us, "gbs": mv_gbs, "frac_of_" + peak_kind + "_peak": mv_gbs / peak},
        "roofline": {
            "kernel": "k_bicg_iter (one BiCGSTAB step: 2 H-matvecs + vector updates + dots)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": ncu_traffic("k_bicg_iter"),
            "alg_bytes_per_launch": bytes_iter,
            "avg_launch_us": per_iter_s * 1e6,
        },
        "clocks": clk,
        "gpu_launches": launches,
    }
    if forms is not None:
        out["forms"] = forms
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(H, b, args)
    return out


def precision_workload(args):
    """--precision-level L: only the precision form, on C2 at level L."""
    import torch
    dev = torch.device("cuda", 0)
    print(json.dumps(precision_form(args, dev, torch.cuda.current_stream(dev), args.precision_level)), flush=True)


def forms_only(args):
    """--forms-only: only the forms on their configurations (one GPU)."""
    import torch
    dev = torch.device("cuda", 0)
    print(json.dumps(measure_forms(args, dev, torch.cuda.current_stream(dev))), flush=True)


def _timed(dev, fn, reps=3):
    """Best host-clock time of fn() over reps runs after one untimed run, with
    the device synchronized on both sides; returns (seconds, last result)."""
    import torch
    best, res = 1e9, None
    for _ in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = fn()
        torch.cuda.synchronize(dev)
        best = min(best, time.perf_counter() - t0)
    return best, res


def measure_forms(args, dev, stream):
    """The forms beside the FP64 drop-in, each on the workload its
    configuration names, each against the FP64 solve of that same workload
    and each verified by the FP64 residual ||b - H u||/||b|| (recomputed
    after the solve):

      precision_c2  C2: FP32 and BF16 factors inside FP64 refinement;
      mrhs_c3       C3: 64 right-hand sides on the tensor cores, against 64
                    FP64 solves one after another;
      adjoint_c4    C4: dJ/dg by the adjoint solve with the transposed
                    product, checked against central differences in 16
                    random directions;
      batch_c5      C5: 256 uneven bodies in one block-diagonal engine,
                    against the same bodies solved one after another;
      autotune_c1   C1: the autotuner's schedule and layout against the
                    defaults (product and solve);
      solvers_c1    C1: the reference's other iterative solvers on the GPU
                    (pipelined BiCGSTAB, GCR(8)), each beside its CPU loop
                    on every host core.

    The H-matrices are filled on the GPU (hbx_fill_leaves)."""
    forms = {"solvers_c1": solvers_form, "autotune_c1": autotune_form, "precision_c2": precision_form,
             "mrhs_c3": mrhs_form, "adjoint_c4": adjoint_form, "batch_c5": batch_form}
    want = getattr(args, "form", "")
    out = {}
    for name, fn in forms.items():
        if want and want != name:
            continue
        try:
            out[name] = fn(args, dev, stream)
        except Exception as e:  # one form's failure is reported beside the others, not fatal to the line
            out[name] = {"error": f"{type(e).__name__}: {e}"[:500]}
    return out


def autotune_form(args, dev, stream, level=5):
    """C1: hbx_autotune's choice (CTA schedule, merged D+U layout, L2 budget)
    against the defaults: the product time of each, and the BiCGSTAB solve
    (CUDA events) with the tuned engine against the default engine."""
    import torch
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    s = stream.cuda_stream
    H, b = configs.c1(level)
    t0 = time.time()
    kw, best_us, def_us = Engine.autotune(H.st, H.nd, reps=20)
    t_tune = time.time() - t0
    bd = torch.from_numpy(b).to(dev)
    ud = torch.zeros_like(bd)
    out = {"workload": f"C1: icosphere L{level}, N = {H.nd}", "tuned_options": kw, "tune_seconds": t_tune,
           "matvec_us": {"tuned": best_us, "default": def_us}}
    for name, opts in (("default", {}), ("tuned", kw)):
        E = Engine(H.st, H.nd, **opts)
        best = 1e9
        for _ in range(4):
            ud.zero_()
            inf = E.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
            best = min(best, inf["seconds"])
        out[f"solve_s_{name}"] = best
        out[f"iterations_{name}"] = inf["iterations"]
        E.close()
    H.close()
    return out


def solvers_form(args, dev, stream, level=5):
    """C1: the pipelined BiCGSTAB (HACApK_SOLVER_PIPE.c:144, :640) and GCR(8)
    (m_HACApK_solve.f90:506-571) to 1e-8, device vectors (CUDA-event time of
    the solve) and host vectors (the reference-facing call with its copies,
    host clock), each beside the same loop on the CPU (the oracle's
    restatement with the reference's OpenMP product on every host core)."""
    import oracle
    import torch
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    s = stream.cuda_stream
    H, b = configs.c1(level, fill="gpu")
    n = H.nd
    E = Engine(H.st, n)
    bd = torch.from_numpy(b).to(dev)
    ud = torch.zeros(n, dtype=torch.float64, device=dev)
    cores = len(os.sched_getaffinity(0))
    out = {"workload": f"C1: icosphere L{level}, N = {n}, rhs 1+N(0,1e-3^2), to 1e-8", "n": n}
    runs = (
        ("bicgstab_pipe", lambda: E.bicgstab_pipe_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol,
                                                      max_iter=args.max_iter, stream=s),
         lambda: E.bicgstab_pipe_host(b, tol=args.tol, max_iter=args.max_iter),
         lambda: oracle.bicgstab_pipe(H.st, b, tol=args.tol, max_iter=args.max_iter, kind="omp", nthreads=cores)),
        ("gcr8", lambda: E.gcr_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, restart=8,
                                   stream=s),
         lambda: E.gcr_host(b, tol=args.tol, max_iter=args.max_iter, restart=8),
         lambda: oracle.gcrm(H.st, b, tol=args.tol, max_iter=args.max_iter, restart=8, kind="omp",
                             nthreads=cores)),
    )
    for name, dev_solve, host_solve, cpu_solve in runs:
        best, inf = 1e9, None
        for _ in range(4):
            ud.zero_()
            inf = dev_solve()
            best = min(best, inf["seconds"])
        t_host, (u, hinf) = _timed(dev, host_solve)
        t0 = time.perf_counter()
        _, n_cpu, hist, _ = cpu_solve()
        t_cpu = time.perf_counter() - t0
        out[name] = {"solve_s": best, "e2e_s": t_host, "iterations": inf["iterations"],
                     "true_relres": hinf["true_relres"], "us_per_step": best / max(inf["iterations"], 1) * 1e6,
                     "cpu": {"solve_s": t_cpu, "iterations": n_cpu, "cores": cores, "kind": "port",
                             "relres": float(hist[-1])},
                     "speedup_e2e_vs_cpu": t_cpu / t_host}
    E.close()
    H.close()
    return out


def precision_form(args, dev, stream, level=7):
    """C2 at `level` (7: the configuration): the FP64 solve, FP32 factors in
    FP64 refinement, BF16 factors in FP64 refinement (inner tolerance 1e-2);
    each with its product's time and stream rate."""
    import torch
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    s = stream.cuda_stream
    t0 = time.time()
    H, b = configs.c2(level, fill="gpu")
    t_build = time.time() - t0
    n = H.nd
    bd = torch.from_numpy(b).to(dev)
    ud = torch.zeros(n, dtype=torch.float64, device=dev)
    peak, peak_kind = peaks()

    def product(Ek):
        x = torch.randn(n, dtype=torch.float64, device=dev)
        y = torch.empty_like(x)
        for _ in range(3):
            Ek.matvec_dev(x.data_ptr(), y.data_ptr(), stream=s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(20):
            Ek.matvec_dev(x.data_ptr(), y.data_ptr(), stream=s)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        Ek.sync(s)
        us = e0.elapsed_time(e1) / 20 * 1e3
        return {"us": us, "stream_gb": Ek.info["stream_bytes"] / 1e9,
                "stream_gbs": Ek.info["stream_bytes"] / (us * 1e-6) / 1e9,
                "frac_of_" + peak_kind + "_peak": Ek.info["stream_bytes"] / (us * 1e-6) / 1e9 / peak}

    E = Engine(H.st, n)

    def solve64():
        ud.zero_()
        return E.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
    t64, inf = _timed(dev, solve64)
    out = {"workload": f"C2: icosphere L{level} + seeded ellipsoid (semi-axes U(0.5,2), gap 3), leaf 32, eta 2, "
                       "ACA+ 1e-6, rhs 1+N(0,1e-3^2); BiCGSTAB to an FP64-verified 1e-8",
           "n": n, "gpu_fill_s": t_build,
           "fp64": {"solve_s": t64, "iterations": inf["iterations"], "true_relres": inf["true_relres"],
                    "product": product(E)}}
    for name, prec, inner in (("fp32_refined", abi.HBX_FP32, 0.0), ("bf16_refined", abi.HBX_BF16, 1e-2)):
        El = Engine(H.st, n, precision=prec)

        def solve_l():
            ud.zero_()
            return E.bicgstab_refined_dev(El, bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter,
                                          inner_tol=inner, stream=s)
        tl, inf = _timed(dev, solve_l)
        out[name] = {"solve_s": tl, "speedup_vs_fp64": t64 / tl, "outer": inf["outer"],
                     "inner_iterations": inf["iterations"], "true_relres": inf["true_relres"],
                     "product": product(El)}
        El.close()
    E.close()
    H.close()
    return out


def mrhs_form(args, dev, stream, level=6):
    """C3: 64 seeded N(0,1) right-hand sides on the L6 sphere solved at once
    (tensor-core products, FP64 refinement, per-RHS masks) against the same
    64 solved one after another by the FP64 solver."""
    import torch
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    s = stream.cuda_stream
    t0 = time.time()
    H, B = configs.c3(level, abi.HBX_NRHS, fill="gpu")
    t_build = time.time() - t0
    n = H.nd
    E = Engine(H.st, n)
    Em = Engine(H.st, n, precision=abi.HBX_FP32, nrhs=abi.HBX_NRHS)
    Bd = torch.from_numpy(B).to(dev)
    Ud = torch.zeros_like(Bd)

    def multi():
        Ud.zero_()
        return E.bicgstab_multi_dev(Em, Bd.data_ptr(), Ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
    t_multi, infos = _timed(dev, multi, reps=2)
    # the 64 right-hand sides one after another (FP64 solver)
    cols = [torch.from_numpy(np.ascontiguousarray(B[:, j])).to(dev) for j in range(abi.HBX_NRHS)]
    u1 = torch.zeros(n, dtype=torch.float64, device=dev)

    def one_by_one():
        res = []
        for bj in cols:
            u1.zero_()
            res.append(E.bicgstab_dev(bj.data_ptr(), u1.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s))
        return res
    t_one, res1 = _timed(dev, one_by_one, reps=1)
    X = torch.randn(n, abi.HBX_NRHS, device=dev).float()
    Y = torch.zeros(n, abi.HBX_NRHS, dtype=torch.float64, device=dev)
    for _ in range(3):
        Em.matmat_dev(X.data_ptr(), Y.data_ptr(), stream=s)
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0.record(stream)
    for _ in range(20):
        Em.matmat_dev(X.data_ptr(), Y.data_ptr(), stream=s)
    m1.record(stream)
    torch.cuda.synchronize(dev)
    Em.sync(s)
    mm_us = m0.elapsed_time(m1) / 20 * 1e3
    its = [i["iterations"] for i in infos]
    out = {"workload": f"C3: icosphere L{level}, leaf 32, eta 2, ACA+ 1e-5, 64 right-hand sides N(0,1) seed 2; "
                       "FP32 tensor-core products in FP64 refinement to an FP64-verified 1e-8",
           "n": n, "rhs": abi.HBX_NRHS, "gpu_fill_s": t_build,
           "solve_s": t_multi, "fp64_one_by_one_s": t_one, "speedup_vs_fp64": t_one / t_multi,
           "worst_true_relres": max(i["true_relres"] for i in infos),
           "converged": int(sum(i["status"] == 0 for i in infos)),
           "inner_iterations": [min(its), max(its)], "outer": max(i["outer"] for i in infos),
           "fp64_iterations": [min(r["iterations"] for r in res1), max(r["iterations"] for r in res1)],
           "matmat_us": mm_us, "matmat_tf32_tflops": abi.HBX_NRHS * Em.info["alg_flops"] / (mm_us * 1e-6) / 1e12}
    Em.close()
    E.close()
    H.close()
    return out


def adjoint_form(args, dev, stream, level=6, ndir=16, step=1e-6):
    """C4: J(g) = 0.5 ||sigma(g) - sigma_t||^2 with H sigma = g on the L6
    sphere (FP64); dJ/dg by the adjoint solve on the transposed engine
    (hbx_gradient_host), checked against central differences in 16 seeded
    random directions (step 1e-6, solves to 1e-12)."""
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    t0 = time.time()
    H, g, st = configs.c4(level, fill="gpu")
    t_build = time.time() - t0
    n = H.nd
    E = Engine(H.st, n)
    Et = Engine(H.st, n, transpose=True)
    t_grad, res = _timed(dev, lambda: E.gradient_host(Et, g, st, tol=1e-12, max_iter=args.max_iter), reps=2)
    J, grad, sigma, fi, ai = res

    def J_of(gv):
        u, _ = E.bicgstab_host(gv, tol=1e-12, max_iter=args.max_iter)
        return 0.5 * float(np.dot(u - st, u - st))
    t_solve, _ = _timed(dev, lambda: E.bicgstab_host(g, tol=1e-12, max_iter=args.max_iter), reps=2)
    rng = np.random.default_rng(16)
    errs = []
    for _ in range(ndir):
        d = rng.standard_normal(n)
        d /= np.linalg.norm(d)
        fd = (J_of(g + step * d) - J_of(g - step * d)) / (2 * step)
        ad = float(np.dot(grad, d))
        errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
    out = {"workload": f"C4: icosphere L{level}, leaf 32, eta 2, ACA+ 1e-5, FP64; g, sigma_t N(0,1) (seeds 3, 4); "
                       "adjoint BiCGSTAB on the transposed H-matvec, 16 central-difference directions (step 1e-6)",
           "n": n, "gpu_fill_s": t_build, "gradient_s": t_grad, "fp64_solve_s": t_solve,
           "gradient_vs_two_solves": t_grad / (2 * t_solve),
           "fd_max_rel_err": max(errs), "fd_median_rel_err": float(np.median(errs)),
           "forward_iterations": fi["iterations"], "adjoint_iterations": ai["iterations"],
           "adjoint_true_relres": ai["true_relres"]}
    Et.close()
    E.close()
    H.close()
    return out


def batch_form(args, dev, stream):
    """C5: the 256 uneven ellipsoids solved in one block-diagonal engine
    (FP64, and FP32 / BF16 corrections in FP64 refinement) against the same
    bodies solved one after another (FP64 each)."""
    import torch
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    s = stream.cuda_stream
    t0 = time.time()
    inst = configs.c5(count=args.c5_count, fill="gpu")
    t_build = time.time() - t0
    Eb = Engine.batch([Hk for Hk, _ in inst])
    bb = torch.from_numpy(np.concatenate([bk for _, bk in inst])).to(dev)
    ub = torch.zeros_like(bb)

    def batch():
        ub.zero_()
        return Eb.bicgstab_batch_dev(bb.data_ptr(), ub.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
    t_batch, infos = _timed(dev, batch, reps=2)
    stream_gb = Eb.info["stream_bytes"] / 1e9
    # the configuration's mixed precision: FP32 (or BF16) factors for the
    # corrections inside FP64 refinement, one batch engine each
    refined = {}
    for name, prec, inner in (("fp32_refined", abi.HBX_FP32, 0.0), ("bf16_refined", abi.HBX_BF16, 1e-2)):
        El = Engine.batch([Hk for Hk, _ in inst], precision=prec)

        def batch_ref():
            ub.zero_()
            return Eb.bicgstab_batch_refined_dev(El, bb.data_ptr(), ub.data_ptr(), tol=args.tol,
                                                 max_iter=args.max_iter, inner_tol=inner, stream=s)
        t_ref, rinf = _timed(dev, batch_ref, reps=2)
        refined[name] = {"solve_s": t_ref, "stream_gb": El.info["stream_bytes"] / 1e9,
                         "outer": max(i["outer"] for i in rinf), "inner_iterations_max": max(i["iterations"] for i in rinf),
                         "worst_true_relres": max(i["true_relres"] for i in rinf),
                         "converged": int(sum(i["status"] == 0 for i in rinf))}
        El.close()
    Eb.close()
    engines = [(Engine(Hk.st, Hk.nd), torch.from_numpy(bk).to(dev)) for Hk, bk in inst]
    us = [torch.zeros_like(bd) for _, bd in engines]

    def one_by_one():
        for (Ek, bd), ud in zip(engines, us):
            ud.zero_()
            Ek.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
    t_one, _ = _timed(dev, one_by_one, reps=1)
    for Ek, _ in engines:
        Ek.close()
    its = [i["iterations"] for i in infos]
    out = {"workload": f"C5: {len(inst)} ellipsoids, semi-axes U(0.3,3), icosphere levels 2-5 (seed 5), leaf 32, "
                       "eta 2, ACA+ 1e-5, FP64; one block-diagonal engine against one solve after another",
           "instances": len(inst), "n_total": int(sum(Hk.nd for Hk, _ in inst)), "stream_gb": stream_gb,
           "gpu_fill_s": t_build, "solve_s": t_batch, "one_by_one_s": t_one, "speedup": t_one / t_batch,
           "iterations": [min(its), max(its)], "worst_true_relres": max(i["true_relres"] for i in infos),
           "converged": int(sum(i["status"] == 0 for i in infos))}
    for name, r in refined.items():
        r["speedup_vs_one_by_one"] = t_one / r["solve_s"]
        out[name] = r
    for Hk, _ in inst:
        Hk.close()
    return out


def profile_products(args):
    """--profile-products L: C2 at level L (GPU fill), one engine per factor
    precision (FP64, FP32, BF16), three single-vector products each, nothing
    timed: the command the product profiles are taken from (launch 1 + 3k of
    k_matvec is precision k's second product)."""
    import torch
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c2(args.profile_products, fill="gpu")
    x = torch.randn(H.nd, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    out = {}
    for name, prec in (("fp64", abi.HBX_FP64), ("fp32", abi.HBX_FP32), ("bf16", abi.HBX_BF16)):
        E = Engine(H.st, H.nd, precision=prec)
        for _ in range(3):
            E.matvec_dev(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        E.sync()
        out[name] = E.info["stream_bytes"]
        E.close()
    print(json.dumps({"profile_products": args.profile_products, "stream_bytes": out}), flush=True)


def profile_matmat(args):
    """Five 64-RHS products on the C1 workload, nothing timed: the command
    the ncu summary of k_matmat is taken from."""
    import torch
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(args.level)
    E = Engine(H.st, H.nd, precision=abi.HBX_FP32, nrhs=abi.HBX_NRHS)
    X = torch.randn(H.nd, abi.HBX_NRHS, device="cuda").float()
    Y = torch.zeros(H.nd, abi.HBX_NRHS, dtype=torch.float64, device="cuda")
    for _ in range(5):
        E.matmat_dev(X.data_ptr(), Y.data_ptr())
    torch.cuda.synchronize()
    E.sync()
    print(json.dumps({"profile_matmat": True, "stream_bytes": E.info["stream_bytes"]}), flush=True)


def cpu_baseline(H, b, args):
    """The compiled reference CPU H-matvec (HACApK_MAGMA.c:5-57, one thread as
    written) inside the BiCGSTAB of HACApK_SOLVER.c:254-417: one full solve."""
    import oracle
    kind = "ref" if oracle.have_ref() else "restated"
    t0 = time.perf_counter()
    u, n, hist, mv_s = oracle.bicgstab(H.st, b, tol=args.tol, max_iter=args.max_iter, kind=kind)
    dt = time.perf_counter() - t0
    return {"value": dt, "unit": "s", "cores": 1, "kind": "reference" if kind == "ref" else "port",
            "sample": f"one full C1 solve on the host: {n} iterations, matvec time {mv_s:.2f} s",
            "iterations": n, "host_matvec": host_matvecs(H)}


def host_matvecs(H, seconds: float = 2.0) -> dict:
    """The reference's CPU products on the host cores, ms per H-matvec (each
    repeated for about `seconds`): the CPU-BLAS path of HACApK_MAGMA.c:140-187
    (one dgemv per leaf; OpenBLAS as bundled with scipy stands in for MKL) on
    one thread and on every core, and the OpenMP product of
    m_HACApK_solve.f90:203-253 (restated in C) on every core."""
    import oracle
    from threadpoolctl import threadpool_limits
    cores = len(os.sched_getaffinity(0))
    x = np.random.default_rng(0).standard_normal(H.nd)

    def per_call(fn):
        fn()
        t0, k = time.perf_counter(), 0
        while time.perf_counter() - t0 < seconds:
            fn()
            k += 1
        return (time.perf_counter() - t0) / k * 1e3

    out = {"cores": cores}
    for nt in (1, cores):
        with threadpool_limits(limits=nt, user_api="blas"):
            out[f"blas_gemv_ms_{nt}_threads"] = per_call(lambda: oracle.matvec_blas(H.st, x))
    out[f"omp_ms_{cores}_threads"] = per_call(lambda: oracle.matvec_omp(H.st, x, nthreads=cores))
    return out


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU H-matvec on every host core.

    The reference's threaded CPU product is the OpenMP "_hyp" form of
    m_HACApK_solve.f90:203-253 (per-thread accumulators over the leaf list,
    summed afterwards); its Fortran needs gfortran, which this image lacks, so
    the oracle's C restatement of it runs here, inside the BiCGSTAB of
    HACApK_SOLVER.c:254-417.  A step is one full solve of the workload."""
    if rank != 0:
        return None
    from hacapk_b200 import configs
    import oracle
    H, b = configs.c1(args.level)
    cores = len(os.sched_getaffinity(0))
    for _ in range(args.warmup):
        oracle.bicgstab(H.st, b, tol=args.tol, max_iter=args.max_iter, kind="omp", nthreads=cores)
    times, n = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, n, _, _ = oracle.bicgstab(H.st, b, tol=args.tol, max_iter=args.max_iter, kind="omp", nthreads=cores)
        times.append(time.perf_counter() - t0)
    v = float(np.mean(times))
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded icosphere mesh and rhs)",
        "config": {"workload": WORKLOAD, "n": H.nd, "iterations": n},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "port",
                         "sample": "full C1 solves: the OpenMP H-matvec of m_HACApK_solve.f90:203-253 (restated in C) "
                                   f"on {cores} threads in the BiCGSTAB of HACApK_SOLVER.c:254-417"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--level", type=int, default=5)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-iter", type=int, default=2000)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the forms on their configurations (C2 precision, C3 multi-RHS, C4 adjoint, C5 batch)")
    ap.add_argument("--c5-count", type=int, default=256, help="instances of the uneven batch (C5: 256)")
    ap.add_argument("--forms-only", action="store_true", help="only the forms on their configurations")
    ap.add_argument("--form", default="", help="with --forms-only: only this form (e.g. solvers_c1)")
    ap.add_argument("--profile-matmat", action="store_true",
                    help="only run five 64-RHS tensor-core products (a short command for ncu)")
    ap.add_argument("--profile-products", type=int, default=0,
                    help="only run a few FP64/FP32/BF16 products on C2 at this level (a short command for ncu)")
    ap.add_argument("--precision-level", type=int, default=0,
                    help="only time the precision form on C2 at this level (7: the config; one GPU)")
    args = ap.parse_args()
    if args.profile_matmat:
        profile_matmat(args)
        return
    if args.profile_products > 0:
        profile_products(args)
        return
    if args.precision_level > 0:
        precision_workload(args)
        return
    if args.forms_only:
        forms_only(args)
        return
    world, rank, local = dist_setup()
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    else:
        out = run_ours(args, world, rank, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

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
    forms = None if (args.no_forms or world > 1) else measure_forms(H, b, E, args, dev, stream, ms / 1e3)
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


def measure_forms(H, b, E, args, dev, stream, fp64_solve_s):
    """The precision and batching forms beside the FP64 solve (same matrix,
    same tolerance, verified by the FP64 residual): FP32 factors inside FP64
    refinement, 64 right-hand sides at once on the tensor cores, and a batch
    of uneven bodies in one block-diagonal engine."""
    import numpy as np
    import torch
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine
    s = stream.cuda_stream
    n = H.nd
    reps = 3
    out = {}
    bd = torch.from_numpy(b).to(dev)
    ud = torch.zeros(n, dtype=torch.float64, device=dev)
    # the FP64 solve timed like the forms (host clock around each call, best
    # of the repetitions), so every speed-up below compares like with like
    best = 1e9
    for _ in range(reps + 1):
        ud.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        E.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
        torch.cuda.synchronize(dev)
        best = min(best, time.perf_counter() - t0)
    fp64_solve_s = best
    out["fp64_solve_s"] = best
    # FP32 factors, FP64 refinement, single right-hand side
    E32 = Engine(H.st, n, precision=abi.HBX_FP32)
    best, inf = 1e9, None
    for _ in range(reps + 1):
        ud.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        inf = E.bicgstab_refined_dev(E32, bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
        torch.cuda.synchronize(dev)
        best = min(best, time.perf_counter() - t0)
    out["fp32_refined"] = {"solve_s": best, "true_relres": inf["true_relres"], "inner_iterations": inf["iterations"],
                           "outer": inf["outer"], "speedup_vs_fp64": fp64_solve_s / best}
    E32.close()
    # 64 right-hand sides: the rhs above plus 63 seeded N(0,1) ones
    Em = Engine(H.st, n, precision=abi.HBX_FP32, nrhs=abi.HBX_NRHS)
    rng = np.random.default_rng(2)
    B = rng.standard_normal((n, abi.HBX_NRHS))
    B[:, 0] = b
    Bd = torch.from_numpy(B).to(dev)
    Ud = torch.zeros_like(Bd)
    best, infos = 1e9, None
    for _ in range(reps + 1):
        Ud.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        infos = E.bicgstab_multi_dev(Em, Bd.data_ptr(), Ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
        torch.cuda.synchronize(dev)
        best = min(best, time.perf_counter() - t0)
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
    out["mrhs64"] = {
        "rhs": abi.HBX_NRHS, "solve_s": best, "per_rhs_s": best / abi.HBX_NRHS,
        "speedup_vs_fp64_per_rhs": fp64_solve_s * abi.HBX_NRHS / best,
        "worst_true_relres": max(i["true_relres"] for i in infos), "converged": sum(i["status"] == 0 for i in infos),
        "inner_iterations": [min(its), max(its)], "outer": infos[0]["outer"],
        "matmat_us": mm_us, "matmat_tf32_tflops": abi.HBX_NRHS * Em.info["alg_flops"] / (mm_us * 1e-6) / 1e12,
        "matmat_per_rhs_gbs": abi.HBX_NRHS * E.info["alg_bytes"] / 2 / (mm_us * 1e-6) / 1e9,
    }
    Em.close()
    # uneven batch: a 64-instance sample of C5 (the config's 256 need a minute of
    # host construction), solved in one block-diagonal engine and one by one
    from hacapk_b200 import configs
    t0 = time.time()
    inst = configs.c5(count=args.c5_count)
    t_build = time.time() - t0
    Eb = Engine.batch([Hk for Hk, _ in inst])
    bb = torch.from_numpy(np.concatenate([bk for _, bk in inst])).to(dev)
    ub = torch.zeros_like(bb)
    best, infos = 1e9, None
    for _ in range(reps + 1):
        ub.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        infos = Eb.bicgstab_batch_dev(bb.data_ptr(), ub.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
        torch.cuda.synchronize(dev)
        best = min(best, time.perf_counter() - t0)
    stream_gb = Eb.info["stream_bytes"] / 1e9
    Eb.close()
    one = 0.0
    for Hk, bk in inst:
        Ek = Engine(Hk.st, Hk.nd)
        bd = torch.from_numpy(bk).to(dev)
        ud = torch.zeros_like(bd)
        tk = 1e9
        for _ in range(2):
            ud.zero_()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            Ek.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter, stream=s)
            torch.cuda.synchronize(dev)
            tk = min(tk, time.perf_counter() - t0)
        one += tk
        Ek.close()
    its = [i["iterations"] for i in infos]
    out["batch_c5"] = {
        "instances": len(inst), "n_total": int(sum(Hk.nd for Hk, _ in inst)), "stream_gb": stream_gb,
        "solve_s": best, "one_by_one_s": one, "speedup": one / best,
        "iterations": [min(its), max(its)], "worst_true_relres": max(i["true_relres"] for i in infos),
        "converged": sum(i["status"] == 0 for i in infos), "host_build_s": t_build,
    }
    return out


def precision_workload(args):
    """The precision form on its own workload (C2 at --precision-level: the
    sphere and the seeded ellipsoid, ACA+ 1e-6), one JSON line: the FP64
    solve, FP32 factors in FP64 refinement and, when HBX_EXPERIMENTAL_BF16=1,
    BF16 factors in FP64 refinement (inner tolerance 1e-2); for each, the
    standalone product's time and stream rate and the solve's time, step
    counts and FP64 residual.  Solves are timed by the host clock around
    each call, best of three after one untimed run."""
    import torch
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    t0 = time.time()
    H, b = configs.c2(args.precision_level)
    t_build = time.time() - t0
    n = H.nd
    bd = torch.from_numpy(b).to(dev)
    ud = torch.zeros(n, dtype=torch.float64, device=dev)
    peak, peak_kind = peaks()

    def best_of(fn):
        best, res = 1e9, None
        for _ in range(4):
            ud.zero_()
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            res = fn()
            torch.cuda.synchronize(dev)
            best = min(best, time.perf_counter() - t)
        return best, res

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
    t64, inf = best_of(lambda: E.bicgstab_dev(bd.data_ptr(), ud.data_ptr(), tol=args.tol, max_iter=args.max_iter,
                                              stream=s))
    out = {"workload": f"C2: icosphere L{args.precision_level} + seeded ellipsoid, ACA+ 1e-6", "n": n,
           "host_build_s": t_build,
           "fp64": {"solve_s": t64, "iterations": inf["iterations"], "true_relres": inf["true_relres"],
                    "product": product(E)}}
    forms = [("fp32_refined", abi.HBX_FP32, 0.0)]
    if os.environ.get("HBX_EXPERIMENTAL_BF16") == "1":
        forms.append(("bf16_refined", abi.HBX_BF16, 1e-2))
    for name, prec, inner in forms:
        El = Engine(H.st, n, precision=prec)
        tl, inf = best_of(lambda: E.bicgstab_refined_dev(El, bd.data_ptr(), ud.data_ptr(), tol=args.tol,
                                                         max_iter=args.max_iter, inner_tol=inner, stream=s))
        out[name] = {"solve_s": tl, "speedup_vs_fp64": t64 / tl, "outer": inf["outer"],
                     "inner_iterations": inf["iterations"], "true_relres": inf["true_relres"],
                     "product": product(El)}
        El.close()
    E.close()
    print(json.dumps(out), flush=True)


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
    ap.add_argument("--no-forms", action="store_true", help="skip the FP32-refined, 64-RHS and batch forms")
    ap.add_argument("--c5-count", type=int, default=64, help="instances of the uneven-batch sample (C5: 256)")
    ap.add_argument("--profile-matmat", action="store_true",
                    help="only run five 64-RHS tensor-core products (a short command for ncu)")
    ap.add_argument("--precision-level", type=int, default=0,
                    help="only time the precision form on C2 at this level (7: the config; one GPU)")
    args = ap.parse_args()
    if args.profile_matmat:
        profile_matmat(args)
        return
    if args.precision_level > 0:
        precision_workload(args)
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

#!/usr/bin/env python
"""Benchmark of the B200 fermion hot path.

Metric: solves per second of the Wilson system D x = b to a true relative
residual of 1e-10 (mixed precision: FP16 inner Krylov iterations inside FP64
defect correction, even-odd, right-hand sides batched), with the Dslash HBM
bandwidth of the dominant kernel as the roofline.

Default workload ``wilson_eo_batched_32x32x32x32`` (the batched multi-RHS
configuration): 32^3 x 32 lattice, links exp(i eps H) with a seeded
traceless-Hermitian Gaussian H and eps = 0.25, kappa = 0.1355, fermion boundary
(+,+,+,-), 12 spin-colour point sources + 16 Z2 noise sources per rank, solved
in one batched call (synthetic data).  A step is one batched solve of all 28
right-hand sides.  ``wilson_eo_32x32x32x16`` (one complex Gaussian source on
32^3 x 16) is measured beside it.  With N GPUs every rank solves its own batch
(independent replicas, weak scaling; the path has no exchange step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Dslash HBM GB/s; solves/s to 1e-10 rel. resid, mixed+batched vs FP64 (1 B200)"
UNIT = "solves/s"
WORKLOADS = {
    "wilson_eo_32x32x32x16": dict(dims=(32, 32, 32, 16), kappa=0.1355, eps=0.25, seed=0xC1A60001, nrhs=1),
    "wilson_eo_16x16x16x8": dict(dims=(16, 16, 16, 8), kappa=0.1355, eps=0.25, seed=0xC1A60001, nrhs=1),
    # 12 spin-colour point sources + 16 Z2 noise sources in one batched solve
    "wilson_eo_batched_32x32x32x32": dict(dims=(32, 32, 32, 32), kappa=0.1355, eps=0.25, seed=0xC1A60003, nrhs=28,
                                          sources="point12_z2_16"),
}
DEFAULT_WORKLOAD = "wilson_eo_batched_32x32x32x32"
TOL = 1e-10
SOLVER_NAMES = {"cg": "CGNE on the Schur system (CG on M_ee M_ee^+)", "gmres": "GMRES(12)"}


def make_solver(clg, ctx, kind, inner):
    if kind == "cg":
        return clg.CSLASolverCG(ctx, inner_precision=inner, tol_true_rel=TOL)
    return clg.CSLASolverGMRES(ctx, inner_precision=inner, tol_true_rel=TOL, MaxDim=12)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    """nvidia-smi sampled every 200 ms by a background process; started before
    the warm-up (its start-up stalls the driver briefly) and filtered to the
    samples that arrive inside the timed window."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.window = (0.0, 0.0)

    def start(self):
        import threading

        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.lines.append((time.monotonic(), line))

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def mark(self, begin: bool):
        t = time.monotonic()
        self.window = (t, self.window[1]) if begin else (self.window[0], t)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        t0, t1 = self.window
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, line in self.lines:
            if not (t0 <= ts <= t1 + 0.25):
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if args.impl != "reference":
            torch.cuda.set_device(local)
        backend = "nccl" if args.impl != "reference" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ our arm
def hop_bytes_per_site(prec: int) -> int:
    """Compulsory HBM bytes of one checkerboard hop per output site: one input
    spinor, one output spinor and eight links (12-real for FP32/FP16)."""
    if prec == 0:
        return (24 + 24 + 8 * 18) * 8
    if prec == 1:
        return (24 + 24 + 8 * 12) * 4
    return (48 + 4) * 2 + 8 * 12 * 2


def hop_bytes_launch(prec: int, nrhs: int) -> int:
    """Compulsory HBM bytes of one hop launch over nrhs right-hand sides, per
    output site: each right-hand side's input and output spinor, the eight
    links once (all right-hand sides of the launch use the same links)."""
    links = 8 * 12 * (2 if prec == 2 else 4) if prec else 8 * 18 * 8
    return (hop_bytes_per_site(prec) - links) * nrhs + links


def cg_iteration(clg, ctx, stream, lat, U, kappa, b, inner, peak, n1=8, n2=24):
    """The inner CG iteration of the batched solve timed live through the public
    solver: the same FP16-inner CGNE solve of the batch b, cut off after n1 and
    after n2 CG iterations (one defect-correction cycle; n2 below the ~24
    iterations after which the first FP16 inner solves reach their 2e-3 floor),
    so (t2 - t1) / (n2 - n1) is one iteration of the solve's own
    kernels without its setup and FP64 residuals.  An iteration is the two odd
    hops, the D^+ hop with its (p, A p) epilogue, the D hop with the x / r update
    epilogue and p = r + beta p; its algorithmic bytes per output site and rhs
    (FP16 spinor 52 B, the links once per hop launch): odd hops 2 x 104, alpha
    hop 156, update hop 364 (the xpay source, x, r, p read, x, r written; A p is
    never stored), p = r + beta p 156."""
    import torch

    nrhs, Vh = b.nrhs, lat.volume // 2
    x = clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=nrhs)
    res = {}
    for n in (n1, n2):
        S = clg.CSLASolverCG(ctx, inner_precision=inner, tol_true_rel=1e-30, inner_tol=1e-30, max_outer=1,
                             max_iterations=2 * n)
        S.Solve(x, b, U, clg.EFO_F_D, raise_on_fail=False)  # graphs captured, launches tuned
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        infos = S.Solve(x, b, U, clg.EFO_F_D, raise_on_fail=False)
        e1.record(stream)
        torch.cuda.synchronize()
        res[n] = (e0.elapsed_time(e1) / 1e3, min(i["iterations"] for i in infos) / 2,
                  max(i["iterations"] for i in infos) / 2)
        S.close()
    x.close()
    (t1, lo1, hi1), (t2, lo2, hi2) = res[n1], res[n2]
    if lo1 != hi1 or lo2 != hi2 or lo2 <= lo1:
        return {"unmeasured": f"iteration counts {lo1}-{hi1} / {lo2}-{hi2} (expected {n1} / {n2} for every rhs)"}
    t_it = (t2 - t1) / (lo2 - lo1)
    links = 8 * 12 * 2
    per_site = 2 * 104 * nrhs + 156 * nrhs + 364 * nrhs + 156 * nrhs + 4 * links
    alg = per_site * Vh
    return {"us_per_iteration": round(t_it * 1e6, 1), "iterations_timed": int(lo2 - lo1),
            "bytes_per_iteration": alg, "achieved_GB/s": round(alg / t_it / 1e9, 1),
            "frac": round(alg / t_it / 1e9 / peak, 4),
            "kernels": "2 odd FP16 tile hops, D^+ hop + (p, A p), D hop + x / r update, p = r + beta p",
            "method": f"(t({n2} iterations) - t({n1} iterations)) / {n2 - n1}, CUDA events on the solver stream"}


def time_hops(clg, ctx, lat, U, prec, stream, reps=60, nrhs=1):
    """Average device duration of the checkerboard Wilson hop (odd -> even).

    The launches cycle over four input/output pairs so that the working set
    (links plus eight spinor half-fields) exceeds the 126 MB L2.  They are
    captured once into a CUDA graph and the graph is replayed between two
    events, so the figure is the kernels' own duration back to back, without
    the host-side cost of one ctypes call per launch."""
    import torch

    kappa = 0.1355
    fields = []
    npairs = 4 if nrhs == 1 else 2  # a batch of right-hand sides alone exceeds L2
    for i in range(npairs):
        a = clg.CFieldFermionWilsonSquareSU3(lat, kappa, precision=prec, nrhs=nrhs)
        for r in range(nrhs):
            a.InitialField(clg.SOURCE_GAUSS, 1234 + i, 2 + r, rhs=r)
        b = clg.CFieldFermionWilsonSquareSU3(lat, kappa, precision=prec, nrhs=nrhs)
        fields.append((a, b))
    for a, b in fields:  # warm-up (also runs the block-size autotuner)
        a.apply_to(clg.OP_DEO, b, U)
    torch.cuda.synchronize()
    k0 = ctx.kernel_count()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        for r in range(reps):
            a, b = fields[r % npairs]
            a.apply_to(clg.OP_DEO, b, U)
    per_replay = ctx.kernel_count() - k0
    replays = 3
    with torch.cuda.stream(stream):
        graph.replay()  # warm replay
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(replays):
            graph.replay()
        e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / (reps * replays)
    launches = per_replay * (replays + 1)
    del graph
    for a, b in fields:
        a.close()
        b.close()
    return t, launches


def hop_form_id(ctx, prec, Vh, nrhs):
    """Short name of the autotuner's Wilson hop form for D_eo at this size."""
    key = f"wilson_p{prec}_d0_V{Vh}_n{nrhs}_r{12 if prec == 1 else 0}"
    tuned = ctx.tuned()
    bs, v = tuned.get(key + "_auto", tuned.get(key, (0, 0)))
    if v >= 24:
        return "mma"
    if v >= 16:
        return "tile_blocked" if v & 2 else "tile_site"
    return "pair" if v >= 8 else "one"


def hop_form(ctx, prec, Vh, nrhs):
    """The Wilson hop kernel the autotuner chose for D_eo at this size."""
    key = f"wilson_p{prec}_d0_V{Vh}_n{nrhs}_r{12 if prec == 1 else 0}"
    tuned = ctx.tuned()
    pname = {0: "P64", 1: "P32", 2: "P16"}[prec]
    if key + "_auto" in tuned:
        bs, v = tuned[key + "_auto"]
        if v >= 24:
            return f"wilson_hop_mma16_kernel (tensor-core colour products; variant {v - 24})"
        if v >= 16:
            cap = {0: "uncapped", 1: "80-register cap", 4: "72-register cap", 5: "64-register cap"}[(v - 16) & 5]
            return (f"wilson_hop_tile16_kernel (32 sites x {nrhs} rhs per block, links staged once in shared memory; "
                    f"{bs // 32} warps, {cap}, {'blocked' if v & 2 else 'site'} tile order)")
        if v >= 8:
            return f"wilson_hop_pair_kernel (2 rhs per thread; block {bs}, variant {v - 8})"
        return f"wilson_hop_kernel<P16,12-real> (1 rhs per thread; block {bs}, variant {v})"
    bs, v = tuned.get(key, (None, None))
    return f"wilson_hop_kernel<{pname},12-real> (block {bs}, variant {v})"


def ours(args, world, rank, local):
    import torch

    import cudalatticegauge_b200 as clg

    W = WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    ctx = clg.Context(local, stream.cuda_stream)
    lat = clg.Lattice(ctx, W["dims"])
    V = lat.volume
    Vh = V // 2
    kappa = W["kappa"]
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, W["seed"], 1, W["eps"])
    nrhs = W["nrhs"]
    b = clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=nrhs)
    seed = W["seed"] + 7919 * rank
    if W.get("sources") == "point12_z2_16":
        # the 12 spin-colour point sources of a meson propagator at the origin
        # (CMeasureMesonCorrelator.cu:320-340) followed by Z2 noise sources
        for r in range(12):
            b.InitialAsSource(0, r, rhs=r)
        for r in range(12, nrhs):
            b.InitialField(clg.SOURCE_Z2, seed, 2 + r, rhs=r)
    else:
        for r in range(nrhs):
            b.InitialField(clg.SOURCE_GAUSS, seed, 2 + r, rhs=r)
    x = clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=nrhs)
    inner = {"single": clg.SINGLE, "half": clg.HALF}[args.inner]
    mixed = make_solver(clg, ctx, args.solver, inner)

    def check(infos):
        for i in infos:
            if i["status"] != 0 or i["true_rel_residual"] > TOL:
                raise RuntimeError(f"solve failed: {i}")
        return infos

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        check(mixed.Solve(x, b, U, clg.EFO_F_D))

    # ---------------- timed region: K solves, inputs resident in HBM
    barrier(world)
    torch.cuda.synchronize()
    k0 = ctx.kernel_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark(True)
    e0.record(stream)
    infos = []
    for _ in range(args.steps):
        infos = check(mixed.Solve(x, b, U, clg.EFO_F_D))
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark(False)
    clk = clocks.stop()
    launches = ctx.kernel_count() - k0
    t_local = e0.elapsed_time(e1) / 1e3
    barrier(world)
    t = max_over_ranks(t_local, world)
    value = args.steps * nrhs * world / t

    # ---------------- end to end through the public API with host buffers
    # Every step copies its source in from pinned host memory and its solution
    # out to pinned host memory.  The copies run on the context's copy stream
    # (clg_field_import_async / export_async) and overlap the neighbouring
    # solves: source k+1 goes in and solution k-1 comes out while solve k runs
    # (two source and two solution fields alternate).
    src = torch.empty((nrhs, V, 4, 3), dtype=torch.complex128, pin_memory=True).numpy()
    dst = [torch.empty((nrhs, V, 4, 3), dtype=torch.complex128, pin_memory=True).numpy() for _ in range(2)]
    for r in range(nrhs):
        b.to_numpy(r, out=src[r])
    bh = [clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=nrhs) for _ in range(2)]
    xh = [clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=nrhs) for _ in range(2)]

    def pipeline(steps):
        for r in range(nrhs):
            bh[0].from_numpy_async(src[r], r)
        for k in range(steps):
            if k + 1 < steps:
                for r in range(nrhs):
                    bh[(k + 1) % 2].from_numpy_async(src[r], r)
            check(mixed.Solve(xh[k % 2], bh[k % 2], U, clg.EFO_F_D))
            for r in range(nrhs):
                xh[k % 2].to_numpy_async(dst[k % 2][r], r)
        for f in xh + bh:
            f.wait()

    pipeline(2)  # untimed: allocates the fields' transfer staging and events
    barrier(world)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    pipeline(args.steps)
    e3.record(stream)  # after the last copy to the host has landed
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e2.elapsed_time(e3) / 1e3, world)
    for r in range(nrhs):  # the copied-out solution is the resident solve's (catches a stale transfer)
        ref = x.to_numpy(r)
        if np.linalg.norm(dst[(args.steps - 1) % 2][r] - ref) > 1e-6 * np.linalg.norm(ref):
            raise RuntimeError("end-to-end solution differs from the resident solve")
    e2e = {"value": args.steps * nrhs * world / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": int(src.nbytes), "d2h_bytes_per_step": int(dst[0].nbytes),
           "transfers": "pinned host memory, copy stream overlapping the neighbouring solves"}
    for f in bh + xh:
        f.close()
    b1 = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b1.from_numpy(src[nrhs - 1])

    # ---------------- the headline solutions against the FP64 oracle: every
    # right-hand side's true residual |b - D x| / |b| recomputed on the host
    oracle_check = None
    if rank == 0 and not args.no_cpu:
        oracle_check = oracle_residuals(U, lat, kappa, b, x, nrhs)

    # ---------------- roofline of the dominant kernel (the checkerboard hop in
    # the inner precision, over all right-hand sides of a step)
    peak, peak_kind = peaks()
    pname = {"single": "fp32", "half": "fp16"}[args.inner]
    t_hop, hop_launches = time_hops(clg, ctx, lat, U, inner, stream, reps=60 if nrhs == 1 else 12, nrhs=nrhs)
    hop_alg = hop_bytes_launch(inner, nrhs) * Vh
    achieved = hop_alg / t_hop / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "hop_traffic.json")
    if os.path.exists(tp):
        d = json.load(open(tp))
        form = hop_form_id(ctx, inner, Vh, nrhs)
        ent = d.get(pname + ("" if nrhs == 1 else f"_{nrhs}rhs" + ("" if form in ("one", "pair") else "_" + form)), {})
        if tuple(ent.get("dims", d.get("dims", ()))) == tuple(W["dims"]):
            traffic = ent.get("bytes_per_launch")
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "kernel": hop_form(ctx, inner, Vh, nrhs) + f", {nrhs} rhs per launch",
            "bytes_per_launch": hop_alg, "launch_us": round(t_hop * 1e6, 2), "peak_source": peak_kind,
            "bytes_model": ("one input and one output spinor per rhs and output site, the 8 links once per site "
                            "for all rhs of the launch")}
    if nrhs > 1:
        # the same launch counted as nrhs separate one-rhs hops (links re-read per rhs)
        roof["frac_links_per_rhs"] = round(hop_bytes_per_site(inner) * nrhs * Vh / t_hop / 1e9 / peak, 4)
    if inner == clg.HALF:
        # the FP16 hop's other bound: its real multiply-adds on the CUDA cores'
        # FMA pipe (HFMA2 / FFMA2 occupy it twice as long as FFMA, so each real
        # operation costs one lane-cycle whatever the precision): per output
        # site and rhs 576 (colour products) + 96 (spin projections) + 192
        # (FP32 accumulation) = 864; peak 128 lanes x SMs x SM clock
        ops = 864 * nrhs * Vh
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        fma = {"lane_ops_per_launch": ops, "achieved_Tops": round(ops / t_hop / 1e12, 2)}
        ck = clk if isinstance(clk, dict) else {}
        for key, mhz in (("frac_at_sm_max_clock", ck.get("sm_max_mhz")), ("frac_at_median_clock", ck.get("sm_mhz"))):
            if mhz:
                fma[key] = round(ops / t_hop / (128 * sms * mhz * 1e6), 4)
        roof["fma_pipe"] = fma

    extra = {}
    if rank == 0 and not args.quick and nrhs > 1:
        extra["cg_iteration_32x32x32x32"] = cg_iteration(clg, ctx, stream, lat, U, kappa, b, inner, peak)
        extra["denominators_32x32x32x32"] = denominators(clg, ctx, stream, lat, U, kappa, W, value)
        extra["single_source_32x32x32x16"] = single_source_side(clg, ctx, stream, args)
        if not args.no_batched:
            extra["batched_uneven_lattices"] = uneven_lattices(clg, ctx, stream, args)
        if not args.no_side:
            extra["wilson_8x8x8x8"] = wilson_small(clg, ctx, stream)
            extra["dslash_48x48x48x24"] = dslash_large(clg, ctx, stream)
            extra["staggered_32x32x32x16"] = staggered_hops(clg, ctx, stream)
            extra["staggered_multishift_32x32x32x16"] = staggered_multishift(clg, ctx, stream)
            extra["wilson_force_32x32x32x16"] = wilson_force_side(clg, ctx, stream)
            extra["staggered_force_32x32x32x16"] = ks_force_side(clg, ctx, stream)
        extra["reference_cuda_build"] = reference_cuda_build()
        if world == 1 and not args.no_cpu:
            extra["cpu_baseline"] = cpu_baseline_bicgstab(
                U, lat, kappa, extra["denominators_32x32x32x32"]["fp64_bicgstab"]["applications"])
    elif rank == 0 and not args.quick:
        # Dslash bandwidth in each precision, FP64 plain solves, CPU baseline
        dsl = {}
        for name, prec in (("fp64", clg.DOUBLE), ("fp32", clg.SINGLE), ("fp16", clg.HALF)):
            th, _ = time_hops(clg, ctx, lat, U, prec, stream, reps=40)
            dsl[name] = {"GB/s": round(hop_bytes_per_site(prec) * Vh / th / 1e9, 1),
                         "GFLOP/s": round(1320 * Vh / th / 1e9, 1), "launch_us": round(th * 1e6, 2)}
        extra["dslash_hop"] = dsl
        plain = {}
        for label, cls, prec in (("fp64_gmres12", clg.CSLASolverGMRES, clg.DOUBLE),
                                 ("fp64_bicgstab", clg.CSLASolverBiCGStab, clg.DOUBLE),
                                 ("fp64_cgne", clg.CSLASolverCG, clg.DOUBLE),
                                 ("mixed_gmres12", clg.CSLASolverGMRES, clg.SINGLE),
                                 ("half_gmres12", clg.CSLASolverGMRES, clg.HALF),
                                 ("mixed_cgne", clg.CSLASolverCG, clg.SINGLE),
                                 ("half_cgne", clg.CSLASolverCG, clg.HALF)):
            s = cls(ctx, inner_precision=prec, tol_true_rel=TOL, MaxDim=12, max_iterations=60000, max_outer=20)
            xs = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
            inf = s.Solve(xs, b1, U, clg.EFO_F_D, raise_on_fail=False)[0]  # warm-up (tuning, graph capture)
            if inf["status"] == 0:  # time a second solve when the first converged
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                inf = s.Solve(xs, b1, U, clg.EFO_F_D, raise_on_fail=False)[0]
                dt = time.perf_counter() - t0
            else:
                dt = inf["seconds"]
            plain[label] = {"solves_per_s": round(1.0 / dt, 3), "seconds": round(dt, 4),
                            "applications": inf["iterations"], "outer": inf["outer"],
                            "true_rel_residual": inf["true_rel_residual"], "status": inf["status"]}
            s.close()
            xs.close()
        extra["solves"] = plain
        if args.workload == DEFAULT_WORKLOAD and not args.no_batched:
            extra["batched_28rhs_32x32x32x32"] = batched_sources(clg, ctx, stream, args)
            extra["batched_uneven_lattices"] = uneven_lattices(clg, ctx, stream, args)
        if args.workload == DEFAULT_WORKLOAD and not args.no_side:
            extra["wilson_8x8x8x8"] = wilson_small(clg, ctx, stream)
            extra["dslash_48x48x48x24"] = dslash_large(clg, ctx, stream)
            extra["staggered_multishift_32x32x32x16"] = staggered_multishift(clg, ctx, stream)
            extra["wilson_force_32x32x32x16"] = wilson_force_side(clg, ctx, stream)
            extra["staggered_force_32x32x32x16"] = ks_force_side(clg, ctx, stream)
        if world == 1 and not args.no_cpu:
            extra["cpu_baseline"] = cpu_baseline(U, lat, kappa, plain["fp64_gmres12"]["applications"])
    result = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("f32" if args.inner == "single" else "f16 storage / f32 arithmetic") + " inner, f64 outer (complex)",
        "data": "synthetic",
        "config": {"workload": args.workload, "dims": list(W["dims"]), "kappa": kappa, "links": f"exp(i eps H), eps={W['eps']}",
                   "source": ("12 spin-colour point sources + 16 Z2 noise sources" if W.get("sources") else
                              "complex Gaussian"),
                   "solver": f"{SOLVER_NAMES[args.solver]}, {'FP32' if args.inner == 'single' else 'FP16'} inner, "
                             "FP64 defect correction, even-odd, all rhs batched in one call",
                   "tol_true_rel": TOL, "rhs_per_gpu": nrhs, "parallelism": f"replicas x{world}",
                   "l2": "working set (links and spinors of the solve) larger than the 126 MB L2"},
        "e2e": e2e, "roofline": roof, "clocks": clk, "gpu_launches": launches,
        "iterations_per_solve": max(i["iterations"] for i in infos) if infos else None,
        "oracle_check": oracle_check,
        # the Wilson hop forms the autotuner chose for this lattice
        # ([block, variant]: variant 0-3 one rhs per thread, 8-9 two, 16-19 the
        # tile form, 24-27 the tensor-core form; see clg_context_tuned)
        "autotuner": {k: list(v) for k, v in ctx.tuned().items()
                      if k.startswith("wilson") and f"_V{Vh}_n{nrhs}_" in k},
    }
    result.update(extra)
    if "cpu_baseline" not in result:
        result["cpu_baseline"] = None
    if rank == 0:
        print(json.dumps(result))
    ctx.close()


def oracle_residuals(U, lat, kappa, b, x, nrhs):
    """|b - D x| / |b| of every right-hand side by the FP64 CPU oracle (the
    checker; nothing of it is timed)."""
    from oracle import oracle as O

    op = O.Operator("WILSON_D", lat.dims, U.CopyDataOut(), kappa)
    res = [op.true_residual(b.to_numpy(r), x.to_numpy(r)) for r in range(nrhs)]
    return {"max_true_rel_residual": max(res), "rhs_checked": nrhs,
            "checker": "FP64 CPU oracle D (the reference's Wilson kernel restated)"}


def timed_solve(S, x, b, U, op, stream):
    """One warm-up solve (tuning, workspace, graphs), then one timed on the device."""
    import torch

    S.Solve(x, b, U, op, raise_on_fail=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    infos = S.Solve(x, b, U, op, raise_on_fail=False)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3, infos


def denominators(clg, ctx, stream, lat, U, kappa, W, batched_value):
    """The plain FP64 solvers on one source of the batched 32^3x32 problem (the
    last Z2 noise source), to the same true residual 1e-10: CGNE on the Schur
    system, BiCGStab (standard omega), and the reference's GMRES(12) with an
    application budget (it stagnates on this operator: its final true residual
    is recorded).  Every solution is checked by the FP64 oracle."""
    from oracle import oracle as O

    n = W["nrhs"]
    b1 = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b1.InitialField(clg.SOURCE_Z2, W["seed"], 2 + n - 1)
    x1 = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    op = O.Operator("WILSON_D", lat.dims, U.CopyDataOut(), kappa)
    bh = b1.to_numpy()
    out = {"source": "Z2 noise (rhs 27 of the batch)"}
    for label, cls, kw in (("fp64_cgne", clg.CSLASolverCG, {}),
                           ("fp64_bicgstab", clg.CSLASolverBiCGStab, {"max_iterations": 60000}),
                           ("fp64_gmres12", clg.CSLASolverGMRES, {"MaxDim": 12, "max_iterations": 6000, "max_outer": 4})):
        S = cls(ctx, inner_precision=clg.DOUBLE, tol_true_rel=TOL, **kw)
        if label == "fp64_gmres12":  # one budget-limited solve (not repeated)
            import time as _t
            t0 = _t.perf_counter()
            inf = S.Solve(x1, b1, U, clg.EFO_F_D, raise_on_fail=False)[0]
            dt = _t.perf_counter() - t0
        else:
            dt, infs = timed_solve(S, x1, b1, U, clg.EFO_F_D, stream)
            inf = infs[0]
        r = op.true_residual(bh, x1.to_numpy())
        out[label] = {"solves_per_s": round(1.0 / dt, 4) if inf["status"] == 0 else 0.0, "seconds": round(dt, 4),
                      "applications": inf["iterations"], "status": inf["status"],
                      "oracle_true_rel_residual": r}
        S.close()
    out["ratio_batched_mixed_vs_fp64_cgne"] = round(batched_value / out["fp64_cgne"]["solves_per_s"], 2)
    if out["fp64_bicgstab"]["solves_per_s"] > 0:
        out["ratio_batched_mixed_vs_fp64_bicgstab"] = round(batched_value / out["fp64_bicgstab"]["solves_per_s"], 2)
    out["fp64_gmres12_note"] = ("budget of 6000 applications; status 4 = not converged (restarted GMRES stagnates "
                                "on this operator), its oracle true residual is the value reached")
    b1.close()
    x1.close()
    return out


def single_source_side(clg, ctx, stream, args, steps=5):
    """32^3x16 (exp(i 0.25 H) links, one complex Gaussian source): the
    single-source solve of the metric's FP16-inner CGNE, the other solvers and
    precisions, and the hop in each precision; every solution checked by the
    FP64 oracle."""
    import torch

    from oracle import oracle as O

    W = WORKLOADS["wilson_eo_32x32x32x16"]
    lat = clg.Lattice(ctx, W["dims"])
    Vh = lat.volume // 2
    kappa = W["kappa"]
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, W["seed"], 1, W["eps"])
    b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b.InitialField(clg.SOURCE_GAUSS, W["seed"], 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    op = O.Operator("WILSON_D", lat.dims, U.CopyDataOut(), kappa)
    bh = b.to_numpy()
    out = {"dims": list(W["dims"])}
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF, tol_true_rel=TOL)
    S.Solve(x, b, U, clg.EFO_F_D)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        inf = S.Solve(x, b, U, clg.EFO_F_D)[0]
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / steps
    out["half_cgne_headline"] = {"solves_per_s": round(1.0 / t, 3), "ms_per_solve": round(t * 1e3, 3),
                                 "applications": inf["iterations"], "outer": inf["outer"],
                                 "oracle_true_rel_residual": op.true_residual(bh, x.to_numpy())}
    S.close()
    dsl = {}
    peak, _ = peaks()
    for name, prec in (("fp64", clg.DOUBLE), ("fp32", clg.SINGLE), ("fp16", clg.HALF)):
        th, _ = time_hops(clg, ctx, lat, U, prec, stream, reps=40)
        gbs = hop_bytes_per_site(prec) * Vh / th / 1e9
        dsl[name] = {"GB/s": round(gbs, 1), "frac": round(gbs / peak, 4), "GFLOP/s": round(1320 * Vh / th / 1e9, 1),
                     "launch_us": round(th * 1e6, 2)}
    out["dslash_hop"] = dsl
    plain = {}
    for label, cls, prec in (("fp64_gmres12", clg.CSLASolverGMRES, clg.DOUBLE),
                             ("fp64_bicgstab", clg.CSLASolverBiCGStab, clg.DOUBLE),
                             ("fp64_cgne", clg.CSLASolverCG, clg.DOUBLE),
                             ("mixed_gmres12", clg.CSLASolverGMRES, clg.SINGLE),
                             ("half_gmres12", clg.CSLASolverGMRES, clg.HALF),
                             ("mixed_cgne", clg.CSLASolverCG, clg.SINGLE)):
        s = cls(ctx, inner_precision=prec, tol_true_rel=TOL, MaxDim=12, max_iterations=60000, max_outer=20)
        dt, infs = timed_solve(s, x, b, U, clg.EFO_F_D, stream)
        i0 = infs[0]
        plain[label] = {"solves_per_s": round(1.0 / dt, 3), "seconds": round(dt, 4), "applications": i0["iterations"],
                        "outer": i0["outer"], "status": i0["status"],
                        "oracle_true_rel_residual": op.true_residual(bh, x.to_numpy())}
        s.close()
    out["solves"] = plain
    b.close()
    x.close()
    U.close()
    return out


def staggered_hops(clg, ctx, stream, reps=40):
    """Staggered checkerboard hop on 32^3x16 (exp(i 0.25 H) links, seed
    0xC1A60004) in FP64 (18-real links), FP32 and FP16 (12-real links):
    compulsory bytes per output site (one input and one output colour vector,
    eight links), 570 flops per site."""
    import torch

    peak, _ = peaks()
    lat = clg.Lattice(ctx, (32, 32, 32, 16))
    Vh = lat.volume // 2
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60004, 1, 0.25)
    bytes_site = {clg.DOUBLE: (6 + 6 + 8 * 18) * 8, clg.SINGLE: (6 + 6 + 8 * 12) * 4, clg.HALF: 2 * (12 + 4) + 8 * 24}
    out = {"dims": [32, 32, 32, 16]}
    for name, prec in (("fp64", clg.DOUBLE), ("fp32", clg.SINGLE), ("fp16", clg.HALF)):
        fields = []
        for i in range(4):
            a = clg.CFieldFermionKSSU3(lat, 0.02, precision=prec)
            a.InitialField(clg.SOURCE_GAUSS, 77 + i, 2)
            c = clg.CFieldFermionKSSU3(lat, 0.02, precision=prec)
            fields.append((a, c))
        for a, c in fields:
            a.apply_to(clg.OP_DEO, c, U)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            for r in range(reps):
                a, c = fields[r % 4]
                a.apply_to(clg.OP_DEO, c, U)
        with torch.cuda.stream(stream):
            g.replay()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(3):
                g.replay()
            e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / (3 * reps)
        del g
        gbs = bytes_site[prec] * Vh / t / 1e9
        out[name] = {"GB/s": round(gbs, 1), "frac": round(gbs / peak, 4), "GFLOP/s": round(570 * Vh / t / 1e9, 1),
                     "launch_us": round(t * 1e6, 2), "bytes_per_site": bytes_site[prec]}
        for a, c in fields:
            a.close()
            c.close()
    U.close()
    return out


def reference_cuda_build():
    """The reference's own CUDA build (CLGLib FP64, sm_100a) timed on a B200 by
    tests/golden/make_ref_golden.py --timing; read from the committed record."""
    p = os.path.join(ROOT, "profiles", "reference_cuda_build_32x32x32x16.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    d["source"] = "recorded by tests/golden/make_ref_golden.py --timing on a B200 (not re-run by bench.py)"
    return d


def batched_sources(clg, ctx, stream, args, steps=2):
    """Measured beside the headline: 32^3x32, 12 spin-colour point
    sources + 16 Z2 noise sources solved in one batched call (CGNE in the
    `--inner` precision inside FP64 defect correction), against one FP64 CGNE
    solve of a single source."""
    import torch

    W = WORKLOADS["wilson_eo_batched_32x32x32x32"]
    lat = clg.Lattice(ctx, W["dims"])
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, W["seed"], 1, W["eps"])
    n = W["nrhs"]
    b = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"], nrhs=n)
    for r in range(12):
        b.InitialAsSource(0, r, rhs=r)
    for r in range(12, n):
        b.InitialField(clg.SOURCE_Z2, W["seed"], 2 + r, rhs=r)
    x = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"], nrhs=n)
    inner = {"single": clg.SINGLE, "half": clg.HALF}[args.inner]
    s = clg.CSLASolverCG(ctx, inner_precision=inner, tol_true_rel=TOL)
    s.Solve(x, b, U, clg.EFO_F_D)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        infos = s.Solve(x, b, U, clg.EFO_F_D)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / steps
    worst = max(i["true_rel_residual"] for i in infos)
    b1 = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"])
    b1.InitialField(clg.SOURCE_Z2, W["seed"], 2 + n - 1)
    x1 = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"])
    s64 = clg.CSLASolverCG(ctx, inner_precision=clg.DOUBLE, tol_true_rel=TOL)
    s64.Solve(x1, b1, U, clg.EFO_F_D)
    torch.cuda.synchronize()
    e0.record(stream)
    i64 = s64.Solve(x1, b1, U, clg.EFO_F_D)[0]
    e1.record(stream)
    torch.cuda.synchronize()
    t64 = e0.elapsed_time(e1) / 1e3
    label = {"single": "FP32", "half": "FP16"}[args.inner]
    out = {"dims": list(W["dims"]), "rhs": n, "solver": f"CGNE, {label} inner, FP64 defect correction, batched",
           "solves_per_s": round(n / t, 3), "ms_per_batch": round(t * 1e3, 2),
           "max_applications": max(i["iterations"] for i in infos), "worst_true_rel_residual": worst,
           "fp64_single_rhs_cgne_solves_per_s": round(1.0 / t64, 3), "fp64_single_rhs_applications": i64["iterations"],
           "ratio_batched_mixed_vs_fp64": round(n / t * t64, 2)}
    for f in (b, x, b1, x1):
        f.close()
    s.close()
    s64.close()
    U.close()
    return out


def wilson_small(clg, ctx, stream):
    """8^4, Haar links (seed 0xC1A60000), kappa 0.1355, one
    Gaussian source.  The full D and D^+ applied in FP64 (the whole problem
    sits in L2, so GB/s here is not a roofline claim) and D x = b solved to the
    true relative residual 1e-10 by GMRES(12), the reference's solver on this
    case, in FP64 and with FP32 / FP16 inner iterations."""
    import torch

    lat = clg.Lattice(ctx, (8, 8, 8, 8))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_HAAR, 0xC1A60000, 1)
    b = clg.CFieldFermionWilsonSquareSU3(lat, 0.1355)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60000, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, 0.1355)
    out = {"dims": [8, 8, 8, 8]}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, op in (("D", clg.EFO_F_D), ("Ddagger", clg.EFO_F_Ddagger)):
        for _ in range(3):
            b.apply_to(op, x, U)
        reps = 200
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            b.apply_to(op, x, U)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        out[name] = {"us": round(t * 1e6, 2), "GB/s": round(960 * lat.volume / t / 1e9, 1)}
    for name, prec in (("fp64_gmres12", clg.DOUBLE), ("mixed_gmres12", clg.SINGLE), ("half_gmres12", clg.HALF)):
        S = clg.CSLASolverGMRES(ctx, inner_precision=prec, tol_true_rel=TOL, MaxDim=12)
        S.Solve(x, b, U, clg.EFO_F_D)
        torch.cuda.synchronize()
        e0.record(stream)
        info = S.Solve(x, b, U, clg.EFO_F_D)[0]
        e1.record(stream)
        torch.cuda.synchronize()
        out[name] = {"solves_per_s": round(1e3 / e0.elapsed_time(e1), 2), "applications": info["iterations"],
                     "true_rel_residual": info["true_rel_residual"], "status": info["status"]}
        S.close()
    for f in (b, x):
        f.close()
    U.close()
    return out


def uneven_lattices(clg, ctx, stream, args, steps=2):
    """The uneven set 8^4, 12^4, 16^4, 16^3x32,
    24^3x16 (442,624 sites), 4 complex Gaussian sources each, every lattice with
    its own gauge field.  All 20 sources are one solve (clg_solve_lattices: CGNE
    in the `--inner` precision, FP64 defect correction; one kernel per step
    covers every lattice); beside it, the five lattices as five batched calls
    back to back.  Unit: one source solved to the true relative residual 1e-10,
    every solution checked by the FP64 oracle."""
    from oracle import oracle as O

    import torch

    dims_set = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (16, 16, 16, 32), (24, 24, 24, 16)]
    kappa, eps, seed, n = 0.1355, 0.25, 0xC1A60003, 4
    inner = {"single": clg.SINGLE, "half": clg.HALF}[args.inner]
    jobs = []
    for d in dims_set:
        lat = clg.Lattice(ctx, d)
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, seed, 1, eps)
        b = clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=n)
        for r in range(n):
            b.InitialField(clg.SOURCE_GAUSS, seed, 100 + r, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, kappa, nrhs=n)
        s = clg.CSLASolverCG(ctx, inner_precision=inner, tol_true_rel=TOL)
        s.Solve(x, b, U, clg.EFO_F_D)  # warm-up (tuning, workspace, graphs)
        jobs.append((lat, U, b, x, s))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    infos = []
    for _ in range(steps):
        infos = []
        for lat, U, b, x, s in jobs:
            infos += s.Solve(x, b, U, clg.EFO_F_D)
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / 1e3 / steps
    # all lattices in one solve
    S = clg.CSLASolverCG(ctx, inner_precision=inner, tol_true_rel=TOL)
    xs = [clg.CFieldFermionWilsonSquareSU3(j[0], kappa, nrhs=n) for j in jobs]
    S.SolveLattices(xs, [j[2] for j in jobs], [j[1] for j in jobs], clg.EFO_F_D)  # warm-up
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        binfo = S.SolveLattices(xs, [j[2] for j in jobs], [j[1] for j in jobs], clg.EFO_F_D)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / steps
    worst_oracle = 0.0
    for (lat, U, b, x, s), xb in zip(jobs, xs):
        op = O.Operator("WILSON_D", lat.dims, U.CopyDataOut(), kappa)
        for r in range(n):
            worst_oracle = max(worst_oracle, op.true_residual(b.to_numpy(r), xb.to_numpy(r)))
    out = {"lattices": [list(d) for d in dims_set], "sites": sum(int(np.prod(d)) for d in dims_set),
           "rhs_per_lattice": n, "solver": "one clg_solve_lattices call (all lattices in every launch)",
           "solves_per_s": round(len(binfo) / t, 3), "ms_per_set": round(t * 1e3, 2),
           "worst_true_rel_residual": max(i["true_rel_residual"] for i in binfo),
           "oracle_worst_true_rel_residual": worst_oracle,
           "max_applications": max(i["iterations"] for i in binfo),
           "five_calls": {"solves_per_s": round(len(infos) / t_seq, 3), "ms_per_set": round(t_seq * 1e3, 2),
                          "max_applications": max(i["iterations"] for i in infos)}}
    S.close()
    for xb in xs:
        xb.close()
    for lat, U, b, x, s in jobs:
        for f in (b, x):
            f.close()
        s.close()
        U.close()
    return out


def dslash_large(clg, ctx, stream):
    """Checkerboard Wilson hop on 48^3x24 (V = 2,654,208) in
    FP64 (18-real links), FP32 (12-real) and FP16 (12-real FP16 links, FP16
    spinors with a per-site FP32 norm); compulsory bytes per output site as in
    hop_bytes_per_site, against the measured copy peak."""
    peak, _ = peaks()
    lat = clg.Lattice(ctx, (48, 48, 48, 24))
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60002, 1, 0.25)
    Vh = lat.volume // 2
    out = {"dims": [48, 48, 48, 24]}
    for name, prec in (("fp64", clg.DOUBLE), ("fp32", clg.SINGLE), ("fp16", clg.HALF)):
        t, _ = time_hops(clg, ctx, lat, U, prec, stream, reps=24)
        gbs = hop_bytes_per_site(prec) * Vh / t / 1e9
        out[name] = {"GB/s": round(gbs, 1), "frac": round(gbs / peak, 4), "GFLOP/s": round(1320 * Vh / t / 1e9, 1),
                     "launch_us": round(t * 1e6, 2)}
    # the solve in each inner precision (CGNE, FP64 defect correction), with the
    # error of each solution against the FP64 oracle: the oracle's true residual
    # and the distance to the FP64 solution
    from oracle import oracle as O

    kappa = 0.1355
    b = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60002, 2)
    x = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    op = O.Operator("WILSON_D", lat.dims, U.CopyDataOut(), kappa)
    bh = b.to_numpy()
    sols = {}
    solves = {}
    for name, prec in (("fp64", clg.DOUBLE), ("fp32", clg.SINGLE), ("fp16", clg.HALF)):
        S = clg.CSLASolverCG(ctx, inner_precision=prec, tol_true_rel=TOL)
        dt, infs = timed_solve(S, x, b, U, clg.EFO_F_D, stream)
        sols[name] = x.to_numpy()
        solves[name] = {"solves_per_s": round(1.0 / dt, 3), "applications": infs[0]["iterations"],
                        "outer": infs[0]["outer"], "oracle_true_rel_residual": op.true_residual(bh, sols[name])}
        S.close()
    for name in ("fp32", "fp16"):
        solves[name]["rel_error_vs_fp64_solution"] = float(np.linalg.norm(sols[name] - sols["fp64"]) /
                                                           np.linalg.norm(sols["fp64"]))
    out["solves_cgne"] = solves
    b.close()
    x.close()
    U.close()
    return out


FORCE_BYTES_PER_SITE = (2 * 24 + 4 * 18 + 2 * 4 * 18) * 8  # X, Y; U; F read + written (FP64)


def wilson_force_side(clg, ctx, stream, dims=(32, 32, 32, 16), kappa=0.1355):
    """The HMC pseudofermion force (CalculateForceS) on the headline lattice.

    kernel: F += force(U, X, Y) alone, FP64, compulsory bytes per site
    FORCE_BYTES_PER_SITE (X, Y read once, four links read, four force links
    read and written) against the measured copy peak; the 1.1 GB working set
    is larger than L2.
    step: the whole force step -- D D^+ X = phi to 1e-10 (CG, FP16 inner),
    cache, Y = D^+ X, force -- from a zero start and from the cache of the
    previous step after a small change of the links (exp(i 0.01 H) U, as one
    molecular-dynamics step moves them)."""
    import torch

    peak, _ = peaks()
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_ZERO)
    X = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    Y = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    X.InitialField(clg.SOURCE_GAUSS, 0xC1A60040, 2)
    Y.InitialField(clg.SOURCE_GAUSS, 0xC1A60041, 2)
    out = {"dims": list(dims), "bytes_per_site": FORCE_BYTES_PER_SITE}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, X, U)
    reps = 20
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, X, U)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    gbs = FORCE_BYTES_PER_SITE * lat.volume / t / 1e9
    out["kernel"] = {"launch_us": round(t * 1e6, 2), "GB/s": round(gbs, 1), "frac": round(gbs / peak, 4)}

    phi = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    phi.InitialField(clg.SOURCE_GAUSS, 0xC1A60042, 2)
    cache = clg.CFieldFermionWilsonSquareSU3(lat, kappa)
    S = clg.CSLASolverCG(ctx, inner_precision=clg.HALF, tol_true_rel=TOL)
    cache.Zero()
    phi.CalculateForceS(U, F, S, cache)  # warm-up (workspace, autotuner)
    steps = {}
    for name, warm in (("cold_start", False), ("cached_start", True)):
        if warm:
            # cache = X of the current links; then move the links in place by a
            # small step, as one molecular-dynamics update does
            phi.CalculateForceS(U, F, S, cache)
            small = clg.CFieldGaugeSU3(lat)
            small.InitialField(clg.GAUGE_EXPH, 0xC1A60043, 1, 0.01)
            U.InitialWithByte(np.ascontiguousarray(small.CopyDataOut() @ U.CopyDataOut()))
            small.close()
        else:
            cache.Zero()
        torch.cuda.synchronize()
        e0.record(stream)
        info = phi.CalculateForceS(U, F, S, cache)[0]
        e1.record(stream)
        torch.cuda.synchronize()
        dt = e0.elapsed_time(e1) / 1e3
        steps[name] = {"force_steps_per_s": round(1.0 / dt, 3), "seconds": round(dt, 4),
                       "applications": info["iterations"], "outer": info["outer"],
                       "true_rel_residual": info["true_rel_residual"], "status": info["status"]}
    out["step"] = steps
    for f in (F, X, Y, phi, cache, U):
        f.close()
    S.close()
    return out


def ks_force_side(clg, ctx, stream, dims=(32, 32, 32, 16), mass=0.02, poles=12):
    """The staggered RHMC force (CalculateForceS of CFieldFermionKSSU3) with 12
    poles on the headline lattice.  kernel: F -= force of 12 (phi_i, phi_id)
    pairs alone, FP64, compulsory bytes per site 12 x 2 x 48 B + U 576 B + F
    read and written 1152 B; step: one multi-shift CG solve of (DD^+ + b_i)
    phi_i = phi (FP32 inner) to 1e-10 for every pole, the 12 D0 applications
    and the force, from a zero start."""
    import torch

    peak, _ = peaks()
    lat = clg.Lattice(ctx, dims)
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60001, 1, 0.25)
    F = clg.CFieldGaugeSU3(lat)
    F.InitialField(clg.GAUGE_ZERO)
    pi = [clg.CFieldFermionKSSU3(lat, mass) for _ in range(poles)]
    pd = [clg.CFieldFermionKSSU3(lat, mass) for _ in range(poles)]
    for k in range(poles):
        pi[k].InitialField(clg.SOURCE_GAUSS, 0xC1A60060, 2 + k)
        pd[k].InitialField(clg.SOURCE_GAUSS, 0xC1A60061, 2 + k)
    a = np.logspace(-3, 0.5, poles)
    b = np.logspace(-4, 1, poles)
    nbytes = poles * 2 * 48 + 4 * 144 + 2 * 4 * 144
    out = {"dims": list(dims), "poles": poles, "bytes_per_site": nbytes}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        clg.CFieldFermionKSSU3.DerivateD0(F, U, pi, pd, a)
    reps = 20
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        clg.CFieldFermionKSSU3.DerivateD0(F, U, pi, pd, a)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    gbs = nbytes * lat.volume / t / 1e9
    out["kernel"] = {"launch_us": round(t * 1e6, 2), "GB/s": round(gbs, 1), "frac": round(gbs / peak, 4)}
    for f in pi + pd:
        f.close()
    phi = clg.CFieldFermionKSSU3(lat, mass)
    phi.InitialField(clg.SOURCE_GAUSS, 0xC1A60062, 2)
    S = clg.CMultiShiftCG(ctx, inner_precision=clg.SINGLE, tol_true_rel=TOL)
    phi.CalculateForceS(U, F, S, a, b)  # warm-up (workspace, autotuner)
    torch.cuda.synchronize()
    e0.record(stream)
    infos = phi.CalculateForceS(U, F, S, a, b)
    e1.record(stream)
    torch.cuda.synchronize()
    dt = e0.elapsed_time(e1) / 1e3
    out["step"] = {"force_steps_per_s": round(1.0 / dt, 3), "seconds": round(dt, 4),
                   "applications": max(i["iterations"] for i in infos),
                   "worst_true_rel_residual": max(i["true_rel_residual"] for i in infos),
                   "status": max(i["status"] for i in infos)}
    S.close()
    for f in (phi, F, U):
        f.close()
    return out


def staggered_multishift(clg, ctx, stream, steps=2):
    """32^3x16 staggered fermions, 2am = 0.02 (the reference's
    `Mass` parameter is 2am), BC (+,+,+,-), 12 shifts sigma_k = 10^(-4 + 5k/11),
    complex Gaussian source on the even sites; multi-shift CG on (DD^+)_ee + sigma_k
    to the FP64 true residual 1e-10 for every shift: the shared iteration in FP64
    until |r| <= 1e-4 |b|, then in FP32, the shifted x_k, p_k in FP64 (any shift
    left above the tolerance is refined in FP64).  Unit: all 12 shifts solved.
    Baseline: the same multi-shift solve in FP64 throughout."""
    import torch

    lat = clg.Lattice(ctx, (32, 32, 32, 16))
    m = 0.02
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, 0xC1A60004, 1, 0.25)
    b = clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN)
    b.InitialField(clg.SOURCE_GAUSS, 0xC1A60004, 2)
    shifts = [10.0 ** (-4 + 5 * k / 11) for k in range(12)]
    xs = [clg.CFieldFermionKSSU3(lat, m, subset=clg.EVEN) for _ in shifts]
    res = {}
    for name, prec in (("mixed", clg.SINGLE), ("fp64", clg.DOUBLE)):
        S = clg.CMultiShiftCG(ctx, inner_precision=prec, tol_true_rel=TOL)
        S.Solve(xs, shifts, b, U, clg.OP_DDDAG_EE)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = steps if name == "mixed" else 1
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            infos = S.Solve(xs, shifts, b, U, clg.OP_DDDAG_EE)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        res[name] = {"units_per_s": round(1.0 / t, 3), "ms_per_unit": round(t * 1e3, 2),
                     "worst_true_rel_residual": max(i["true_rel_residual"] for i in infos),
                     "max_iterations": max(i["iterations"] for i in infos)}
        S.close()
    for f in xs + [b]:
        f.close()
    U.close()
    return {"dims": [32, 32, 32, 16], "mass_2am": m, "shifts": len(shifts),
            "solver": "multi-shift CG (Jegerlehner): FP64 until |r| <= 1e-4 |b|, then FP32; x_k, p_k FP64",
            **res,
            "ratio_mixed_vs_fp64": round(res["fp64"]["ms_per_unit"] / res["mixed"]["ms_per_unit"], 2)}


def cpu_baseline(U, lat, kappa, fp64_applications):
    """Oracle FP64 M_ee on the host cores; solves/s = 1 / (t_apply * A), A the FP64
    GMRES(12) applications this run's solve needed."""
    from oracle import oracle as O

    Uh = U.CopyDataOut()
    L = lat.dims
    V = lat.volume
    op = O.Operator("WILSON_MEE", L, Uh, kappa)
    psi = O.gauss(V, 12, 5, 2).reshape(V, 4, 3)
    psi[O.parity_mask(L) == 1] = 0
    op(psi)
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        op(psi)
    t_apply = (time.perf_counter() - t0) / reps
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": round(1.0 / (t_apply * max(fp64_applications, 1)), 6), "unit": UNIT, "cores": cores,
            "kind": "port",
            "sample": f"{reps} FP64 M_ee applications of the C/OpenMP oracle on {L} ({t_apply*1e3:.1f} ms each); "
                      f"solves/s = 1/(t_apply x {fp64_applications} applications of the FP64 GMRES(12) solve)"}


def bicgstab_iteration_time(L, kappa, seed, eps, iters):
    """Seconds per iteration of the oracle's FP64 BiCGStab (the reference's
    CSLASolverBiCGStab restated, with the residual-minimising omega) on the
    even-odd Wilson system M_ee of lattice L, timed over `iters` iterations on
    the host cores (OpenMP)."""
    from oracle import oracle as O

    V = int(np.prod(L))
    U = O.gauge_expH(L, seed, eps)
    b = O.gauss(V, 12, seed, 2).reshape(V, 4, 3)
    b[O.parity_mask(L) == 1] = 0
    op = O.Operator("WILSON_MEE", L, U, kappa)
    O.bicgstab(op, b, dev_step=1, max_step=1, restart=1, accuracy=0.0, std_omega=True)  # warm-up
    t0 = time.perf_counter()
    _, info = O.bicgstab(op, b, dev_step=iters, max_step=1, restart=1, accuracy=0.0, std_omega=True)
    return (time.perf_counter() - t0) / iters


def cpu_baseline_bicgstab(U, lat, kappa, fp64_applications, iters=3):
    """Oracle FP64 BiCGStab on the host cores for the batched 32^3x32 problem:
    solves/s = 1 / (t_iteration x iterations of this run's FP64 BiCGStab solve)."""
    W = WORKLOADS["wilson_eo_batched_32x32x32x32"]
    t_it = bicgstab_iteration_time(W["dims"], kappa, W["seed"], W["eps"], iters)
    n_it = max(fp64_applications // 2, 1)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": round(1.0 / (t_it * n_it), 8), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{iters} iterations of the oracle's FP64 even-odd BiCGStab on {tuple(W['dims'])} "
                      f"({t_it:.3f} s each, 2 M_ee applications per iteration); solves/s = 1/(t_iteration x "
                      f"{n_it} iterations of this run's FP64 BiCGStab solve)"}


# ------------------------------------------------------------------ reference arm
def reference(args, world, rank):
    """The reference algorithm on the host cores: the oracle's restatement of
    CSLASolverGMRES (MGS Arnoldi, Givens; CSolverGMRES.cpp:111-358) on the
    even-odd system in FP64.  Each step is one GMRES(12) restart cycle (a bounded
    sample); solves/s = 1 / (t_cycle * cycles per solve), the cycle count of a
    full solve of this workload recorded by oracle/measure_reference_cycles.py."""
    if rank != 0:
        return
    from oracle import oracle as O

    W = WORKLOADS[args.workload]
    L, kappa = W["dims"], W["kappa"]
    V = int(np.prod(L))
    cp = os.path.join(ROOT, "oracle", "reference_cycles.json")
    counts = json.load(open(cp)) if os.path.exists(cp) else {}
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if W["nrhs"] > 1:
        # batched 32^3x32: the reference's GMRES(12) stagnates on this operator
        # and its BiCGStab with the conjugated omega diverges, so the reference
        # algorithm timed is CSLASolverBiCGStab with the residual-minimising
        # omega (the oracle's std_omega), FP64, even-odd, one right-hand side at
        # a time as the reference solves sources; a step is one iteration
        apps = counts.get(args.workload, {}).get("bicgstab_applications")
        t_it = bicgstab_iteration_time(L, kappa, W["seed"], W["eps"], max(args.steps, 1))
        value = 1.0 / (t_it * apps / 2) if apps else None
        sample = (f"{args.steps} FP64 even-odd BiCGStab iterations of the C/OpenMP oracle on {tuple(L)} "
                  f"({t_it:.3f} s each); {apps} applications per solve (oracle/reference_cycles.json)")
        out = {"metric": METRIC, "value": round(value, 8) if value else None, "unit": UNIT, "impl": "reference",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64 (complex)", "data": "synthetic",
               "ms_per_step": round(t_it * 1e3, 3),
               "config": {"workload": args.workload, "dims": list(L), "kappa": kappa,
                          "links": f"exp(i eps H), eps={W['eps']}",
                          "solver": "BiCGStab even-odd FP64 (reference algorithm, residual-minimising omega, CPU), "
                                    "one source at a time"},
               "cpu_baseline": {"value": round(value, 8) if value else None, "unit": UNIT, "cores": cores,
                                "kind": "port", "sample": sample},
               "e2e": {"value": round(value, 8) if value else None, "unit": UNIT, "h2d_bytes_per_step": 0,
                       "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return
    U = O.gauge_expH(L, W["seed"], W["eps"])
    b = O.gauss(V, 12, W["seed"], 2).reshape(V, 4, 3)
    pm = O.parity_mask(L)
    be, bo = b.copy(), b.copy()
    be[pm == 1] = 0
    bo[pm == 0] = 0
    bt = be + kappa * O.wilson_hop(L, U, bo, 0)
    op = O.Operator("WILSON_MEE", L, U, kappa)
    x = None
    for _ in range(args.warmup):
        x, _ = O.gmres(op, bt, x0=x, maxdim=12, restart=1, accuracy=0.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        x, _ = O.gmres(op, bt, x0=x, maxdim=12, restart=1, accuracy=0.0)
    t_cycle = (time.perf_counter() - t0) / args.steps
    cycles = counts.get(args.workload, {}).get("cycles")
    if cycles:
        value = 1.0 / (t_cycle * cycles)
        how = f"{cycles} GMRES(12) cycles per solve (oracle/reference_cycles.json)"
    else:
        value = None
        how = "cycle count of a full solve not recorded"
    sample = (f"{args.steps} FP64 even-odd GMRES(12) restart cycles of the C/OpenMP oracle on {L} "
              f"({t_cycle:.3f} s each); {how}")
    out = {"metric": METRIC, "value": round(value, 6) if value else None, "unit": UNIT, "impl": "reference",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64 (complex)", "data": "synthetic",
           "ms_per_step": round(t_cycle * 1e3, 3),
           "config": {"workload": args.workload, "dims": list(L), "kappa": kappa, "links": f"exp(i eps H), eps={W['eps']}",
                      "solver": "GMRES(12) even-odd FP64 (reference algorithm, CPU)"},
           "cpu_baseline": {"value": round(value, 6) if value else None, "unit": UNIT, "cores": cores,
                            "kind": "port", "sample": sample},
           "e2e": {"value": round(value, 6) if value else None, "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def profile_driver(args):
    """A small, fixed launch sequence for ncu captures.  The first hop call
    runs the block-size autotuner (28 launches of the Wilson hop for FP32 and
    FP16: 4 block sizes + 3 register-capped ones, 4 launches each), so
    `-k regex:wilson -s 28` lands on the tuned kernel; under `CLG_AUTOTUNE=0`
    every launch uses the default configuration instead."""
    import cudalatticegauge_b200 as clg

    W = WORKLOADS[args.workload]
    ctx = clg.Context(0)
    lat = clg.Lattice(ctx, W["dims"])
    U = clg.CFieldGaugeSU3(lat)
    U.InitialField(clg.GAUGE_EXPH, W["seed"], 1, W["eps"])
    if args.profile.startswith("hop"):
        prec = {"hop-double": clg.DOUBLE, "hop-single": clg.SINGLE, "hop-half": clg.HALF}[args.profile]
        n = W["nrhs"]  # the workload's right-hand sides in every launch
        a = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"], precision=prec, nrhs=n)
        for r in range(n):
            a.InitialField(clg.SOURCE_GAUSS, 5, 2 + r, rhs=r)
        o = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"], precision=prec, nrhs=n)
        for _ in range(args.steps):
            a.apply_to(clg.OP_DEO, o, U)
    elif args.profile == "force":
        F = clg.CFieldGaugeSU3(lat)
        F.InitialField(clg.GAUGE_ZERO)
        X = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"])
        Y = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"])
        X.InitialField(clg.SOURCE_GAUSS, 5, 2)
        Y.InitialField(clg.SOURCE_GAUSS, 6, 2)
        for _ in range(args.steps):
            clg.CFieldFermionWilsonSquareSU3.DerivateDOperator(F, Y, X, U)
    elif args.profile == "ks-force":
        F = clg.CFieldGaugeSU3(lat)
        F.InitialField(clg.GAUGE_ZERO)
        pi = [clg.CFieldFermionKSSU3(lat, 0.02) for _ in range(12)]
        pd = [clg.CFieldFermionKSSU3(lat, 0.02) for _ in range(12)]
        for k in range(12):
            pi[k].InitialField(clg.SOURCE_GAUSS, 7, 2 + k)
            pd[k].InitialField(clg.SOURCE_GAUSS, 8, 2 + k)
        for _ in range(args.steps):
            clg.CFieldFermionKSSU3.DerivateD0(F, U, pi, pd, np.logspace(-3, 0.5, 12))
    elif args.profile.startswith("multishift"):
        # the 12-shift staggered solve of staggered_multishift (32^3x16)
        lat = clg.Lattice(ctx, (32, 32, 32, 16))
        U = clg.CFieldGaugeSU3(lat)
        U.InitialField(clg.GAUGE_EXPH, 0xC1A60004, 1, 0.25)
        b = clg.CFieldFermionKSSU3(lat, 0.02, subset=clg.EVEN)
        b.InitialField(clg.SOURCE_GAUSS, 0xC1A60004, 2)
        shifts = [10.0 ** (-4 + 5 * k / 11) for k in range(12)]
        xs = [clg.CFieldFermionKSSU3(lat, 0.02, subset=clg.EVEN) for _ in shifts]
        prec = clg.DOUBLE if args.profile == "multishift-double" else clg.SINGLE
        S = clg.CMultiShiftCG(ctx, inner_precision=prec, tol_true_rel=TOL)
        for _ in range(args.steps):
            infos = S.Solve(xs, shifts, b, U, clg.OP_DDDAG_EE)
            print(max(i["iterations"] for i in infos), max(i["true_rel_residual"] for i in infos), flush=True)
    else:
        b = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"], nrhs=W["nrhs"])
        for r in range(W["nrhs"]):
            b.InitialField(clg.SOURCE_GAUSS, W["seed"], 2 + r, rhs=r)
        x = clg.CFieldFermionWilsonSquareSU3(lat, W["kappa"], nrhs=W["nrhs"])
        inner = {"single": clg.SINGLE, "half": clg.HALF}[args.inner]
        s = make_solver(clg, ctx, args.solver, inner)
        for _ in range(args.steps):
            print(s.Solve(x, b, U, clg.EFO_F_D)[0], flush=True)
    ctx.synchronize()
    tf = os.environ.get("CLG_TUNE_FILE")
    if tf and not os.path.exists(tf):  # the autotuner's choices for a later (profiled) run of the same command
        with open(tf, "w") as f:
            for k, (bs, v) in ctx.tuned().items():
                f.write(f"{k}={bs | (v << 16)}\n")
    print("profile driver done, kernels", ctx.kernel_count())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--quick", action="store_true", help="skip the per-precision and FP64 side measurements")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--inner", default="half", choices=["single", "half"],
                    help="inner Krylov precision (half: FP16 storage with a per-site FP32 norm, FP32 arithmetic)")
    ap.add_argument("--solver", default="cg", choices=["gmres", "cg"], help="inner Krylov method")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched config-4 side measurements")
    ap.add_argument("--no-side", action="store_true",
                    help="skip the config-3 Dslash and config-5 staggered multi-shift side measurements")
    ap.add_argument("--profile", default=None, choices=["hop-double", "hop-single", "hop-half", "solve", "force", "ks-force",
                             "multishift", "multishift-double"],
                    help="profiling driver (no JSON line): `--steps` hop launches on the workload lattice, "
                         "or `--steps` solves without warm-up")
    args = ap.parse_args()
    if args.profile:
        profile_driver(args)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            reference(args, world, rank)
        else:
            ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()

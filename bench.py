"""Benchmark: FP64 upwind DG advection operator apply (GenDiL's matrix-free path) on B200.

Workload (one "step" = one operator apply over the whole mesh): 3D upwind DG advection, cell
term + interior faces + boundary faces with inflow value 0, 64^3 Cartesian hexahedra on the unit
cube, order p = 3 GLL basis (16,777,216 DoFs), 4-point Gauss-Legendre quadrature, velocity
beta(x) = (1 + 0.5 sin 2 pi y, 0.5 + 0.25 cos 2 pi z, 0.25); input u ~ U[-1,1] from
FillRandom(seed 1).  x and y are 134 MB each (> 126 MB L2), so no L2 flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  ``value`` = GDoF/s of the device-resident apply (all ranks);
``e2e`` = the same apply through the C ABI with the input copied from pinned host memory and
the result copied back inside the timed region; ``roofline`` = algorithmic bytes (read x +
write y, 16 B/DoF) per launch over the measured launch time, against the measured HBM copy
bandwidth; ``cpu_baseline`` = the GenDiL reference operator (compiled from its own headers,
OpenMP) timed on this host.  ``--impl reference`` times that reference alone.
For N > 1 each rank runs an independent replica (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_AXIS, ORDER, NQ = 64, 3, 4
METRIC = "GDoF/s per operator apply vs HBM roofline; mixed vs FP64 solve time @1e-10"
WORKLOAD = "fp64 upwind DG advection apply, 3D 64^3 hex, p=3 GLL, q=4 GL, sin/cos velocity, inflow 0"
WORKLOAD_6D = ("fp64 upwind DG advection apply, 6D phase space 8^6 hypercubes on [0,1]^3 x [-1,1]^3, p=2 GLL, "
               "q=3 GL, beta = (v, -x + 0.5), inflow 0")
FALLBACK_HBM_GBS = 6650.0
HOST_SLABS = 4  # slabs of z planes per host-vector apply (consecutive steps overlap, so few slabs suffice)
# DRAM bytes (read + write) of one launch measured by ncu (one-pass capture of the full workload),
# by (workload, kernel variant, elements per axis)
TRAFFIC_BYTES = {("3d", "stage1-tile", 64): 221.3e6, ("3d", "tma1-tile", 64): 223.3e6,
                 ("6d", "nd-grouped2", 8): 4.25e9}


def workload_config(world, n=N_AXIS):
    """The `config` of the default (3D advection) line, identical in both arms."""
    nd = n ** 3 * (ORDER + 1) ** 3
    return {"workload": WORKLOAD.replace("64^3", f"{n}^3"), "dofs": nd, "elements": n ** 3,
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": f"inputs larger than L2 (x, y {8 * nd / 1e6:.0f} MB each)"}


def case_dict(n=N_AXIS):
    return {"D": 3, "P": ORDER, "Q": NQ, "basis": 0, "sizes": [n] * 3, "h": [1.0 / n] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "beta_kind": 2, "g": 0.0}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


# FP64 work of the Kronecker-form apply: 9 n x n passes, each n FMA per DoF (n = 4), 2 flop per FMA
# (face terms, about 3 FMA per DoF more, not counted)
KRON_FLOP_PER_DOF = 9 * (ORDER + 1) * 2


def fp64_gemm_peak(torch, dev):
    """Measured FP64 dense throughput of this GPU: cuBLAS DGEMM 8192^3 through torch, best of 3
    (CUDA events).  The denominator of the FP64 roofline of the apply kernel."""
    n = 8192
    a = torch.rand(n, n, dtype=torch.float64, device=dev)
    b = torch.rand(n, n, dtype=torch.float64, device=dev)
    c = torch.empty_like(a)
    torch.matmul(a, b, out=c)
    best = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [v.strip() for v in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for name, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
            os.unlink(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline(x_np, seconds_target=12.0):
    """The GenDiL reference operator (oracle/_ref, OpenMP) on this host's cores."""
    from oracle.bindings import Reference, have_reference
    if not have_reference():
        return None
    ref = Reference()
    case = case_dict()
    t1 = ref.time_advection(case, x_np, 1)
    pairs = max(1, min(20, int(seconds_target / max(2 * t1, 1e-3))))
    t = ref.time_advection(case, x_np, pairs)
    ndofs = len(x_np)
    return {"value": ndofs / t / 1e9, "unit": "GDoF/s", "cores": ref.num_threads(), "kind": "reference",
            "sample": f"full 64^3 p=3 mesh, {2 * pairs} applies (op(x,y); op(y,x) pairs) after 2 warm-up applies, "
                      f"GenDiL AdvectionOperator WithBC, SerialKernelConfiguration + OpenMP, mean {t * 1e3:.1f} ms/apply"}


def cpu_baseline_6d(seconds_target=12.0, n=6):
    """The GenDiL reference operator (oracle/_ref, OpenMP) on this host's cores for the 6D phase-space
    operator, on a bounded sample: the same operator on an n^6 mesh (per-DoF work does not depend on
    the mesh size)."""
    import numpy as np
    from oracle.bindings import Reference, have_reference
    if not have_reference():
        return None
    ref = Reference()
    case = {"D": 6, "P": 2, "Q": 3, "basis": 0, "sizes": [n] * 6, "h": [1.0 / n] * 3 + [2.0 / n] * 3,
            "origin": [0.0] * 3 + [-1.0] * 3, "periodic": [0] * 6, "beta_kind": 3, "g": 0.0}
    x = np.random.default_rng(1).uniform(-1, 1, n ** 6 * 3 ** 6)
    t1 = ref.time_advection(case, x, 1)
    pairs = max(1, min(10, int(seconds_target / max(2 * t1, 1e-3))))
    t = ref.time_advection(case, x, pairs)
    return {"value": len(x) / t / 1e9, "unit": "GDoF/s", "cores": ref.num_threads(), "kind": "reference",
            "sample": f"the same 6D operator on a {n}^6 mesh ({len(x)} DoFs), {2 * pairs} applies after 2 warm-up "
                      f"applies, GenDiL AdvectionOperator WithBC, SerialKernelConfiguration + OpenMP, "
                      f"mean {t * 1e3:.1f} ms/apply"}


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle.bindings import Reference, have_reference
    if not have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libgendil_ref.so was not built"}))
        return 0
    # everything on this arm comes from the reference compiled from its own headers: the input is
    # its FillRandom(seed 1) (Algebra/vector.hpp:632), the operator its AdvectionOperator WithBC
    ref = Reference()
    case = case_dict()
    x = ref.fill_random((N_AXIS ** 3) * (ORDER + 1) ** 3, 1)
    ref.time_advection(case, x, max(1, args.warmup // 2))
    t = ref.time_advection(case, x, max(1, args.steps // 2))
    v = len(x) / t / 1e9
    line = {"metric": METRIC, "value": v, "unit": "GDoF/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (FillRandom seed 1)", "impl": "reference",
            "config": workload_config(world),
            "cpu_baseline": {"value": v, "unit": "GDoF/s", "cores": ref.num_threads(), "kind": "reference",
                             "sample": f"full 64^3 mesh, {2 * max(1, args.steps // 2)} applies "
                                       "(op(x,y); op(y,x) pairs), GenDiL AdvectionOperator WithBC, OpenMP"},
            "e2e": {"value": v, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def mass_c1(g, torch, dev, steps, warmup, hbm):
    """Configuration 1's apply: FP64 mass, 16^3 hexahedra, p = 3 GLL, q = 4 GL, sigma = 1, input
    FillRandom(seed 0).  A launch of its 262,144 DoFs lasts a few microseconds, so the applies
    are replayed from CUDA graphs (no host launch cost in the timing).  Its 2 MB vectors fit in
    L2, so two figures: back-to-back applies (L2-resident, the way a solver's iterations see them)
    and applies each after a 256 MB L2 flush (cold inputs: the HBM roofline applies to these),
    timed as graph(flush; apply) x K minus graph(flush) x K."""
    space = g.Space(3, [16] * 3, order=3)
    op = g.MassOperator(space, 4, 1.0)
    nd = space.num_dofs
    x = torch.from_numpy(g.fill_random(nd, 0)).to(dev)
    y = torch.empty_like(x)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device=dev)
    reps = max(steps, 50)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(warmup):
            op(x, y)  # the operator's launches, and torch's, before capture
            flush.fill_(1.0)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()

    def capture(body):
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr):
            for _ in range(reps):
                body()
        return gr

    def timed(gr):
        gr.replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        gr.replay()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    g_apply = capture(lambda: op(x, y))
    g_flush = capture(lambda: flush.fill_(1.0))

    def flush_apply():
        flush.fill_(1.0)
        op(x, y)

    g_both = capture(flush_apply)
    ms_warm = timed(g_apply) / reps
    ms_cold = max(timed(g_both) - timed(g_flush), 0.0) / reps
    del g_apply, g_flush, g_both, flush
    alg = 16.0 * nd
    out = {"workload": "fp64 mass apply, 3D 16^3 hex, p=3 GLL, q=4 GL, sigma=1 (FillRandom seed 0)", "dofs": nd,
           "kernel": op.kernel, "variant": op.variant,
           "l2_resident": {"ms_per_apply": ms_warm, "gdofs_per_s": nd / (ms_warm * 1e-3) / 1e9,
                           "gbs": alg / (ms_warm * 1e-3) / 1e9, "applies": reps,
                           "note": "back-to-back applies replayed from a CUDA graph; x and y (2 MB each) stay "
                                   "in L2, no HBM roofline"},
           "after_l2_flush": {"ms_per_apply": ms_cold, "gdofs_per_s": nd / (ms_cold * 1e-3) / 1e9,
                              "roofline": {"bound": "hbm", "achieved": alg / (ms_cold * 1e-3) / 1e9, "peak": hbm,
                                           "unit": "GB/s", "frac": alg / (ms_cold * 1e-3) / 1e9 / hbm},
                              "applies": reps,
                              "note": "graph(256 MB flush; apply) x K minus graph(flush) x K, per apply"}}
    op.close()
    return out


def mass_large(g, torch, dev, steps, warmup, hbm, n, space=None, q=4, label=None):
    """The FP64 mass apply (sigma = 1) on the bench's mesh (3D n^3 p = 3 GLL, q = 4 unless `space`,
    `q` and `label` name another): 16 B/DoF moved per apply with inputs larger than L2, the regime
    where the HBM roofline binds."""
    space = space or g.Space(3, [n] * 3, order=3)
    op = g.MassOperator(space, q, 1.0)
    nd = space.num_dofs
    x = torch.from_numpy(g.fill_random(nd, 0)).to(dev)
    y = torch.empty_like(x)
    for _ in range(warmup):
        op(x, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        op(x, y)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    alg = 16.0 * nd
    out = {"workload": label or f"fp64 mass apply, 3D {n}^3 hex, p=3 GLL, q=4 GL, sigma=1", "dofs": nd,
           "kernel": op.kernel,
           "variant": op.variant, "ms_per_apply": ms, "gdofs_per_s": nd / (ms * 1e-3) / 1e9,
           "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                        "frac": alg / (ms * 1e-3) / 1e9 / hbm},
           "l2": f"inputs larger than L2 (x, y {8 * nd / 1e6:.0f} MB each)"}
    op.close()
    return out


def solve_leg(g, C, space, dev, dt=1e-3, restart=30, tol=1e-10, q=None, beta=None, seed=2, max_iters=20000,
              plain=True, bf16=False):
    """Implicit-Euler system (M/dt + A) x = b, b = FillRandom(seed), GMRES(restart) to tol
    relative FP64 residual from x0 = 0, timed on the device (CUDA events around the whole solve):
    FP64 GMRES with the reference's modified Gram-Schmidt, then the refinement solver with FP64
    and with FP32 inner cycles (fused classical Gram-Schmidt, FP64 residual and update).  Each leg reports the
    residual it reached, recomputed here with the FP64 operator, and the mixed leg its max-norm
    distance to the FP64 solution."""
    import torch
    A = g.SystemOperator(space, q or NQ, beta or C.velocity_sincos(3), sigma=1.0 / dt, bc=g.BC_INFLOW, g=0.0)
    b = torch.from_numpy(g.fill_random(space.num_dofs, seed)).to(dev)
    bnorm = torch.linalg.vector_norm(b).item()
    out = {"system": f"M/dt + A, dt={dt}, GMRES({restart}), tol {tol}, at most {max_iters} iterations, x0 = 0, "
                     f"b = FillRandom(seed {seed})", "kernel": A.kernel}
    sols = {}
    P = g.MassInverseOperator(space, q or NQ, 1.0 / dt)  # element mass inverse (right preconditioner)
    legs = [("fp64_gmres", lambda: g.GMRESSolver(A, restart)),
            ("fp64_gmres_ir", lambda: g.GMRESIRSolver(A, restart, inner="fp64")),
            ("mixed_gmres_ir", lambda: g.GMRESIRSolver(A, restart, inner="fp32")),
            ("mixed_gmres_ir_one_graph", lambda: g.GMRESIRSolver(A, restart, inner="fp32").use_graphs("whole"))]
    if not plain:
        legs = []
    legs += [("fp64_gmres_massprec", lambda: g.GMRESSolver(A, restart).precondition(P)),
             ("mixed_gmres_ir_massprec", lambda: g.GMRESIRSolver(A, restart, inner="fp32").precondition(P)),
             # the same solve as ONE graph launch (conditional WHILE node over the restart cycles)
             ("mixed_gmres_ir_massprec_one_graph",
              lambda: g.GMRESIRSolver(A, restart, inner="fp32").precondition(P).use_graphs("whole"))]
    if bf16:
        # inner applies with BF16 tensor-core contractions (FP32 accumulation, per-element max-abs
        # scaling), FP32 basis, FP64 refinement
        legs.append(("bf16_gmres_ir_massprec", lambda: g.GMRESIRSolver(A, restart, inner="bf16").precondition(P)))
    for name, make in legs:
        solver = make()
        x = torch.zeros_like(b)
        solver.solve(b, x, 2, tol)  # warm-up (kernels, caches)
        x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        info = solver.solve(b, x, max_iters, tol)
        e1.record()
        torch.cuda.synchronize()
        ax = torch.empty_like(x)
        A(x, ax)
        true_rel = torch.linalg.vector_norm(b - ax).item() / bnorm
        out[name] = {"seconds": e0.elapsed_time(e1) * 1e-3, "iterations": info["iterations"],
                     "relative_residual": info["relative_error"], "true_relative_residual": true_rel,
                     "converged": info["success"]}
        sols[name] = x
        solver.close()
    ref = "fp64_gmres" if plain else "fp64_gmres_massprec"
    for name in sols:
        if name != ref:
            d = (sols[name] - sols[ref]).abs().max() / sols[ref].abs().max()
            out[name][f"rel_max_diff_vs_{ref}"] = d.item()
    if plain:
        out["fp64_over_mixed_time"] = out["fp64_gmres"]["seconds"] / out["mixed_gmres_ir"]["seconds"]
    out["fp64_over_mixed_time_massprec"] = (out["fp64_gmres_massprec"]["seconds"] /
                                            out["mixed_gmres_ir_massprec"]["seconds"])
    if "bf16_gmres_ir_massprec" in out:
        out["fp64_over_bf16_time_massprec"] = (out["fp64_gmres_massprec"]["seconds"] /
                                               out["bf16_gmres_ir_massprec"]["seconds"])
    A.close()
    P.close()
    return out


def run_ours(args):
    import numpy as np
    import torch
    import gendil_b200 as g
    from gendil_b200 import coefficients as C

    from gendil_b200.replicas import Replicas
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    reps = Replicas("nccl")  # independent replicas: only barriers and the max-over-ranks timing

    six = args.workload == "6d"
    if six:
        # configuration 3: 8^6 elements on [0,1]^3 x [-1,1]^3, p = 2, q = 3, beta = (v, -x + 0.5)
        n6 = args.size_6d
        space = g.Space(6, [n6] * 6, [1.0 / n6] * 3 + [2.0 / n6] * 3, [0.0] * 3 + [-1.0] * 3, None, 2)
        op = g.AdvectionOperator(space, 3, C.velocity_phase_space(6), bc=g.BC_INFLOW, g=0.0)
    else:
        space = g.Space(3, [args.size] * 3, order=ORDER)
        op = g.AdvectionOperator(space, NQ, C.velocity_sincos(3), bc=g.BC_INFLOW, g=0.0)
    if args.variant and op.kernel in ("kron", "kronnd"):
        op.set_variant(args.variant)  # a fixed kernel for profiling; the autotuner's pick otherwise
    nd = space.num_dofs
    x_np = g.fill_random(nd, 1)
    x = torch.from_numpy(x_np).to(dev)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    barrier = reps.barrier

    for _ in range(args.warmup):
        op(x, y)
    # the K timed applies are replayed from one CUDA graph captured after the warm-up: the same K
    # kernel launches as direct calls, without the host's per-call latency inside the timed region
    applies = torch.cuda.CUDAGraph()
    with torch.cuda.graph(applies):
        for _ in range(args.steps):
            op(x, y)
    torch.cuda.synchronize()
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        applies.replay()
        stop.record(stream)
        barrier()
    ms = reps.max(start.elapsed_time(stop))
    ms_step = ms / args.steps
    value = reps.throughput(nd * args.steps, ms) / 1e9

    # the speed-of-light operator (y = x element by element, MakeSpeedOfLightOperator) on the same
    # vectors: the in-framework bandwidth reference of an apply
    sol = g.SpeedOfLightOperator(space)
    for _ in range(args.warmup):
        sol(x, y)
    copies = torch.cuda.CUDAGraph()
    with torch.cuda.graph(copies):
        for _ in range(args.steps):
            sol(x, y)
    torch.cuda.synchronize()
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    copies.replay()
    s1.record(stream)
    barrier()
    del copies
    sol.close()
    ms_sol = reps.max(s0.elapsed_time(s1)) / args.steps

    # end to end through the C ABI on host vectors: every step uploads its input from pinned host
    # memory, applies and downloads its result (dgop_host_io_apply_async: upload / apply /
    # download pipelined over slabs of z planes, and one step's uploads overlapping the previous
    # step's downloads); the timed region ends when the last result is in host memory
    xh = torch.from_numpy(x_np).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    io = g.HostIO(op, slabs=HOST_SLABS)
    for _ in range(2):
        io.apply(xh, yh, stream)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_steps = max(3, min(args.steps, 20))
    e0.record(stream)
    for _ in range(e_steps):
        io.apply_async(xh, yh, stream)
    io.wait(stream)
    e1.record(stream)
    barrier()
    io.close()
    ems = reps.max(e0.elapsed_time(e1))
    e2e_value = reps.throughput(nd * e_steps, ems) / 1e9

    hbm, peak_kind = peaks()
    alg_bytes = 16.0 * nd
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    # dram__bytes_read.sum + dram__bytes_write.sum of one launch (ncu, summarized under profiles/)
    traffic = TRAFFIC_BYTES.get(("6d", op.variant, args.size_6d) if six else ("3d", op.variant, args.size))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (FillRandom seed 1)",
                "config": (workload_config(world, args.size) if not six else
                           {"workload": WORKLOAD_6D.replace("8^6", f"{n6}^6"), "dofs": nd,
                            "elements": space.num_elements,
                            "parallelism": f"replicas{world}" if world > 1 else "single",
                            "l2": f"inputs larger than L2 (x, y {8 * nd / 1e6:.0f} MB each)"}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                             "algorithmic_bytes_per_launch": alg_bytes},
                "e2e": {"value": e2e_value, "unit": "GDoF/s", "h2d_bytes_per_step": 8 * nd,
                        "d2h_bytes_per_step": 8 * nd, "steps": e_steps,
                        "path": f"dgop_host_io_apply_async + dgop_host_io_wait (pinned host vectors, {HOST_SLABS} slabs, "
                                "consecutive steps overlapped)"},
                "gpu_launches": args.steps,
                "timed_region": "the K applies replayed from one CUDA graph captured after the warm-up (one kernel "
                                "launch per apply), CUDA events on the launching stream",
                "clocks": clocks.summary(),
                "speed_of_light": {"ms_per_apply": ms_sol, "gdofs_per_s": nd / (ms_sol * 1e-3) / 1e9,
                                   "gbs": 16.0 * nd / (ms_sol * 1e-3) / 1e9,
                                   "frac_of_measured_hbm": 16.0 * nd / (ms_sol * 1e-3) / 1e9 / hbm,
                                   "apply_time_over_copy_time": ms_step / ms_sol,
                                   "note": "SpeedOfLightOperator (y = x, 16 B/DoF) on the same vectors, same steps"}}
        if op.kernel in ("kron", "kronnd"):
            # FP64 work: D^2 n x n passes (D terms x D axes), n FMA per DoF each, 2 flop per FMA
            D, n = space.dim, space.order + 1
            flop = D * D * n * 2
            peak64 = fp64_gemm_peak(torch, dev)
            a64 = flop * nd / (ms_step * 1e-3) / 1e12
            line["roofline_fp64"] = {"bound": "fp64", "achieved": a64, "peak": peak64, "unit": "TFLOP/s",
                                     "frac": a64 / peak64, "flop_per_dof": flop,
                                     "peak_kind": "measured: cuBLAS DGEMM 8192^3 (torch), best of 3"}
        line["kernel"] = {"family": op.kernel}
        if op.variant:
            line["kernel"]["variant"] = op.variant
            line["kernel"]["autotuner_ms_per_launch"] = {k: round(v, 4) for k, v in op.variant_times().items() if v}
            v32, ms32 = op.variant_f32()
            line["kernel"]["fp32_variant"] = v32
            line["kernel"]["fp32_autotuner_ms_per_launch"] = {k: round(v, 4) for k, v in ms32.items() if v > 0}
        if not six and world == 1:
            line["mass_c1"] = mass_c1(g, torch, dev, args.steps, args.warmup, hbm)
            line["mass_64cubed"] = mass_large(g, torch, dev, args.steps, args.warmup, hbm, args.size)
        if six and world == 1:
            line["mass_6d"] = mass_large(g, torch, dev, min(args.steps, 20), args.warmup, hbm, n6, space=space, q=3,
                                         label=f"fp64 mass apply, 6D {n6}^6 hypercubes, p=2 GLL, q=3 GL, sigma=1")
        if world == 1 and not args.no_solve:
            if six:
                # configuration 3: dt = 5e-3, inner GMRES(20), b from seed 3.  The unpreconditioned
                # system's tensor-product mass matrix is ill-conditioned in 6D (GMRES(20) stands at
                # a relative residual of 0.12 after 200 iterations), so the legs solve it with the
                # element mass inverse as right preconditioner (same 1e-10 on |b - A x| / |b|).
                line["solve"] = solve_leg(g, C, space, dev, dt=5e-3, restart=20, q=3,
                                          beta=C.velocity_phase_space(6), seed=3, max_iters=2000, plain=False,
                                          bf16=True)
            else:
                line["solve"] = solve_leg(g, C, space, dev)
        if six and world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline_6d()
            except Exception as exc:  # the baseline is reported, never required
                line["cpu_baseline"] = {"unavailable": str(exc)}
        if world == 1 and not args.no_cpu_baseline and args.size == N_AXIS and not six:
            try:
                line["cpu_baseline"] = cpu_baseline(x_np)
            except Exception as exc:  # the baseline is reported, never required
                line["cpu_baseline"] = {"unavailable": str(exc)}
        print(json.dumps(line))
    reps.close()
    return 0


def batch_instances(count, seed=7):
    """Configuration 5: `count` instances from one seeded generator.  Per instance: dimension
    uniform in {2, 3, 4}, order uniform in 1..5, element count log-uniform in [1e3, 1e5] turned
    into balanced Cartesian extents, constant velocity with components uniform in [-1, 1]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        D = int(rng.integers(2, 5))
        p = int(rng.integers(1, 6))
        E = float(np.exp(rng.uniform(np.log(1e3), np.log(1e5))))
        sizes = []
        rem = E
        for k in range(D):
            n = max(1, int(round(rem ** (1.0 / (D - k)))))
            sizes.append(n)
            rem /= n
        beta = list(rng.uniform(-1.0, 1.0, D))
        out.append({"D": D, "P": p, "sizes": sizes, "beta": beta, "seed": seed * 100000 + i})
    return out


def run_batch(args):
    """Configuration 5: independent implicit systems M/dt + A (dt = 1e-3, inflow 0), q = p + 2.
    (1) every operator applied once: one dgop_batch_apply (one persistent launch per (dimension,
    order) group) against one launch per instance; (2) every system solved to 1e-10 relative
    residual with the element mass inverse as right preconditioner: all systems together by the
    batched FP32-inner refinement GMRES(20) (dgop_batch_solver) against FP64 GMRES(20) one
    instance after the other."""
    import threading
    import numpy as np
    import torch
    import gendil_b200 as g
    from gendil_b200 import coefficients as C

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    inst = batch_instances(args.instances)
    ops, precs, bs = [], [], []
    t0 = time.time()
    for d in inst:
        sp = g.Space(d["D"], d["sizes"], [1.0 / n for n in d["sizes"]], [0.0] * d["D"], None, d["P"])
        q = d["P"] + 2
        ops.append(g.SystemOperator(sp, q, C.velocity_constant(d["beta"]), sigma=1e3, bc=g.BC_INFLOW, g=0.0))
        precs.append(g.MassInverseOperator(sp, q, 1e3))
        gen = torch.Generator(device=dev).manual_seed(d["seed"])
        bs.append(torch.rand(sp.num_dofs, dtype=torch.float64, device=dev, generator=gen) * 2.0 - 1.0)
    setup_s = time.time() - t0
    dofs = [o.space.num_dofs for o in ops]
    total = float(sum(dofs))
    ys = [torch.empty_like(b) for b in bs]

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    batch = g.Batch(ops)
    ms_batch = timed(lambda: batch.apply(bs, ys))
    ms_each = timed(lambda: [o(b, y) for o, b, y in zip(ops, bs, ys)])
    batch.close()

    def solve_all(kind, streams):
        """Every system solved by its own solver object, one after the other on `streams`
        concurrent streams (the one-launch-each baseline)."""
        times = [0.0] * len(ops)
        iters = [0] * len(ops)
        ok = [False] * len(ops)
        order = sorted(range(len(ops)), key=lambda i: -dofs[i])  # largest first
        lock = threading.Lock()
        errors = []

        def worker():
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                while True:
                    with lock:
                        if not order:
                            return
                        i = order.pop(0)
                    A, P, b = ops[i], precs[i], bs[i]
                    try:
                        s = (g.GMRESSolver(A, 20) if kind == "fp64" else
                             g.GMRESIRSolver(A, 20, inner="fp32")).precondition(P)
                        x = torch.zeros_like(b)
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(st)
                        info = s.solve(b, x, 2000, 1e-10, stream=st)
                        e1.record(st)
                        e1.synchronize()
                        times[i] = e0.elapsed_time(e1) * 1e-3
                        iters[i], ok[i] = info["iterations"], info["success"]
                        s.close()
                        del x
                    except Exception as exc:  # reported as an unconverged instance
                        with lock:
                            errors.append(f"instance {i}: {exc}")

        torch.cuda.synchronize()
        w0 = time.time()
        threads = [threading.Thread(target=worker) for _ in range(streams)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        torch.cuda.synchronize()
        wall = time.time() - w0
        ts = np.array(times)
        return {"wall_s": wall, "solved_gdofs_per_s": total / wall / 1e9, "converged": int(sum(ok)),
                "errors": errors[:3],
                "iterations_median": float(np.median(iters)), "iterations_max": int(max(iters)),
                "instance_s": {"p50": float(np.percentile(ts, 50)), "p90": float(np.percentile(ts, 90)),
                               "p99": float(np.percentile(ts, 99)), "max": float(ts.max())}}

    fp64 = solve_all("fp64", 1)

    # all systems together: lockstep refinement GMRES(20) with FP32 inner cycles (dgop_batch_solver)
    t0 = time.time()
    bsolver = g.BatchSolver(ops, precs, restart=20, inner="fp32")
    bsolver_setup_s = time.time() - t0
    xs = [torch.zeros_like(b) for b in bs]
    torch.cuda.synchronize()
    w0 = time.time()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    bres, bsecs = bsolver.solve(bs, xs, 2000, 1e-10)
    e1.record()
    torch.cuda.synchronize()
    bwall = time.time() - w0
    bdev = e0.elapsed_time(e1) * 1e-3
    worst = 0.0
    for A, b, x in zip(ops, bs, xs):
        ax = torch.empty_like(x)
        A(x, ax)
        worst = max(worst, (torch.linalg.vector_norm(b - ax) / torch.linalg.vector_norm(b)).item())
    ts = np.array(bsecs)
    its = [r["iterations"] for r in bres]
    batched = {"wall_s": bwall, "device_s": bdev, "solved_gdofs_per_s": total / bwall / 1e9,
               "converged": int(sum(r["success"] for r in bres)), "max_true_relative_residual": worst,
               "waves": bsolver.waves, "setup_s": bsolver_setup_s,
               "iterations_median": float(np.median(its)), "iterations_max": int(max(its)),
               "instance_completion_s": {"p50": float(np.percentile(ts, 50)), "p90": float(np.percentile(ts, 90)),
                                         "p99": float(np.percentile(ts, 99)), "max": float(ts.max())},
               "note": "every system advanced in lockstep: one launch per vector operation over all systems of a "
                       "wave, one apply per system, restart cycles replayed from one CUDA graph; completion "
                       "time = end of the restart cycle after which the system was found finished"}
    bsolver.close()
    del xs
    kinds = {}
    for o in ops:
        kinds[o.kernel] = kinds.get(o.kernel, 0) + 1
    line = {"metric": "GDoF/s of batched applies and solves, 512 uneven implicit DG systems", "value": total / ms_batch / 1e6,
            "unit": "GDoF/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic (seed 7)",
            "config": {"workload": f"batch of {len(ops)} instances (d in 2..4, p in 1..5, E log-uniform 1e3..1e5, "
                                   "constant velocity, dt 1e-3)", "total_dofs": int(total), "kernels": kinds,
                       "groups": len({(o.space.dim, o.space.order, o.variant) for o in ops if o.kernel == "kronnd"}),
                       "setup_s": setup_s},
            "apply": {"batched_ms": ms_batch, "one_launch_each_ms": ms_each,
                      "batched_gdofs_per_s": total / ms_batch / 1e6, "one_launch_each_gdofs_per_s": total / ms_each / 1e6},
            "solve": {"tol": 1e-10, "preconditioner": "element mass inverse (right)",
                      "fp64_gmres20_one_launch_each": fp64, "batched_mixed_ir_gmres20": batched,
                      "fp64_over_batched_wall": fp64["wall_s"] / batched["wall_s"]}}
    print(json.dumps(line))
    return 0


WORKLOAD_SIPDG = ("fp64 symmetric interior-penalty DG diffusion, 3D 32^3 hex, p=4 GLL, q=6 GL, mu_e = exp(z_e) "
                  "z ~ N(0, 0.5^2) seed 4, tau = 10 (p+1)^2 / h, Dirichlet 0")


def run_sipdg(args):
    """Configuration 4: the SIPDG apply (value), the forward CG solve A(mu) u = f to 1e-12, the
    gradient of J = 1/2 |u - u*|^2 with respect to z (mu = exp z) by one adjoint CG solve and one
    coefficient-gradient launch, checked by central differences (eps = 1e-6) on `--fd` random
    elements (each difference solve warm-started from u) and by the linearity identity
    sum_e dmu_e dA/dmu_e = A(dmu)."""
    import numpy as np
    import torch
    import gendil_b200 as g

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    n, p, q = args.size_sipdg, 4, 6
    space = g.Space(3, [n] * 3, order=p)
    ne, nd = space.num_elements, space.num_dofs
    z = torch.tensor(np.random.default_rng(4).normal(0.0, 0.5, ne), device=dev)
    mu = torch.exp(z)
    kappa = 10.0 * (p + 1) ** 2
    op = g.SIPDGOperator(space, q, mu, sigma=-1.0, kappa=kappa, boundary=True)
    f = torch.from_numpy(g.fill_random(nd, 5)).to(dev)
    ustar = torch.from_numpy(g.fill_random(nd, 6)).to(dev)
    x = torch.from_numpy(g.fill_random(nd, 1)).to(dev)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    for _ in range(args.warmup):
        op(x, y)
    torch.cuda.synchronize()
    e0, e1 = events()
    with ClockSampler(0) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            op(x, y)
        e1.record(stream)
        torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / args.steps
    value = nd / (ms_step * 1e-3) / 1e9

    def cg(rhs, x0=None, tol=1e-12):
        u = torch.zeros_like(rhs) if x0 is None else x0.clone()
        s = g.CGSolver(op)
        a, b = events()
        a.record(stream)
        info = s.solve(rhs, u, 100000, tol)
        b.record(stream)
        torch.cuda.synchronize()
        s.close()
        return u, info, a.elapsed_time(b) * 1e-3

    if args.no_solve:
        print(json.dumps({"metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": 1, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
                          "dtype": "f64", "data": "synthetic", "gpu_launches": args.steps,
                          "config": {"workload": WORKLOAD_SIPDG.replace("32^3", f"{n}^3"), "dofs": nd,
                                     "kernel": op.kernel, "note": "apply only (--no-solve)"}}))
        op.close()
        return 0
    cg(f, tol=1e-2)  # warm-up
    u, info_f, t_fwd = cg(f)
    r = torch.empty_like(u)
    op(u, r)
    fwd_res = (torch.linalg.vector_norm(f - r) / torch.linalg.vector_norm(f)).item()
    lam, info_a, t_adj = cg(u - ustar)
    a, b = events()
    gmu = op.coefficient_gradient(u, lam)  # warm-up of the launch
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(10):
        op.coefficient_gradient(u, lam, out=gmu)
    b.record(stream)
    torch.cuda.synchronize()
    t_grad_ms = a.elapsed_time(b) / 10
    gz = -mu * gmu  # dJ/dz_e = mu_e dJ/dmu_e = -mu_e lam^T (dA/dmu_e) u

    # linearity identity: sum_e dmu_e lam^T (dA/dmu_e) u = lam^T A(dmu) u
    dmu = torch.tensor(np.random.default_rng(11).normal(0.0, 1.0, ne), device=dev)
    opd = g.SIPDGOperator(space, q, dmu, sigma=-1.0, kappa=kappa, boundary=True)
    w = torch.empty_like(u)
    opd(u, w)
    opd.close()
    lhs, rhs = float(dmu @ gmu), float(lam @ w)
    lin_rel = abs(lhs - rhs) / max(abs(rhs), 1e-300)

    fd = []
    if args.fd > 0:
        # central differences: each perturbed solve warm-started from u, to 1e-10 of its initial
        # residual (the perturbation touches one element's rows, so the correction is of order
        # eps), and J(z+) - J(z-) = 1/2 (u+ - u-) . (u+ + u- - 2 u*) without cancellation
        eps = 1e-6
        for e in np.random.default_rng(12).choice(ne, args.fd, replace=False):
            sols = []
            for sgn in (1.0, -1.0):
                zp = z.clone()
                zp[int(e)] += sgn * eps
                mup = torch.exp(zp)
                opp = g.SIPDGOperator(space, q, mup, sigma=-1.0, kappa=kappa, boundary=True)
                up = u.clone()
                sv = g.CGSolver(opp)
                sv.solve(f, up, 100000, 1e-10)
                sv.close()
                opp.close()
                sols.append(up)
            up, um = sols
            dj = 0.5 * float(torch.sum((up - um) * (up + um - 2.0 * ustar)))
            fd.append((dj / (2 * eps), float(gz[int(e)])))
    gmax = float(gz.abs().max())
    fd_err = max((abs(a_ - b_) for a_, b_ in fd), default=None)
    fd_rel = max((abs(a_ - b_) / abs(b_) for a_, b_ in fd), default=None)

    hbm, peak_kind = peaks()
    alg = 16.0 * nd + 8.0 * ne
    achieved = alg / (ms_step * 1e-3) / 1e9
    D, N = 3, p + 1
    # per DoF: the D axis passes (Khat_a, N FMA, plus the rank-one face terms: own and neighbour
    # value / derivative traces and the four-term update, 12 FMA) and D(D-1) tangential mass
    # passes (N FMA each); 2 flop per FMA
    flop = 2 * (D * (N + 12) + D * (D - 1) * N)
    peak64 = fp64_gemm_peak(torch, dev)
    a64 = flop * nd / (ms_step * 1e-3) / 1e12
    line = {"metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (FillRandom seeds 1, 5, 6; numpy normal seed 4)",
            "config": {"workload": WORKLOAD_SIPDG.replace("32^3", f"{n}^3"), "dofs": nd, "elements": ne, "kernel": op.kernel,
                       "l2": f"inputs smaller than L2 ({8 * nd / 1e6:.0f} MB each); applies back to back"},
            # the 33 MB vectors stay in L2 across back-to-back applies: this is an L2-resident
            # figure, not an HBM roofline (ncu: 34.3 MB of DRAM traffic per 32^3 launch, x and mu
            # read once, y still in L2 when the launch ends)
            "roofline": {"bound": "l2-resident", "achieved": achieved, "unit": "GB/s",
                         "hbm_peak_for_reference": hbm, "traffic": 34.3e6 if n == 32 else None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg},
            "roofline_fp64": {"bound": "fp64", "achieved": a64, "peak": peak64, "unit": "TFLOP/s", "frac": a64 / peak64,
                              "flop_per_dof": flop, "peak_kind": "measured: cuBLAS DGEMM 8192^3 (torch), best of 3"},
            "gpu_launches": args.steps, "clocks": clocks.summary(),
            "gradient": {"loss": "J = 1/2 |u - u*|^2, A(exp z) u = f", "forward_cg_s": t_fwd,
                         "forward_iterations": info_f["iterations"], "forward_true_relative_residual": fwd_res,
                         "adjoint_cg_s": t_adj, "adjoint_iterations": info_a["iterations"],
                         "gradient_kernel_ms": t_grad_ms, "gradient_total_s": t_fwd + t_adj + t_grad_ms * 1e-3,
                         "max_abs_dJdz": gmax, "linearity_rel_err": lin_rel,
                         "fd_elements": len(fd), "fd_eps": 1e-6, "fd_max_abs_err": fd_err,
                         "fd_max_rel_err_vs_max_grad": None if fd_err is None else fd_err / gmax,
                         "fd_max_rel_err_per_element": fd_rel}}
    print(json.dumps(line))
    op.close()
    return 0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--no-solve", action="store_true", help="skip the GMRES solve leg")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", type=int, default=None,
                    help="elements per axis (profiling runs only; defaults 64 for 3d, 8 for 6d, 32 for sipdg)")
    ap.add_argument("--variant", default=None, help="force a Kronecker-kernel variant (profiling runs only)")
    ap.add_argument("--workload", choices=["3d", "6d", "batch", "sipdg"], default="3d",
                    help="3d: the 64^3 p=3 advection apply (default); 6d: the 8^6 p=2 phase-space configuration; "
                         "batch: 512 uneven implicit systems; sipdg: 32^3 p=4 diffusion apply, solve and gradient")
    ap.add_argument("--fd", type=int, default=64, help="sipdg workload: elements checked by central differences")
    ap.add_argument("--instances", type=int, default=512, help="batch workload: number of instances")
    args = ap.parse_args(argv)
    args.size_6d = args.size or 8
    args.size_sipdg = args.size or 32
    args.size = args.size or N_AXIS
    if args.warmup < 3:
        args.warmup = 3
    return args


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "sipdg":
        return run_sipdg(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

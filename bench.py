#!/usr/bin/env python
"""Benchmark of the B200 numeric phase of smf: factor + solve ms.

Default workload (the headline metric's configuration): the SPD
variable-coefficient 7-point operator on a 64^3 grid (n = 262,144; edge
conductivities log-uniform in [1e-3, 1e3], seed 0) on smf's own METIS
analysis (rebuilt from the record tests/golden/spd3d64_smf_partition.npz),
one right-hand side uniform in [-1, 1]. One step = numeric factorization of
the values + one solve + refinement to the metric's backward-error bar.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config spd3d|spd3d40|lap2d|traj|kkt|kkt3|batch] [--precision fp64|mixed|both]

`value` is device time (CUDA events on the engine's stream) with the
inputs already in HBM; `e2e` is the same step through the C ABI with host
buffers (values and right-hand side copied in, solution copied out).
Multi-GPU: one process per GPU; the 64^3 factorization does not shard, so
N ranks run N replicas ("replicas only") and the max over ranks is reported.
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

CONFIGS = {
    # name: (description, builder, posdef, nrhs)
    "spd3d": ("SPD variable-coefficient 7-point 64^3 (n=262,144), 1 RHS", "varcoef_3d(64)", True, 1),
    "lap2d": ("2D 5-point Laplacian 150x150 (n=22,500), 1 RHS", "laplacian_2d(150)", True, 1),
    "traj": ("trajectory KKT T=200 (n=5,612), 8 RHS", "traj200", False, 8),
    "kkt": ("IPM KKT 20^3 + 4,000 constraints (n=12,000), smf's METIS ordering, 1 RHS N(0,1)",
            "kkt_ipm(20, 4000)", False, 1),
    # configuration 3 at full size on smf's own METIS analysis
    "kkt3": ("IPM KKT 40^3 + 32,000 constraints (n=96,000), Sigma 10^U[-8,8], delta 1e-8, smf's METIS "
             "ordering, u=0.01, 1 RHS N(0,1)", "kkt_ipm(40, 32000)", False, 1),
    # the same generator as spd3d at 40^3: the small case of the ncu captures
    "spd3d40": ("SPD variable-coefficient 7-point 40^3 (n=64,000), 1 RHS", "varcoef_3d(40)", True, 1),
    # configuration 4: 1,024 trajectory KKTs (T uniform in 10..200) in one batch
    "batch": ("1,024 trajectory KKT systems, T in {10..200} (n = 28T + 12 each), 8 RHS each",
              "trajectory_batch(1024)", False, 8),
}
BATCH_COUNT = 1024
# configuration 5: interior-point refactor streams, the analysis reused
STREAMS = {
    # the 64^3 pattern with the barrier diagonal Sigma_k added (SPD)
    "stream": ("refactor stream: 64^3 SPD pattern + Sigma_k on the diagonal, 60 refactors, 1 RHS", "spd3d", True),
    # the KKT at the size the reference factors, Sigma_k on the primal block
    "kktstream": ("refactor stream: IPM KKT 20^3 + 4,000 (n=12,000), Sigma_k on the primal diagonal, "
                  "60 refactors, 1 RHS", "kkt", False),
}
STREAM_LEN = 60


def batch_systems(rank: int = 0, world: int = 1):
    """This rank's contiguous share of configuration 4's systems."""
    from opt_solver_b200 import workloads as W
    from opt_solver_b200.batch import shard
    mats = W.trajectory_batch(BATCH_COUNT, seed=0)
    lo, hi = shard(BATCH_COUNT, rank, world)
    return mats[lo:hi]


class _Workload:
    """One system (Solver) or a batch of systems merged into one forest
    (BatchSolver), with its values and right-hand sides."""

    def __init__(self, cfg, device, rank=0, world=1):
        from opt_solver_b200 import smfg
        from opt_solver_b200 import workloads as W
        from opt_solver_b200.batch import BatchSolver
        self.desc, _, self.posdef, self.nrhs = CONFIGS[cfg]
        t0 = time.time()
        if cfg == "batch":
            mats = batch_systems(rank, world)
            ans = [smfg.analyse(n, cp, ri) for n, cp, ri, v in mats]
            self.analyse_s = time.time() - t0
            self.solver = BatchSolver(ans, device=device)
            self.values = np.concatenate([m[3] for m in mats])
            self.b = self.solver.stack_rhs([W.rhs(m[0], self.nrhs, seed=i, kind="normal")
                                            for i, m in enumerate(mats)])
            self.n = self.solver.n
            self.nnz = int(sum(int(m[1][-1]) for m in mats))
            self.nsn = self.solver.merged.nsn
            self.systems = len(mats)
            self.sv = self.solver.solver
            self.scale = None
            self.expected = [(16 * ((m[0] - 12) // 28) + 12, 12 * ((m[0] - 12) // 28), 0) for m in mats]
        else:
            n, cp, ri, v = build_matrix(cfg)
            rec = smf_record(cfg)
            if rec is not None:
                from opt_solver_b200 import smf_analysis
                a = smf_analysis.load(rec, n, cp, ri)
                self.ordering = "smf's own analysis (%s), rebuilt from its record %s" % (
                    SMF_RECORDS[cfg][1], os.path.relpath(rec, ROOT))
            else:
                a = smfg.analyse(n, cp, ri)
                self.ordering = "engine nested dissection (smfg_analyse)"
            self.analyse_s = time.time() - t0
            self.sv = smfg.Solver(a, device=device)
            self.solver = self.sv
            self.values = v
            self.b = W.rhs(n, self.nrhs, seed=1, kind="normal" if cfg.startswith("kkt") else "uniform")
            # the KKT configurations run with max-product matching scaling on
            self.scale = smfg.matching_scale(n, cp, ri, v)[0] if cfg.startswith("kkt") else None
            self.n = n
            self.nnz = int(cp[-1])
            self.nsn = a.nsn
            self.systems = 1
            self.expected = None

    def inertia_ok(self, rank=0, world=1):
        """Every system's inertia exact: on N ranks each rank's slice of the
        batch is gathered in system order first."""
        if self.expected is None:
            return True
        if world == 1:
            return [s[:3] for s in self.solver.system_stats()] == self.expected
        from opt_solver_b200.batch import gather_system_stats, shard
        lo, _ = shard(BATCH_COUNT, rank, world)
        allst = gather_system_stats(self.solver.system_stats(), lo, BATCH_COUNT, world)
        want = [(16 * ((m[0] - 12) // 28) + 12, 12 * ((m[0] - 12) // 28), 0) for m in batch_systems()]
        return [tuple(int(x) for x in r[:3]) for r in allst] == want


# smf's analysis of each workload, recorded by the reference itself
# (tests/golden/make_smf_partitions.py): (record, ordering smf used)
SMF_RECORDS = {"spd3d": ("spd3d64", "METIS"), "lap2d": ("lap2d150", "its minimum degree (AMD)"),
               "kkt": ("kkt20_4000", "METIS"), "kkt3": ("kkt40_32000", "METIS")}


def smf_record(cfg: str):
    """The record of smf's analysis of a workload (perm and supernode
    partition), or None: the engine's own analysis orders the matrix."""
    if cfg not in SMF_RECORDS:
        return None
    return os.path.join(ROOT, "tests", "golden", f"{SMF_RECORDS[cfg][0]}_smf_partition.npz")


def build_matrix(cfg: str):
    from opt_solver_b200 import workloads as W
    if cfg == "spd3d":
        return W.varcoef_3d(64, seed=0)
    if cfg == "lap2d":
        return W.laplacian_2d(150)
    if cfg == "traj":
        return W.trajectory_kkt(200, np.random.default_rng(0))
    if cfg == "kkt":
        return W.kkt_ipm(20, 4000, seed=0)
    if cfg == "kkt3":
        return W.kkt_ipm(40, 32000, seed=0)
    if cfg == "spd3d40":
        return W.varcoef_3d(40, seed=0)
    raise ValueError(cfg)


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl" if _cuda_ok() else "gloo", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device="cuda" if _cuda_ok() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except Exception:  # noqa: BLE001
        return {}


def dgemm_peak_tflops():
    """cuBLAS FP64 GEMM throughput on this GPU (the FP64 roofline's
    denominator: the driver's peak file measures bf16 and copy bandwidth)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def dominant_roofline(prof: dict, head: str, A: dict, peaks: dict, dgemm_peak=None, solve=None) -> dict:
    """The roofline object of the JSON line for the step's dominant kernel by
    device time, from the profiled factorization's counters (``prof``), the
    timed arm (``A``: its factor_ms) and the measured peaks. Candidates: the
    streamed FP64 deferred updates (HBM-bound), the FP64 Schur updates, the
    tensor-core passes of the mixed fronts, the pivoting panels, and the
    solves of the step (``solve``: ms per solve, solves per step including
    the refinement's, algorithmic bytes per solve)."""
    dgemm_peak = dgemm_peak or dgemm_peak_tflops
    defer_ms = max(prof.get("gemm_ms", 0.0) - prof.get("schur_ms", 0.0), 0.0)
    cands = {"defer": defer_ms, "tc": prof.get("tc_ms", 0.0) if head == "mixed" else 0.0,
             "fp64": prof.get("gemm_ms", 0.0) if defer_ms <= 0.0 else prof.get("schur_ms", 0.0),
             "solve": solve["ms"] * solve["count"] if solve and solve.get("bytes") else 0.0}
    kernel_ms = {"defer": defer_ms, "schur_fp64": prof.get("schur_ms"), "tc": prof.get("tc_ms"),
                 "pivoting_panels": prof.get("panel_ms"), "solves": cands["solve"]}
    dom = max(cands, key=cands.get) if max(cands.values()) > 0 else None
    hbm = peaks.get("hbm_gbs") or 6650.0
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (burst copy)" if peaks.get("hbm_gbs") else "fallback 6650 GB/s"
    if dom == "solve":
        achieved = solve["bytes"] / (solve["ms"] * 1e-3) / 1e9
        roof = {
            "kernel": "supernodal forward + backward sweeps (k_fwd_* / k_bwd_*, gather and scatter), one solve",
            "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": solve.get("traffic"), "traffic_source": solve.get("traffic_source"),
            "peak_source": hbm_src, "solves_per_step": solve["count"], "avg_solve_ms": solve["ms"],
            "algorithmic_bytes_per_solve": solve["bytes"],
            "algorithmic_bytes_source": "2 sweeps x (8 |L| + 4 sum f + 16 n nrhs)",
            "kernel_ms": kernel_ms,
        }
    elif dom == "defer" and prof.get("defer_bytes", 0) > 0:
        # bytes: every entry of each deferred update's trapezoid read and
        # written once (16 bytes), summed on the device
        achieved = prof["defer_bytes"] / (defer_ms * 1e-3) / 1e9
        nupd = max(prof.get("defer_updates", 0), 1)
        roof = {
            "kernel": "k_large_defer (streamed FP64 deferred updates of the large fronts, rank <= 16)",
            "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": DEFER_DRAM_BYTES_PER_ENTRY * (prof["defer_bytes"] / 16.0) / max(prof["gemm_launches"], 1),
            "traffic_source": "per launch, scaled by updated entries from the ncu capture of one "
                              "8,000-row front of the kernel",
            "peak_source": hbm_src,
            "launches": prof["gemm_launches"], "front_updates": prof.get("defer_updates"),
            "front_updates_of_at_most_2_pivots": prof.get("defer_small"),
            "avg_launch_ms": defer_ms / max(prof["gemm_launches"], 1),
            "algorithmic_bytes_per_launch": prof["defer_bytes"] / max(prof["gemm_launches"], 1),
            "algorithmic_bytes_per_front_update": prof["defer_bytes"] / nupd,
            "kernel_ms": kernel_ms,
        }
    elif dom == "tc":
        # the tensor-core trailing updates (split + product kernels) against
        # the tensor pipe's rate for TF32 (half the measured BF16 dense
        # rate) divided by the 3 split products each algorithmic product costs
        bf = peaks.get("bf16_tflops") or 1590.0
        peak = bf / 2.0 / 3.0
        achieved = prof["tc_flops"] / (prof["tc_ms"] * 1e-3) / 1e12
        roof = {
            "kernel": "k_tc_split + k_tc_syrk (tcgen05 TF32x3 trailing updates of the mixed fronts)",
            "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": None,
            "peak_source": ("MEASURED_PEAKS.json bf16_tflops" if peaks.get("bf16_tflops") else "fallback 1590")
            + " / 2 (TF32 rate) / 3 (split products per algorithmic product)",
            "launches": prof["tc_passes"], "avg_launch_ms": prof["tc_ms"] / max(prof["tc_passes"], 1),
            "algorithmic_flops_per_launch": prof["tc_flops"] / max(prof["tc_passes"], 1),
        }
    elif dom == "fp64":
        dpeak = dgemm_peak()
        achieved = prof["gemm_flops"] / (prof["gemm_ms"] * 1e-3) / 1e12
        roof = {
            "kernel": "k_large_defer + k_large_schur (FP64 FMA updates of the large fronts)",
            "bound": "tensor", "achieved": achieved, "peak": dpeak, "unit": "TFLOP/s",
            "frac": achieved / dpeak if dpeak else None, "traffic": None,
            "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (FP64 is not in MEASURED_PEAKS.json)",
            "launches": prof["gemm_launches"], "avg_launch_ms": prof["gemm_ms"] / max(prof["gemm_launches"], 1),
            "algorithmic_flops_per_launch": prof["gemm_flops"] / max(prof["gemm_launches"], 1),
        }
    else:
        # no large fronts (the batch of small systems): the factor as a
        # whole against HBM, its algorithmic bytes the front arena written by
        # assembly and read + written by the front kernels (3 passes)
        achieved = 3.0 * prof.get("arena_bytes", 0.0) / (A["factor_ms"] * 1e-3) / 1e9 if A["factor_ms"] else 0.0
        roof = {
            "kernel": "whole factorization (level kernels of small fronts)", "bound": "hbm",
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
            "peak_source": hbm_src,
            "algorithmic_bytes_per_factor": 3.0 * prof.get("arena_bytes", 0.0),
        }
    return roof


OMEGA_GATE = 1e-12  # the metric's scaled backward error bar
# DRAM bytes k_large_defer moves per updated entry, from one ncu capture of
# the kernel on an 8,000-row front (192.8 MB read + 134.8 MB written for
# 23.9 M entries); the bench's traffic
# per launch is this times the entries its launches update
DEFER_DRAM_BYTES_PER_ENTRY = (192.8e6 + 134.8e6) / 23.9e6
GRAPH_REPLAY = {"kkt": False, "kkt3": False}  # configurations whose steps replay a CUDA graph (default: yes)
# repeats of the full workload in the CPU-baseline leg (about 10-30 s of host work)
CPU_REPS = {"spd3d": 3, "lap2d": 30, "kkt": 5, "traj": 30, "batch": 1}


def run_ours(args, rank, world, local):
    """Both arms on the same workload: plain FP64 and mixed precision, each
    step = factor + solve + refinement (auto: FGMRES on a mixed factor, classical
    then FGMRES on an FP64 one) until
    eta_inf <= 1e-10 and omega <= 1e-12, all on the device; per arm the
    mean device time of K steps after W warm-up steps, max over ranks."""
    import torch
    from opt_solver_b200 import smfg

    torch.cuda.set_device(local)
    wl = _Workload(args.config, local, rank, world)
    sv, posdef = wl.sv, wl.posdef
    d_vals = torch.from_numpy(np.ascontiguousarray(wl.values)).cuda()
    d_b0 = torch.from_numpy(np.ascontiguousarray(wl.b)).cuda()
    d_x = d_b0.clone()
    arms = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    # the refactor of an unchanged pattern replays the captured factor
    # sequence (the first warm-up step captures); the KKT configurations'
    # pivoting runs data-dependent step counts (a fixed-budget graph gains
    # nothing there), so they launch directly
    use_graph = GRAPH_REPLAY.get(args.config, True)
    head = "mixed" if "mixed" in arms else "fp64"
    res = {}
    xs = {}
    clocks = None
    for arm in arms:
        prec = smfg.PREC_MIXED if arm == "mixed" else smfg.PREC_FP64

        def step():
            info = sv.factor(d_vals, posdef=posdef, precision=prec, scale=wl.scale, graph=use_graph)
            d_x.copy_(d_b0)
            sv.solve(d_x)
            eta, om, its = sv.refine_device(d_b0, d_x, nrhs=wl.nrhs, max_steps=args.refine_max,
                                            omega_target=OMEGA_GATE, method=smfg.REFINE_AUTO)
            f, so, rf = sv.last_times()
            return f + so + rf, (f, so, rf), info, (eta, om, its)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        barrier(world)
        dev, parts = [], []
        sampler = ClockSampler(local)
        with sampler as clk:
            for _ in range(args.steps):
                ms, pr, info, acc = step()
                dev.append(ms)
                parts.append(pr)
        torch.cuda.synchronize()
        barrier(world)
        xs[arm] = d_x.cpu().numpy().copy()
        if arm == head:
            clocks = clk.summary()
        ms_step = allmax(sum(dev) / len(dev), world)
        fm = [p_[0] for p_ in parts]
        sm_ = [p_[1] for p_ in parts]
        rm = [p_[2] for p_ in parts]
        res[arm] = {
            "ms": ms_step, "factor_ms": sum(fm) / len(fm), "solve_ms": sum(sm_) / len(sm_),
            "refine_ms": sum(rm) / len(rm), "eta_inf": acc[0], "omega": acc[1], "refine_solves": acc[2],
            "inertia": list(info.inertia), "inertia_exact_per_system": wl.inertia_ok(rank, world),
            "mixed_fronts": int(info.mixed_fronts), "kernel_launches": int(info.kernel_launches),
            "flops": info.flops, "delayed": int(info.delayed_pivots),
            "info": info,
        }
    # the arms agree on the inertia; the mixed arm's forward error against
    # the plain FP64 arm's solution
    if len(arms) == 2:
        res["inertia_same"] = res["fp64"]["inertia"] == res["mixed"]["inertia"]
        res["mixed"]["forward_error_vs_fp64"] = forward_error(xs["mixed"], xs["fp64"])
    # e2e: host buffers through the C ABI (copies inside the timed region)
    prec = smfg.PREC_MIXED if head == "mixed" else smfg.PREC_FP64
    e2e = []
    # the caller's host buffers in pinned memory (values, right-hand side,
    # solution): the copies inside the timed region are DMA transfers
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory().numpy()
    h_vals, h_b = pinned(wl.values), pinned(wl.b)
    h_x = pinned(np.zeros_like(wl.b))
    # one untimed call first: it captures the factor graph for the staged
    # host values (the timed calls replay it, as a refactor loop would)
    sv.factor(h_vals, posdef=posdef, precision=prec, scale=wl.scale, graph=use_graph)
    for _ in range(max(2, min(args.steps, 5))):
        torch.cuda.synchronize()
        t = time.perf_counter()
        sv.factor(h_vals, posdef=posdef, precision=prec, scale=wl.scale, graph=use_graph)
        x = sv.solve(h_b, out=h_x)
        x, _, _, _ = sv.refine(h_b, x, max_steps=args.refine_max, omega_target=OMEGA_GATE,
                               method=smfg.REFINE_AUTO, inplace=True)
        e2e.append((time.perf_counter() - t) * 1e3)
    e2e_ms = allmax(sum(e2e) / len(e2e), world)
    _, eta, om = sv.residual(wl.b, x)
    prof = sv.profile_factor(d_vals, posdef=posdef, precision=prec, scale=wl.scale)
    A_info = res[head]["info"]
    front_rows = int(sv.factor_sizes()[1])
    return {
        "arms": res, "head": head, "e2e_ms": e2e_ms, "e2e_eta": eta, "e2e_omega": om,
        "analyse_s": wl.analyse_s, "n": wl.n, "nnz": wl.nnz, "nrhs": wl.nrhs, "desc": wl.desc,
        "graph": use_graph,
        "ordering": getattr(wl, "ordering", "engine nested dissection (smfg_analyse)"),
        "clocks": clocks, "nsn": wl.nsn, "systems": wl.systems,
        "h2d": wl.nnz * 8 + wl.n * wl.nrhs * 8, "d2h": wl.n * wl.nrhs * 8, "profile": prof,
        "x_fp64": xs.get("fp64"), "b": wl.b, "values": wl.values,
        "factor_entries": int(A_info.factor_entries), "front_rows": front_rows,
    }


SELECTOR_FILE = os.path.join(ROOT, "opt_solver_b200", "data", "selector.npz")


def run_stream(args, rank, world, local):
    """Configuration 5: one analysis, then refactors of a barrier-parameter
    stream; per step factor + solve + refinement (auto) to omega <= 1e-12,
    device time. Arms: plain FP64; and graph replay + mixed precision +
    the learned selector's mask (decided once from the stream's first, plain
    factorization) with the FP64 judge (fronts whose counts changed against
    the previous step are refactored in FP64 and leave the mask)."""
    import torch
    from opt_solver_b200 import selector as S
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W

    torch.cuda.set_device(local)
    desc, base, posdef = STREAMS[args.config]
    n, cp, ri, v = build_matrix(base)
    t0 = time.time()
    rec = smf_record(base)
    if rec is not None:
        from opt_solver_b200 import smf_analysis
        a = smf_analysis.load(rec, n, cp, ri)
    else:
        a = smfg.analyse(n, cp, ri)
    analyse_s = time.time() - t0
    dslot = W.diagonal_slots(n, cp, ri)
    base_vals = np.array(v, dtype=np.float64)
    if posdef:
        sig_idx = np.arange(n)
        expected = (n, 0, 0)
    else:
        nh = 20 ** 3
        sig_idx = np.arange(nh)
        base_vals[dslot[:nh]] = 6.0  # H's diagonal without the barrier term
        expected = (nh, n - nh, 0)
    sig = W.sigma_stream(sig_idx.size, STREAM_LEN, seed=5)
    vals = np.repeat(base_vals[None, :], STREAM_LEN, axis=0)
    vals[:, dslot[sig_idx]] += sig
    scale = None if posdef else smfg.matching_scale(n, cp, ri, vals[0])[0]
    d_all = torch.from_numpy(vals).cuda()
    d_vals = torch.empty(vals.shape[1], dtype=torch.float64, device="cuda")
    b = W.rhs(n, 1, seed=1, kind="normal")
    d_b0 = torch.from_numpy(b).cuda()
    d_x = d_b0.clone()
    sv = smfg.Solver(a, device=local)
    sel = S.load(SELECTOR_FILE, device=local) if os.path.exists(SELECTOR_FILE) else None
    res = {}
    clocks = None
    for arm in ("fp64", "mixed"):
        lat, fac, sol, ref_ms, solves, inertia_ok, fallbacks = [], [], [], [], [], 0, 0
        prev = None
        mask = None
        sampler = ClockSampler(local)
        with sampler as clk:
            for it in range(args.warmup + args.steps):
                k = it % STREAM_LEN
                d_vals.copy_(d_all[k])
                nbad = 0
                if arm == "fp64" or prev is None:
                    info = sv.factor(d_vals, posdef=posdef, scale=scale)
                    f_ms = info.factor_ms
                else:
                    if mask is None:
                        X = S.front_features(a, vals[k], posdef, prev, scale)
                        mask = sel.mask(a, X) if sel is not None else S.candidates(a).astype(np.int8)
                    info, mask, nbad = S.factor_checked(sv, a, d_vals, posdef, mask, prev, expected, scale,
                                                        graph=True)
                    f_ms = info.total_ms
                if arm == "mixed":
                    prev = sv.front_stats()
                d_x.copy_(d_b0)
                sv.solve(d_x)
                eta, om, its = sv.refine_device(d_b0, d_x, nrhs=1, max_steps=args.refine_max,
                                                omega_target=OMEGA_GATE, method=smfg.REFINE_AUTO)
                _, s_ms, r_ms = sv.last_times()
                if it >= args.warmup:
                    lat.append(f_ms + s_ms + r_ms)
                    fac.append(f_ms)
                    sol.append(s_ms)
                    ref_ms.append(r_ms)
                    solves.append(its)
                    inertia_ok += int(tuple(info.inertia) == expected and om <= OMEGA_GATE)
                    fallbacks += nbad
        if arm == "mixed":
            clocks = clk.summary()
        res[arm] = {
            "ms_mean": float(np.mean(lat)), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "factor_ms_mean": float(np.mean(fac)),
            "solve_ms_mean": float(np.mean(sol)), "refine_ms_mean": float(np.mean(ref_ms)),
            "refine_solves_mean": float(np.mean(solves)), "refine_solves_max": int(np.max(solves)),
            "steps_inertia_exact_and_omega_met": inertia_ok, "steps": len(lat),
            "fp64_fallback_fronts": fallbacks,
            "mixed_fronts": int(mask.sum()) if (arm == "mixed" and mask is not None) else 0,
        }
    sv.close()
    M, P = res["mixed"], res["fp64"]
    return {
        "metric": "factor+solve ms", "value": allmax(M["ms_mean"], world), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": allmax(M["ms_mean"], world),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (tf32x3 tensor-core updates on the selected fronts)",
        "data": "synthetic (seeded generator of the configuration)",
        "config": {"workload": desc, "n": n, "nnz_lower": int(cp[-1]), "stream_length": STREAM_LEN,
                   "analysis_s": analyse_s, "selector": "trained (opt_solver_b200/data/selector.npz)"
                   if sel is not None else "none (every large front mixed)",
                   "step": "refactor + solve + refinement (auto) to eta_inf <= 1e-10, omega <= 1e-12",
                   "l2": "inputs larger than L2" if vals.shape[1] * 8 > 126e6 else "per-step values fit L2"},
        "arms": res, "mixed_speedup_vs_plain": P["ms_mean"] / M["ms_mean"],
        "gpu_launches": None, "clocks": clocks,
    }


def forward_error(x, x_ref):
    """max |x - x_ref| / max |x_ref| (both n x nrhs)."""
    den = float(np.max(np.abs(x_ref))) if np.size(x_ref) else 0.0
    return float(np.max(np.abs(np.asarray(x) - np.asarray(x_ref)))) / den if den > 0 else None


# Configuration 3 at full size is beyond the reference: its root front of
# 32,150 rows exceeds smf's factor storage cap (kMaxFactorStorageEntries =
# 2^29 entries, solver/include/smf/types.hpp:13, checked in
# solver/src/factor_indef.cpp:33-54)
REF_REFUSES = {"kkt3": "smf refuses it: its 32,150-row root front exceeds kMaxFactorStorageEntries = 2^29 "
                       "(types.hpp:13, factor_indef.cpp:33-54)"}
REF_BLAS = "smf's own portable BLAS loops (SMF_BLAS_REFERENCE; the image has no BLAS library)"


def reference_step(cfg, threads, reps):
    """The reference smf solver (oracle/_ref, compiled from its sources) on
    the host cores in its fastest host mode (non-deterministic, `threads`
    threads, LAPACK-style SPD front kernel, its own analysis with the
    ordering the GPU arm's record holds): factor + solve ms of the full
    workload, median of `reps` runs, the analysis outside the timed region
    as in the GPU arm (a refactor). Configuration 4 times its first 64
    systems and scales by the system count. Returns (ms, sample, x of the
    first right-hand side or None)."""
    from oracle import oracle as O
    from opt_solver_b200 import workloads as W
    posdef, nrhs = CONFIGS[cfg][2], CONFIGS[cfg][3]
    if cfg == "batch":
        mats, scale = batch_systems()[:64], BATCH_COUNT / 64
        sample = "the first 64 of the 1,024 systems (one smf analyse, then factor + solve each); time x16"
    else:
        mats, scale = [build_matrix(cfg)], 1.0
        sample = "the full workload"
    order = {"spd3d": O.ORDER_METIS, "kkt": O.ORDER_METIS, "lap2d": O.ORDER_AMD}.get(cfg, O.ORDER_AUTO_PARALLEL)
    refs = []
    for i, (n, cp, ri, v) in enumerate(mats):
        ref = O.Reference(posdef=posdef, ordering=order, deterministic=False, num_threads=threads,
                          scaling=O.SCALE_AUTO, posdef_kernel=O.POSDEF_KERNEL_LAPACK)
        ref.analyse(n, cp, ri, v)
        refs.append((ref, v, W.rhs(n, nrhs, seed=i if cfg == "batch" else 1,
                                   kind="normal" if cfg != "spd3d" and cfg != "lap2d" else "uniform")))
    times, x0 = [], None
    for _ in range(max(1, reps)):
        t = time.perf_counter()
        for ref, v, b in refs:
            ref.factor(v, export=False)
            x, _ = ref.solve(b)
            if x0 is None:
                x0 = x
        times.append((time.perf_counter() - t) * 1e3)
    sample += f"; {REF_BLAS}; median of {len(times)} run(s)"
    return statistics.median(times) * scale, sample, (x0 if cfg != "batch" else None)


def run_reference_arm(args, rank, world):
    if rank != 0:
        return None
    from oracle import oracle as O
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (the reference sources were absent at build time)"}
    cfg = STREAMS[args.config][1] if args.config in STREAMS else args.config
    if cfg in REF_REFUSES:
        return {"impl": "reference", "unavailable": REF_REFUSES[cfg]}
    threads = os.cpu_count() or 1
    times = []
    sample = ""
    for i in range(args.warmup + args.steps):
        ms, sample, _ = reference_step(cfg, threads, 1)
        if i >= args.warmup:
            times.append(ms)
    ms_step = statistics.median(times)
    desc = STREAMS[args.config][0] if args.config in STREAMS else CONFIGS[args.config][0]
    return {
        "impl": "reference", "metric": "factor+solve ms", "value": ms_step, "unit": "ms",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators of the configuration)",
        "config": {"workload": desc, "precision": "fp64"},
        "cpu_baseline": {"value": ms_step, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": ms_step, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def ncu_step(args):
    """One factorization and one solve of the workload, nothing else: the
    command the committed ncu launch lists are taken from."""
    import torch
    from opt_solver_b200 import smfg
    wl = _Workload(args.config, 0)
    prec = smfg.PREC_FP64 if args.precision == "fp64" else smfg.PREC_MIXED
    d_vals = torch.from_numpy(np.ascontiguousarray(wl.values)).cuda()
    d_b = torch.from_numpy(np.ascontiguousarray(wl.b)).cuda()
    info = wl.sv.factor(d_vals, posdef=wl.posdef, precision=prec, scale=getattr(wl, "scale", None))
    fl = info.kernel_launches
    wl.sv.solve(d_b)
    torch.cuda.synchronize()
    print(json.dumps({"factor_launches": fl, "factor_ms": info.factor_ms,
                      "solve_ms": wl.sv.info.solve_ms}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="spd3d", choices=sorted(list(CONFIGS) + list(STREAMS)))
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"],
                    help="both: time the plain FP64 and the mixed arm; the value is the mixed one")
    ap.add_argument("--refine-max", type=int, default=30, help="refinement solves per step, at most")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--defer-kernel", nargs=3, type=int, metavar=("F", "NE", "K"),
                    help="time the streamed deferred-update kernel alone on one synthetic front "
                         "(F rows, NE eligible columns, K pending pivots) and exit")
    ap.add_argument("--ncu-step", action="store_true",
                    help="one factorization + solve and exit (for an ncu launch list)")
    args = ap.parse_args()
    if args.defer_kernel:
        from opt_solver_b200 import smfg
        f, ne, k = args.defer_kernel
        r = smfg.kernel_bench_defer(f, ne, k, reps=max(args.steps, 1))
        peaks = measured_peaks()
        hbm = peaks.get("hbm_gbs") or 6650.0
        print(json.dumps({"kernel": "k_large_defer", "f": f, "ne": ne, "k": k, **r,
                          "hbm_frac": r["gbs"] / hbm, "hbm_peak_gbs": hbm}), flush=True)
        return
    if args.ncu_step:
        ncu_step(args)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank, world, local = dist_init()
    if args.impl == "reference":
        line = run_reference_arm(args, rank, world)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return
    if args.config in STREAMS:
        line = run_stream(args, rank, world, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    r = run_ours(args, rank, world, local)
    if rank != 0:
        return
    head = r["head"]
    A = r["arms"][head]
    peaks = measured_peaks()
    prof = r["profile"]
    # the solves of the step: one, plus the refinement's
    sol = {"ms": A["solve_ms"], "count": 1 + int(A["refine_solves"] or 0),
           "bytes": 2.0 * (8.0 * r["factor_entries"] + 4.0 * r["front_rows"] + 16.0 * r["n"] * r["nrhs"])}
    roof = dominant_roofline(prof, head, A, peaks, solve=sol)
    cpu = None
    x_ref = None
    if not args.no_cpu_baseline:
        try:
            from oracle import oracle as O
            if args.config in REF_REFUSES:
                cpu = {"value": None, "unit": "ms", "cores": 0, "kind": "reference",
                       "sample": REF_REFUSES[args.config]}
            elif O.ref_available():
                threads = os.cpu_count() or 1
                # about 10-30 s of host work: repeats of the full workload
                ms, sample, x_ref = reference_step(args.config, threads, CPU_REPS.get(args.config, 3))
                cpu = {"value": ms, "unit": "ms", "cores": threads, "kind": "reference",
                       "sample": sample}
        except Exception as exc:  # noqa: BLE001
            cpu = {"value": None, "unit": "ms", "cores": 0, "kind": "reference", "sample": f"failed: {exc}"}
    if x_ref is not None and r.get("x_fp64") is not None and "fp64" in r["arms"]:
        # the plain arm's solution against the reference's own (its FP64
        # factor on the host, unrefined)
        r["arms"]["fp64"]["forward_error_vs_reference"] = forward_error(
            r["x_fp64"].reshape(np.shape(x_ref)), x_ref)
    batch = args.config == "batch"
    arms = {}
    for k, v in r["arms"].items():
        if isinstance(v, dict):
            arms[k] = {kk: vv for kk, vv in v.items() if kk != "info"}
    line = {
        "metric": "factor+solve ms", "value": A["ms"], "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": A["ms"],
        "higher_is_better": False, "scaling": "strong" if batch else "weak", "vs_baseline": None,
        "dtype": "f64" if head == "fp64" else "f64 (tf32x3 tensor-core trailing updates)",
        "data": "synthetic (seeded generator of the configuration)",
        "config": {"workload": r["desc"], "n": r["n"], "nnz_lower": r["nnz"], "nrhs": r["nrhs"],
                   "supernodes": r["nsn"], "systems_this_rank": r["systems"],
                   "analysis": r["ordering"],
                   "precision": head, "omega_gate": OMEGA_GATE,
                   "step": "factor + solve + refinement (auto: FGMRES on a mixed factor) to eta_inf <= 1e-10, "
                           "omega <= 1e-12",
                   "parallelism": ("systems sharded over ranks" if batch else "replicas") if world > 1 else "1 GPU",
                   "factor_graph_replay": r["graph"],
                   "l2": "inputs larger than L2 (front arena %.1f GB)" % (prof.get("arena_bytes", 0) / 1e9)},
        "e2e": {"value": r["e2e_ms"], "unit": "ms", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"], "omega": r["e2e_omega"]},
        "gpu_launches": int(A["kernel_launches"]),
        "factor_ms": A["factor_ms"], "solve_ms": A["solve_ms"], "refine_ms": A["refine_ms"],
        "flops": A["flops"],
        "gflops": A["flops"] / (A["factor_ms"] * 1e-3) / 1e9 if A["factor_ms"] else None,
        "inertia": A["inertia"], "inertia_exact_per_system": A["inertia_exact_per_system"],
        "eta_inf": A["eta_inf"], "omega": A["omega"],
        "arms": arms,
        "mixed_speedup_vs_plain": (r["arms"]["fp64"]["ms"] / r["arms"]["mixed"]["ms"])
        if len(arms) == 2 else None,
        "inertia_same_both_arms": r["arms"].get("inertia_same"),
        "roofline": roof, "cpu_baseline": cpu, "clocks": r["clocks"],
        "measured_peaks": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops")},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Edge-update throughput of the dynamic label-propagation hot path (B200).

Workload (one GPU): Erdos-Renyi n=1,000,000, mean degree 10, unit weights, k=8 classes assigned
uniformly, 0.5% of vertices labelled; a stream of batches of 10,000 edge updates (50% insertions of
uniform random non-edges, 50% deletions of uniform random edges). One step = one batch: the
on-device CSR patch, connected components of the unlabelled graph with the labels as a sink (the
label-free components leave the solved set), the equations and residual of the changed rows, and
the certified solve back to relative residual <= 1e-6 (fp32 PCG sweeps, fp64 residual refinement).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line. `value` times the step with the batch already in device memory; `e2e` times
the same step through the public API from pinned host arrays, including the host->device copy of
the batch and the device->host read of the step's result. The L2 cache is flushed before every
timed step. With N GPUs every rank runs an independent replica (the path does not shard), and the
throughput is the sum over ranks with the time taken as the maximum over ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge-updates/s at rel-res 1e-6 (p50/p99 relabel latency; SpMM GB/s vs HBM peak)"
# The CPU port's work is SciPy sparse products and NumPy elementwise reductions, which run on one
# thread whatever the core count: that is the thread count both CPU legs report.
CPU_PORT_THREADS = 1
CPU_PORT_NOTE = (f"NumPy/SciPy on one thread (sparse products and elementwise reductions do not thread; "
                 f"{os.cpu_count()} host cores present)")


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--deg", type=float, default=10.0)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--label-frac", type=float, default=0.005)
    ap.add_argument("--batch", type=int, default=10_000)
    ap.add_argument("--target-relres", type=float, default=1e-6)
    ap.add_argument("--tol", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-budget-s", type=float, default=150.0, help="wall budget of the CPU reference legs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the fp64 reference solve between timed steps (err_vs_fp64, label agreement)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch the PCG kernels one by one instead of as a CUDA graph (for kernel profilers)")
    ap.add_argument("--lowp", action="store_true", help="edge-stream: BF16 gathers in the PCG sweeps")
    ap.add_argument("--no-class-sum", action="store_true",
                    help="edge-stream: corrections solve all k class columns (default for k = 4, 8, 12: k-1, the last derived)")
    ap.add_argument("--refine-share", type=float, default=0.2,
                    help="edge-stream: share of the rel-res target a correction round aims for (the fp64 "
                         "residual after it decides whether another round runs)")
    ap.add_argument("--three-kernel", action="store_true",
                    help="edge-stream: the three-kernel PCG iteration instead of the two-kernel one")
    ap.add_argument("--workload", default="edge-stream",
                    choices=["edge-stream", "static", "amg", "batched", "serving", "kernels"],
                    help="edge-stream: the headline (ER 1M edge batches); static: SBM 100k solve + one "
                         "1000-update batch; amg: SBM 1M lognormal, AMG-PCG to rel-res 1e-8; batched: 256 SBM "
                         "instances in one batched solve; serving: resident SBM with mixed Poisson requests")
    ap.add_argument("--requests", type=int, default=200, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: offered load (requests/s)")
    return ap.parse_args(argv)


def workload_name(a):
    return (f"er-n{a.n}-deg{a.deg:g}-k{a.k}-lab{a.label_frac:g}-batch{a.batch}-relres{a.target_relres:g}")


def config(a):
    return {"workload": workload_name(a), "n": a.n, "mean_degree": a.deg, "k": a.k, "label_frac": a.label_frac,
            "batch_updates": a.batch, "insert_frac": 0.5, "target_relres": a.target_relres, "tol": a.tol,
            "l2": "flushed before every timed step (256 MB write)", "parallelism": "replicas",
            "pcg_iteration": "three kernels" if a.three_kernel else "two kernels (fp32 whole rows)",
            "class_sum": "off" if a.no_class_sum else "auto (on for k = 4, 8, 12)",
            "refine_share": a.refine_share,
            "python_gc": "collected before the timed loops, paused during them"}


# ---------------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling every 20 ms on a reader thread; `wait_first` blocks (a few seconds at
    most) until the first sample is in, so the timed region is covered from its start."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        import threading
        self.p, self.lines, self.first = None, [], threading.Event()
        self.t0 = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "20"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.p.stdout:
            if line.strip():
                self.lines.append((time.perf_counter(), line.strip()))
                self.first.set()

    def wait_first(self, timeout=10.0):
        if self.p is not None:
            self.first.wait(timeout)
        self.t0 = time.perf_counter()

    def mark(self):
        """The timed region starts now (samples before it are not summarised)."""
        self.t0 = time.perf_counter()

    def stop(self):
        if self.p is None:
            return None
        t1 = time.perf_counter()
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.th.join(timeout=5)
        # samples taken inside the timed region (plus the last one before it, for short regions)
        inside = [ln for ts, ln in self.lines if self.t0 is None or self.t0 <= ts <= t1 + 0.05]
        before = [ln for ts, ln in self.lines if self.t0 is not None and ts < self.t0][-1:]
        rows = [r.split(", ") for r in (before + inside)]
        rows = [r for r in rows if len(r) >= 8]
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][1]),
                "reasons": reasons, "samples": len(rows), "samples_inside_timed_region": len(inside)}


# ---------------------------------------------------------------------------------------------
# the CPU legs: the oracle port of the reference's path, timed on the host cores
# ---------------------------------------------------------------------------------------------
def cpu_batches(a, A0_csr, labels, lab, Z0, batches, budget_s):
    """Run the oracle over `batches` until the budget is spent; returns (updates/s, batches done, cores)."""
    from oracle import edge_cpu
    st = edge_cpu.EdgeSolverCPU(A0_csr, labels, lab, a.k, Z0, target_relres=a.target_relres)
    t0 = time.perf_counter()
    done, t_work = 0, 0.0
    for b in batches:
        t = time.perf_counter()
        st.step(b)
        t_work += time.perf_counter() - t
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    return done * a.batch / t_work, done, t_work


def reference_arm(a):
    """--impl reference: the oracle port of the reference's path on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from dynlplus_b200 import graphs
    from oracle import edge_cpu
    import torch
    ds = graphs.er_graph(a.n, a.deg, a.k, seed=a.seed, device="cpu")
    lab = graphs.label_mask(a.n, a.label_frac, seed=a.seed, device="cpu").numpy()
    A = ds.A.to_scipy()
    y = ds.y.numpy()
    up = graphs.EdgeUpdates(ds.A, seed=a.seed)
    Z0 = edge_cpu.static_solve(A, y, lab, a.k, a.target_relres)
    batches = [up.next(a.batch) for _ in range(max(a.warmup, 0) + a.steps)]
    st = edge_cpu.EdgeSolverCPU(A, y, lab, a.k, Z0, target_relres=a.target_relres)
    for b in batches[: min(a.warmup, 1)]:
        st.step(b)
    t0 = time.perf_counter()
    times = []
    for b in batches[a.warmup:]:
        t = time.perf_counter()
        st.step(b)
        times.append(time.perf_counter() - t)
        if time.perf_counter() - t0 > a.cpu_budget_s:
            break
    value = len(times) * a.batch / sum(times)
    cores = CPU_PORT_THREADS
    sample = (f"{len(times)} of {a.steps} requested batches of {a.batch} updates on the full graph "
              f"(timed budget {a.cpu_budget_s:g} s); {CPU_PORT_NOTE}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "edge-updates/s", "n_gpus": a.gpus,
            "steps": len(times), "steps_requested": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(a),
            "cpu_baseline": {"value": value, "unit": "edge-updates/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "edge-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "latency_ms": {"p50": 1e3 * float(np.percentile(times, 50)), "p99": 1e3 * float(np.percentile(times, 99))}}
    print(json.dumps(line), flush=True)
    del torch
    return 0


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------
def spmm_roofline(es, C, peaks):
    """Average duration of the SpMM (apply_A form, the PCG's dominant kernel) on the stream's
    operator with CUDA events on the launching stream, and its algorithmic bytes per launch."""
    import torch
    from dynlplus_b200 import _lib, kernels, solvers
    G = es.solver_csr()  # the operator the PCG iterates on (live entries of W_UU)
    n = es.n
    X = solvers.padded_empty(n, C, torch.float32, es.dev)
    X.copy_(torch.rand((n, C), device=es.dev))
    a = es.diag32
    Y = solvers.padded_empty(n, C, torch.float32, es.dev)  # 16-byte rows: whole-row stores, as the PCG's AP
    for _ in range(3):
        kernels.spmm_axpy(G, X, a=a, b=-1.0, out=Y)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=es.dev)
    reps = 20
    cold = []
    for _ in range(reps):  # after an L2 flush
        flush.fill_(1.0)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        kernels.spmm_axpy(G, X, a=a, b=-1.0, out=Y)
        e.record()
        e.synchronize()
        cold.append(s.elapsed_time(e))
    # back to back, as inside the PCG iteration (the operand was written by the previous kernel)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        kernels.spmm_axpy(G, X, a=a, b=-1.0, out=Y)
    e.record()
    e.synchronize()
    ms = s.elapsed_time(e) / reps
    nnz = G.nnz
    sx = 4
    # gather model of the reference's kernel benchmark, extended with the row pointers, the a-term
    # read and the output write: 4(n+1) + nnz (4 + s_w + C s_x) + n s_a + n C s_x + n C s_y
    algo = 4 * (n + 1) + nnz * (4 + 4 + C * sx) + n * 4 + n * C * sx + n * C * 4
    achieved = algo / (ms * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs") or 6650.0
    # the same product with the gathered rows and the weights in bf16 (fp32 accumulation, fp32 own
    # row and output; dlp_spmm_lowp, the SpMM of the BF16 sweeps): 4(n+1) + nnz (4 + 2 + 2C) + n s_a
    # + n C 4 (own row) + n C 4 (output)
    from dynlplus_b200.backend import ld as _ld, ptr as _ptr, stream as _stream
    wb = solvers.bf16_weights(G)
    Xb = solvers.padded_empty(n, C, torch.bfloat16, es.dev)
    Xb.copy_(X)

    def lowp():
        _lib.call("dlp_spmm_lowp", _ptr(G.rbeg), _ptr(G.rend), _ptr(G.indices), _ptr(wb), n, C, _ptr(Xb), _ld(Xb),
                  _ptr(X), _ld(X), _ptr(a), 1.0, -1.0, _ptr(Y), _ld(Y), 0, G.nnz / max(n, 1), _stream())

    for _ in range(3):
        lowp()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        lowp()
    e.record()
    e.synchronize()
    ms_lo = s.elapsed_time(e) / reps
    algo_lo = 4 * (n + 1) + nnz * (4 + 2 + C * 2) + n * 4 + n * C * 4 + n * C * 4
    bf16 = {"kernel": "dlp_spmm_lowp (k_spmm, apply_A form, bf16 weights and gathered rows, fp32 accumulation, own row "
                      "and output, C=%d, ld=%d)" % (C, Xb.stride(0)),
            "achieved": algo_lo / (ms_lo * 1e-3) / 1e9, "frac": algo_lo / (ms_lo * 1e-3) / 1e9 / (peaks.get("hbm_gbs") or 6650.0),
            "algorithmic_bytes": int(algo_lo), "ms_per_launch": ms_lo}
    return {"bound": "hbm", "kernel": "k_spmm (apply_A form, fp32, C=%d, ld=%d for X and Y, compact CSR of W_UU)" % (C, X.stride(0)),
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks.get("hbm_gbs") else "fallback",
            "algorithmic_bytes": int(algo), "ms_per_launch": ms, "ms_per_launch_after_l2_flush": float(np.mean(cold)),
            "achieved_after_l2_flush": algo / (float(np.mean(cold)) * 1e-3) / 1e9, "traffic": None,
            "note": "gather model counts every neighbour-row gather as HBM bytes; on this graph the "
                    "gathered matrix (n x ld x 4 B) fits in L2", "bf16": bf16}


def aggregate_replicas(dev_ms, e2e_ms, units_per_step, world, device="cpu"):
    """Whole-job throughput of `world` independent replicas (one per rank): the slowest rank's summed
    step times (max over ranks, on the device) against all ranks' units. Every rank takes the same
    collective steps. Returns (t_dev_ms, t_e2e_ms, value, e2e) with value, e2e in units per second."""
    import torch
    total = torch.tensor([float(sum(dev_ms)), float(sum(e2e_ms))], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
        dist.barrier()
    t_dev, t_e2e = float(total[0]), float(total[1])
    value = world * units_per_step * len(dev_ms) / (t_dev * 1e-3)
    e2e = world * units_per_step * len(e2e_ms) / (t_e2e * 1e-3) if e2e_ms else float("nan")
    return t_dev, t_e2e, value, e2e


def pcg_iteration_bytes(n, nnz, C, s=4):
    """Algorithmic bytes of one fused PCG iteration on an n-row operator with nnz entries and C
    columns of s-byte values, the byte model of the hot-path measurement spec: the SpMM by the gather
    model, B_spmm = 4 (n + 1) + nnz (4 + s_w + C s) + n C s (AP written) + n s (diag) + n C s (own row
    of P), plus 6 n C s (R, P and Z read and written) and n s (diag). The implementation moves more
    (AP is read back by the residual update and R twice; its three kernels are separate passes), so
    this is the floor its time is measured against."""
    spmm = 4 * (n + 1) + nnz * (4 + 4 + C * s) + n * C * s + n * s + n * C * s
    return spmm + 6 * n * C * s + n * s


def pcg_steady(es, C, iters=100):
    """The PCG iteration in steady state on the stream's final system with the C columns of the timed
    solves: one dlp_pcg call from zero that runs `iters` iterations to its cap (a target it cannot
    meet), timed with CUDA events on the launching stream, so the per-call start and host reads
    weigh 1/iters of it."""
    import torch
    from dynlplus_b200 import solvers
    S = es.system.astype(torch.float32)
    rhs = S.rhs_h.to(torch.float32)
    if C < rhs.shape[1]:  # the class-sum corrections: all class columns but the last, and h
        k = rhs.shape[1] - 1
        rhs = torch.cat([rhs[:, : k - 1], rhs[:, k:]], dim=1)
    rhs = rhs.contiguous()
    Z = solvers.padded_empty(rhs.shape[0], rhs.shape[1], torch.float32, rhs.device, fill=0.0)
    rn = [1.0] * rhs.shape[1]
    ev, solvers.PCG_EVENTS = solvers.PCG_EVENTS, None
    try:
        for _ in range(2):  # the first call captures the loop graph
            st = solvers.Stats()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s.record()
            solvers.pcg(S, Z, rhs, None, solvers.jacobi_M(S), iters, st, target_relres=1e-30, rhs_norm=rn,
                        zero_start=True)
            e.record()
            e.synchronize()
    finally:
        solvers.PCG_EVENTS = ev
    return s.elapsed_time(e) / max(st.iters, 1), st.iters


def pcg_roofline(events, nnz, peaks, traffic_file, steady=None):
    """The fused PCG iteration (k_pcg_apply + k_pcg_update + k_pcg_dir), timed live: CUDA events
    around every dlp_pcg call of the timed steps (on the launching stream); time per iteration =
    the calls' total device time / their iterations (so it also carries each call's start, stop
    checks and recheck, a conservative figure). steady: (ms per iteration, iterations) of
    pcg_steady, reported beside it."""
    from dynlplus_b200 import solvers
    ms = sum(s.elapsed_time(e) for s, e, _, _, _ in events)
    iters = sum(it for _, _, it, _, _ in events)
    if not iters:
        return None
    n, C = events[0][3], events[0][4]
    algo = pcg_iteration_bytes(n, nnz, C)
    t = ms / iters
    achieved = algo / (t * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs") or 6650.0
    traffic, tsrc = None, None
    if os.path.exists(traffic_file):
        tr = json.load(open(traffic_file))
        if tr.get("n") == n and tr.get("C") == C and ("k_pcg_fused" in tr.get("per_kernel", {})) == solvers.TWO_KERNEL:
            traffic, tsrc = tr.get("dram_bytes_per_iteration"), tr.get("source")
    # the sweep is one row per thread (k_pcg_fused_rows8) for rows of at most 8 floats on a 32-byte
    # pitch, else one element per thread (k_pcg_fused)
    sweep = "k_pcg_fused_rows8" if C <= 8 else "k_pcg_fused"
    ks = "k_pcg_apply + " + sweep if solvers.TWO_KERNEL else "k_pcg_apply + k_pcg_update + k_pcg_dir"
    return {"bound": "hbm", "kernel": "PCG iteration: %s (fp32, C=%d, compact CSR of W_UU, nnz=%d)" % (ks, C, nnz),
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks.get("hbm_gbs") else "fallback",
            "traffic": traffic, "traffic_source": tsrc, "algorithmic_bytes_per_iteration": int(algo),
            "ms_per_iteration": t, "iterations_timed": int(iters), "pcg_calls": len(events),
            "byte_model": "4(n+1) + nnz(4 + s_w + C s) + n C s (AP) + n s (diag) + n C s (own P) + 6 n C s + n s",
            "steady": None if steady is None else {
                "ms_per_iteration": steady[0], "iterations": steady[1],
                "achieved": algo / (steady[0] * 1e-3) / 1e9, "frac": algo / (steady[0] * 1e-3) / 1e9 / peak,
                "note": "one dlp_pcg call of that many iterations on the final system, outside the timed steps"}}


def ours(a):
    import torch
    import torch.distributed as dist
    from dynlplus_b200 import _lib, graphs, solvers, stream

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))

    solvers.TWO_KERNEL = not a.three_kernel
    seed = a.seed + 1000 * rank  # independent replicas
    ds = graphs.er_graph(a.n, a.deg, a.k, seed=seed)
    lab = graphs.label_mask(a.n, a.label_frac, seed=seed)
    es = stream.EdgeStream(ds, lab, components=True)  # component ids after every batch (side stream)

    def make_solver():
        return solvers.IncrementalLP(a.n, a.k, "float32", tol=a.tol, method="pcg", target_relres=a.target_relres,
                                     full_every=16, lowp=a.lowp, class_sum=False if a.no_class_sum else "auto",
                                     refine_share=a.refine_share)

    solver = make_solver()
    solver.solve(es.system)  # the static solve of the initial graph (untimed)
    A0 = ds.A.to_scipy() if (rank == 0 and not a.no_cpu_baseline) else None
    Z0 = solver.Z.cpu().numpy() if A0 is not None else None
    up = graphs.EdgeUpdates(ds.A, seed=seed)
    nb = a.warmup + 2 * a.steps
    batches = [up.next(a.batch) for _ in range(nb)]
    cpu_sample = [up.next(a.batch) for _ in range(2)] if A0 is not None else None
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def to_dev(b):
        return {k: torch.from_numpy(v).to(dev) for k, v in b.items()}

    def to_pinned(b):
        return {k: torch.from_numpy(v).pin_memory() for k, v in b.items()}

    # relabelled rows read back with the counts in one round trip: up to `cap` of them (a step that
    # relabels more reads the rest in a second one and doubles the buffers for the next steps)
    rb = {"cap": 65536}
    h_cnt = torch.zeros(3, dtype=torch.int32).pin_memory()
    rb["rows"] = torch.zeros(rb["cap"], dtype=torch.int32).pin_memory()
    rb["labs"] = torch.zeros(rb["cap"], dtype=torch.int32).pin_memory()
    d2h = []

    def step(b, host_result=False):
        """One batch: patch, grounding, component ids (side stream), solve, labels. With host_result
        the step's result comes back to the host: the number of relabelled rows, the component and
        active-unlabelled counts, and every relabelled row with its new label."""
        S = es.apply_edges(**b)
        st = solver.solve(S)
        _, chg, chg_lab, nchg = solver.relabel(S)
        es.join_components()
        if not host_result:
            return st, None
        cap, h_rows, h_labs = rb["cap"], rb["rows"], rb["labs"]
        m = min(cap, int(chg.numel()))
        h_cnt[0:1].copy_(nchg, non_blocking=True)
        h_cnt[1:3].copy_(es._cc_counts[0:2], non_blocking=True)
        h_rows[:m].copy_(chg[:m], non_blocking=True)
        h_labs[:m].copy_(chg_lab[:m], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        k = int(h_cnt[0])
        nbytes = 12 + 8 * m
        rows, labs = h_rows[:min(k, m)].numpy().copy(), h_labs[:min(k, m)].numpy().copy()
        if k > m:
            rows = np.concatenate([rows, chg[m:k].cpu().numpy()])
            labs = np.concatenate([labs, chg_lab[m:k].cpu().numpy()])
            nbytes += 8 * (k - m)
            while rb["cap"] < k:
                rb["cap"] *= 2
            rb["rows"] = torch.zeros(rb["cap"], dtype=torch.int32).pin_memory()
            rb["labs"] = torch.zeros(rb["cap"], dtype=torch.int32).pin_memory()
        d2h.append(nbytes)
        return st, (k, int(h_cnt[1]), int(h_cnt[2]), rows, labs)

    fstar = {}

    def check_fp64(S, solver):
        """The solver's scores for system S against an fp64 solve of S (fp64 block PCG to a relative
        residual of 1e-11, started from the previous batch's fp64 solution): the score error relative
        to the largest score, label agreement and near-ties (rows whose two best fp64 scores differ
        by at most twice the score error)."""
        S64 = S.astype(torch.float64)
        C = solver.C
        Zs = fstar.get("Z")
        if Zs is None:
            Zs = solvers.padded_empty(a.n, C, torch.float64, dev, fill=0.0)
        st = solvers.Stats()
        rhs = S64.rhs.contiguous()
        ev, solvers.PCG_EVENTS = solvers.PCG_EVENTS, None  # not part of the timed PCG calls
        solvers.pcg(S64, Zs, rhs, None, solvers.jacobi_M(S64), 10_000, st, target_relres=1e-11)
        solvers.PCG_EVENTS = ev
        fstar["Z"] = Zs
        U = S.solved
        F, Fs = solver.Z[:, :C][U], Zs[U]
        err = float((F - Fs).abs().max())
        scale = float(Fs.abs().max())
        labels = solver._labels[U]
        want = Fs.argmax(dim=1).to(torch.int32) if C > 1 else (Fs[:, 0] > 0.5).to(torch.int32)
        if C > 1:
            top = torch.topk(Fs, 2, dim=1).values
            tie = top[:, 0] - top[:, 1] <= 2 * err
        else:
            tie = (Fs[:, 0] - 0.5).abs() <= err
        bad = labels != want
        return {"err": err / scale, "agree": float(1.0 - bad.double().mean()), "near_ties": int(tie.sum()),
                "mismatch_outside_ties": int((bad & ~tie).sum()), "fp64_iters": st.iters, "fp64_relres": st.relres}

    dev_batches = [to_dev(b) for b in batches[a.warmup: a.warmup + a.steps]]
    host_batches = [to_pinned(b) for b in batches[a.warmup + a.steps:]]
    # the clock sampler starts before the warm-up, so the timed steps follow the last warm-up step
    # directly (an idle gap before them would let the clocks drop)
    clocks = Clocks(torch.cuda.current_device()) if not a.no_clocks else None
    if clocks is not None:
        clocks.wait_first()
    # warm-up (not timed)
    for b in batches[: a.warmup]:
        step(to_dev(b))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    if clocks is not None:
        clocks.mark()
    launches0 = _lib.lib().dlp_launch_count()
    solvers.PCG_EVENTS = []  # CUDA events around the fused PCG calls of the timed steps
    # Python's cyclic collector: run once now and paused through the timed loops (as a serving
    # process would tune it), so a collection pass does not land inside one step
    gc.collect()
    gc.disable()
    torch.cuda.nvtx.range_push("timed")  # lets a profiler filter the timed steps (--nvtx-include timed/)
    times, relres, paths, iters, events, checks = [], [], [], [], {}, []
    for k, b in enumerate(dev_batches):
        c0 = dict(es.counters)
        flush.fill_(0.0)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        st, _ = step(b)
        e.record()
        e.synchronize()
        times.append(s.elapsed_time(e))
        relres.append(st.relres)
        paths.append(st.path)
        iters.append(st.iters)
        ev = {c: es.counters[c] - c0[c] for c in ("rebuilds", "ground_fallbacks") if es.counters[c] != c0[c]}
        if ev:
            events[k] = ev
    launches = _lib.lib().dlp_launch_count() - launches0
    torch.cuda.nvtx.range_pop()
    pcg_events, solvers.PCG_EVENTS = solvers.PCG_EVENTS, None
    # end to end: host arrays in, host result out (the clock sampling covers this region too)
    e2e_times = []
    h2d = sum(v.numel() * v.element_size() for v in host_batches[0].values()) if host_batches else 0
    relabelled, res = [], None
    for b in host_batches:
        flush.fill_(0.0)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        st, res = step(b, host_result=True)
        e.record()
        e.synchronize()
        e2e_times.append(s.elapsed_time(e))
        relres.append(st.relres)
        relabelled.append(res[0])
    gc.enable()
    cc_last = res[1:3] if res is not None else None
    clk = clocks.stop() if clocks else None
    if rank == 0 and not a.no_fp64_check:
        # after the timed loops (nothing runs between timed steps): a second resident stream and
        # solver replay the warm-up and timed batches, and each timed batch's scores are checked
        # against an fp64 solve of its system, on a stream of their own
        check_stream = torch.cuda.Stream(device=dev)
        with torch.cuda.stream(check_stream):
            es_r, solver_r = stream.EdgeStream(ds, lab, components=True), make_solver()
            solver_r.solve(es_r.system)
            for i, b in enumerate(batches[: a.warmup + a.steps]):
                S = es_r.apply_edges(**to_dev(b))
                solver_r.solve(S)
                solver_r.relabel(S)
                es_r.join_components()
                if i >= a.warmup:
                    checks.append(check_fp64(es_r.system, solver_r))
        torch.cuda.synchronize()
        del es_r, solver_r
    t_dev, t_e2e, value, e2e = aggregate_replicas(times, e2e_times, a.batch, world, dev)
    roof = None
    if rank == 0:
        c_pcg = pcg_events[0][4] if pcg_events else a.k + 1  # columns the correction solves iterate on
        roof = pcg_roofline(pcg_events, es.solver_csr().nnz, peaks,
                            os.path.join(ROOT, "profiles", "pcg_iteration_traffic.json"),
                            steady=pcg_steady(es, c_pcg))
        if roof is not None:
            roof["spmm_alone"] = spmm_roofline(es, c_pcg, peaks)
            if c_pcg != a.k + 1:  # every class column and h (the static solve's width)
                roof["spmm_alone_all_columns"] = spmm_roofline(es, a.k + 1, peaks)
    cpu = None
    if rank == 0 and not a.no_cpu_baseline and world == 1:
        v, done, tw = cpu_batches(a, A0, ds.y.cpu().numpy(), lab.cpu().numpy(), Z0, cpu_sample, a.cpu_budget_s)
        cpu = {"value": v, "unit": "edge-updates/s", "cores": CPU_PORT_THREADS,
               "kind": "port", "sample": f"{done} batch(es) of {a.batch} updates on the full graph ({tw:.1f} s): "
                                         "oracle patch + system rebuild + fp64 Jacobi-PCG correction to the same "
                                         f"rel-res; {CPU_PORT_NOTE}"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "edge-updates/s", "n_gpus": world, "steps": len(times),
                "warmup": a.warmup, "ms_per_step": t_dev / len(times), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16" if a.lowp else "f32", "data": "synthetic", "config": config(a),
                "latency_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99)),
                               "e2e_p50": float(np.percentile(e2e_times, 50)),
                               "e2e_p99": float(np.percentile(e2e_times, 99))},
                "relres_max": float(max(relres)), "paths": sorted(set(paths)),
                "stream_events": {str(k): v for k, v in events.items()},
                "pcg_iters_per_batch": float(np.mean(iters)),
                "step_ms": [round(t, 3) for t in times],
                "e2e_step_ms": [round(t, 3) for t in e2e_times],
                "e2e": {"value": e2e, "unit": "edge-updates/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(np.mean(d2h)) if d2h else 0,
                        "result": "relabelled rows with their new labels; component and active-unlabelled counts",
                        "relabelled_rows_per_step": float(np.mean(relabelled)) if relabelled else None},
                "parity_vs_fp64": ({"err_vs_fp64_max": max(c["err"] for c in checks),
                                    "label_agree_min": min(c["agree"] for c in checks),
                                    "near_ties_max": max(c["near_ties"] for c in checks),
                                    "mismatch_outside_near_ties": sum(c["mismatch_outside_ties"] for c in checks),
                                    "batches": len(checks),
                                    "replay": "a second resident stream and solver over the warm-up and timed "
                                              "batches, after the timed loops",
                                    "reference": "fp64 block Jacobi-PCG of the same system to rel-res 1e-11"}
                                   if checks else None),
                "components": {"n_comp": cc_last[0], "label_free_vertices": cc_last[1] - es.system.n_solved}
                if cc_last else None,
                "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                "precision": ("bf16 gathers (fp32 accumulation)" if a.lowp else "fp32 sweeps (SpMM, PCG)") +
                             " with fp64 residual refinement, fp64 inner products"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------------------------
# the other workloads (one JSON line each; the driver's headline is edge-stream)
# ---------------------------------------------------------------------------------------------
def _line(a, metric, value, unit, ms, cfg, hib=True, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
         "ms_per_step": ms, "higher_is_better": hib, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
         "data": "synthetic", "config": cfg}
    d.update(extra)
    print(json.dumps(d), flush=True)


def _events(fn):
    import torch
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    out = fn()
    e.record()
    e.synchronize()
    return s.elapsed_time(e), out


def wl_static(a):
    """Config 1: SBM n=100,000 (4 blocks, degree 12 in + 4 cross, unit weights), 1% labelled, k=4:
    the static solve by Jacobi-PCG to rel-res 1e-6, then one batch of 1,000 edge updates."""
    import torch
    from dynlplus_b200 import graphs, solvers, stream
    ms_s, ms_u, rel = [], [], []
    for rep in range(a.warmup + a.steps):
        ds = graphs.planted_partition(100_000, 4, 12.0, 4.0, seed=rep)
        lab = graphs.label_mask(100_000, 0.01, seed=rep)
        es = stream.EdgeStream(ds, lab)
        solver = solvers.IncrementalLP(100_000, 4, "float32", tol=1e-3, method="pcg", target_relres=1e-6)
        b = graphs.EdgeUpdates(ds.A, seed=rep).next(1000)
        t0, st0 = _events(lambda: solver.solve(es.system))
        t1, st1 = _events(lambda: solver.solve(es.apply_edges(**b)))
        if rep >= a.warmup:
            ms_s.append(t0)
            ms_u.append(t1)
            rel.append(max(st0.relres, st1.relres))
    _line(a, "edge-updates/s of the 1,000-update batch after the static solve (rel-res 1e-6)",
          1000 / (np.mean(ms_u) * 1e-3), "edge-updates/s", float(np.mean(ms_s) + np.mean(ms_u)),
          {"workload": "sbm-n100000-b4-d12+4-unit-lab0.01-k4", "static_solve_ms": float(np.mean(ms_s)),
           "update_batch_ms": float(np.mean(ms_u)), "l2": "not flushed (fresh graph per repetition)"},
          relres_max=float(max(rel)))


def wl_amg(a):
    """Config 3: SBM n=1,000,000, 16 blocks, degree 24 in + 8 cross, lognormal(0, 0.5) weights,
    1% labelled, k=16: AMG-preconditioned block PCG with BF16 SpMM (bf16 weights and scores, fp32
    accumulation) and fp64 residual refinement to rel-res 1e-8, the loop on the device. Beside it,
    on the same system: fp32 sweeps with AMG and with the Jacobi preconditioner, each with its error
    against an fp64 solve (fp64 Jacobi-PCG to rel-res 1e-12), the hierarchy and one V-cycle's time."""
    import torch
    from dynlplus_b200 import amg as amg_mod
    from dynlplus_b200 import graphs, solvers, stream
    ds = graphs.planted_partition(1_000_000, 16, 24.0, 8.0, weights="lognormal", seed=3)
    lab = graphs.label_mask(1_000_000, 0.01, seed=3)
    S = stream.build_system(ds, torch.ones(ds.n, dtype=torch.bool, device="cuda"), lab, dtype="float32")
    S64 = S.astype(torch.float64)
    C = S.rhs.shape[1]
    Fs = torch.zeros((S.n_u, C), dtype=torch.float64, device="cuda")
    solvers.pcg(S64, Fs, S64.rhs.contiguous(), None, solvers.jacobi_M(S64), 100_000, solvers.Stats(),
                target_relres=1e-12)
    scale = float(Fs.abs().max())

    def run(method, lowp):
        times, st, solver = [], None, None
        for rep in range(a.warmup + a.steps):
            solver = solvers.DynLPPlus(ds.n, 16, "float32", method=method, tol=1e-3, target_relres=1e-8, lowp=lowp)
            t, st = _events(lambda: solver.solve(S))
            if rep >= a.warmup:
                times.append(t)
        err = float((solver.scores(S).double() - Fs).abs().max()) / scale
        return {"ms": float(np.mean(times)), "pcg_iters": st.iters, "relres": st.relres, "err_vs_fp64": err,
                "setup_ms": st.setup_ms}

    res = {"amg_bf16": run("amg", True), "amg_fp32": run("amg", False), "jacobi_fp32": run("pcg", False)}
    M = amg_mod.AMG(S.W, S.s)
    R = torch.randn((S.n_u, C + 1), dtype=torch.float32, device="cuda")
    for _ in range(3):
        M(R)
    t_cycle, _ = _events(lambda: [M(R) for _ in range(10)])
    head = res["amg_bf16"]
    _line(a, "AMG-PCG solve time to rel-res 1e-8 (BF16 SpMM, fp32 accumulation, fp64 refinement)", head["ms"], "ms",
          head["ms"], {"workload": "sbm-n1000000-b16-d24+8-lognormal-lab0.01-k16"}, hib=False,
          relres_max=head["relres"], err_vs_fp64=head["err_vs_fp64"], pcg_iters=head["pcg_iters"],
          amg_setup_ms=head["setup_ms"], variants=res, amg_levels=M.sizes, vcycle_ms=t_cycle / 10,
          precision="bf16 SpMM (weights and gathered scores) with fp32 accumulation in the CG, fp32 V-cycle, "
                    "fp64 refinement; error relative to the largest fp64 score")


def wl_batched(a):
    """Config 4: 256 SBM graphs, n log-uniform in [2,000, 200,000], blocks = k in {2,4,8}, mean degree
    U[8,24] (3:1 in:cross), unit weights, 1% labelled: all solves batched, rel-res 1e-6."""
    import torch
    from dynlplus_b200 import batched, graphs, stream
    rng = np.random.default_rng(4)
    systems = []
    for i in range(256):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(200_000))))
        k = int(rng.choice([2, 4, 8]))
        deg = float(rng.uniform(8, 24))
        ds = graphs.planted_partition(n, k, 0.75 * deg, 0.25 * deg, seed=1000 + i)
        lab = graphs.label_mask(n, 0.01, seed=1000 + i)
        systems.append(stream.build_system(ds, torch.ones(n, dtype=torch.bool, device="cuda"), lab, dtype="float32"))
    def timed(fn):
        times, info = [], None
        for rep in range(a.warmup + a.steps):
            t, (Fs, info) = _events(fn)
            if rep >= a.warmup:
                times.append(t)
        return float(np.mean(times)), info

    # two precisions on the same 256 systems: fp32 sweeps with fp64 refinement, and fp64 sweeps
    # (fp32 weights both); the faster is the headline, the other is reported beside it
    t_mix, info_mix = timed(lambda: batched.solve_many_mixed(systems, target_relres=1e-6, autotune=True))
    t64, info64 = timed(lambda: batched.solve_many(systems, target_relres=1e-6, dtype=torch.float64, autotune=True))
    rows = sum(s.n_u for s in systems)
    runs = {"fp32 sweeps + fp64 refinement": (t_mix, info_mix), "fp64 sweeps": (t64, info64)}
    head = min(runs, key=lambda k: runs[k][0])
    t, info = runs[head]

    def summary(t, info):
        return {"solves_per_s": 256 / (t * 1e-3), "ms": t, "relres_max": float(max(r for _, _, r in info)),
                "converged": int(sum(s == 5 for _, s, _ in info)),
                "iterations_total": int(sum(i for i, _, _ in info))}

    _line(a, "independent harmonic solves per second, 256 instances batched (rel-res 1e-6)",
          256 / (t * 1e-3), "solves/s", t,
          {"workload": "256x sbm n~logU[2e3,2e5] k in {2,4,8} deg~U[8,24] lab0.01", "rows": int(rows),
           "precision": head},
          relres_max=float(max(r for _, _, r in info)), converged=int(sum(s == 5 for _, s, _ in info)),
          iterations_total=int(sum(i for i, _, _ in info)), dtype="f64" if head == "fp64 sweeps" else "f32",
          variants={k: summary(*v) for k, v in runs.items()})


def wl_serving(a):
    """Config 5: resident SBM n=4,000,000, 32 blocks, degree 16 (12 in + 4 cross), lognormal weights,
    1% labelled, k=32; Poisson arrivals at `--rate`: 60% edge-update batches (size log-uniform in
    [10, 50,000]), 30% label queries (1 to 10,000 ids), 10% fresh solves (n log-uniform in
    [10,000, 500,000], k=32)."""
    import time as _t
    import torch
    from dynlplus_b200 import graphs, serve
    n = 4_000_000
    ds = graphs.planted_partition(n, 32, 12.0, 4.0, weights="lognormal", seed=5)
    lab = graphs.label_mask(n, 0.01, seed=5)
    up = graphs.EdgeUpdates(ds.A, seed=5, weights="lognormal")
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(a.requests):
        u = rng.random()
        if u < 0.6:
            b = up.next(int(np.exp(rng.uniform(np.log(10), np.log(50_000)))))
            reqs.append(serve.EdgeUpdate(b["ins_u"], b["ins_v"], b["ins_w"], b["del_u"], b["del_v"]))
        elif u < 0.9:
            reqs.append(serve.LabelQuery(rng.integers(0, n, int(rng.integers(1, 10_001)))))
        else:
            m = int(np.exp(rng.uniform(np.log(10_000), np.log(500_000))))
            reqs.append(serve.FreshSolve(graphs.planted_partition(m, 32, 12.0, 4.0, weights="lognormal", seed=i),
                                         graphs.label_mask(m, 0.01, seed=i)))
    gaps = rng.exponential(1.0 / a.rate, len(reqs))
    updates = sum(r.size for r in reqs if isinstance(r, serve.EdgeUpdate))

    def run(mode, lowp, precision=None):
        srv = serve.Server(ds, lab, target_relres=1e-6, mode=mode, lowp=lowp, precision=precision)
        t0 = _t.perf_counter()
        futs = []
        for r, g in zip(reqs, gaps):
            _t.sleep(g)
            futs.append(srv.submit(r))
        res = [f.result(timeout=1200) for f in futs]
        wall = _t.perf_counter() - t0
        lat = {k: srv.latency(k) for k in ("update", "query", "fresh")}
        srv.close()
        rel = max([x["relres"] for x in res if isinstance(x, dict) and "relres" in x] + [0.0])
        return {"edge_updates_per_s": updates / wall, "requests_per_s": len(reqs) / wall, "wall_s": wall,
                "latency_ms": lat, "relres_max": float(rel)}

    # the plain FP32 path served one request at a time, the mixed-precision solvers one request at a
    # time, then the continuous-batching loop with FP32 and with BF16 sweeps (the same request trace
    # and arrival times for all four)
    seq = run("sequential", False)
    seq_mixed = run("sequential", False, "mixed")
    cont = run("continuous", False)
    cont_bf16 = run("continuous", True)
    best = max((cont, cont_bf16), key=lambda r: r["edge_updates_per_s"])
    p99 = lambda r: r["latency_ms"]["update"]["p99_ms"]  # noqa: E731
    _line(a, "served edge-updates/s under mixed Poisson load (p50/p99 per request kind)", best["edge_updates_per_s"],
          "edge-updates/s", 1e3 * best["wall_s"] / len(reqs),
          {"workload": "serving sbm-n4000000-b32-d12+4-lognormal-lab0.01-k32", "rate_req_s": a.rate,
           "requests": len(reqs), "headline": "continuous" + ("+bf16" if best is cont_bf16 else "")},
          latency_ms=best["latency_ms"], requests_per_s=best["requests_per_s"],
          modes={"sequential_fp32": seq, "sequential_mixed": seq_mixed, "continuous_fp32": cont,
                 "continuous_bf16": cont_bf16},
          speedup_vs_sequential={"edge_updates_per_s": best["edge_updates_per_s"] / seq["edge_updates_per_s"],
                                 "update_p99": p99(seq) / p99(best)},
          speedup_vs_sequential_mixed={"edge_updates_per_s": best["edge_updates_per_s"] /
                                       seq_mixed["edge_updates_per_s"], "update_p99": p99(seq_mixed) / p99(best)})


def wl_kernels(a):
    """The row kernels one by one on the headline graph (ER n=1M, mean degree 10, k=8 plus the h
    column) after one batch of updates, each timed alone with CUDA events on its launching stream
    after an L2 flush, against its algorithmic bytes:
      spmm             the apply_A SpMM over all rows (fp32, the PCG's gather);
      frontier_jacobi  the batch's changed rows (fp32): 12 nf + e (8 + 4C) + nf (12C + 5);
      push_fp64 / _fp32  the residual push from the batch's residual to eps = tol / (1.25 hmax) (the
                       incremental solver's small-batch branch), the whole dlp_fused_push call:
                       per frontier row 12 + 2C s_r + 2C s_z + s_d, per live entry 8 + s_w + 2C s_r,
                       per touched row 8 + C s_r + s_d."""
    import ctypes as ct
    import torch
    from dynlplus_b200 import _lib, graphs, kernels, solvers, stream
    from dynlplus_b200.backend import code, ld, ptr
    from dynlplus_b200.backend import stream as cur_stream
    dev = torch.device("cuda", torch.cuda.current_device())
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs") or 6650.0
    ds = graphs.er_graph(a.n, a.deg, a.k, seed=a.seed)
    lab = graphs.label_mask(a.n, a.label_frac, seed=a.seed)
    es = stream.EdgeStream(ds, lab)
    solver = solvers.IncrementalLP(a.n, a.k, "float32", tol=a.tol, method="pcg", target_relres=a.target_relres)
    solver.solve(es.system)
    Zprev = solver.Z.clone()
    S = es.apply_edges(**graphs.EdgeUpdates(ds.A, seed=a.seed).next(a.batch))
    C = solver.C + 1
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def timed(fn, reps):
        ms = []
        for _ in range(reps):
            flush.fill_(1.0)
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s0.record()
            fn()
            s1.record()
            s1.synchronize()
            ms.append(s0.elapsed_time(s1))
        return float(np.median(ms))

    def line(name, algo, ms, **extra):
        gbs = algo / (ms * 1e-3) / 1e9
        return {"kernel": name, "algorithmic_bytes": int(algo), "ms": ms, "achieved_gbs": gbs, "peak_gbs": peak,
                "frac": gbs / peak, **extra}

    out = {"spmm": spmm_roofline(es, C, peaks)}
    # frontier Jacobi over the batch's changed rows
    W = es.solver_csr()
    f = S.changed.to(torch.int32).contiguous()
    nf = int(f.numel())
    rows = f.long()
    e_f = int((W.indptr[1:][rows] - W.indptr[:-1][rows]).sum())
    X = solvers.padded_empty(a.n, C, torch.float32, dev)
    X.copy_(solver.Z[:, :C])
    rhs = S.rhs_h
    Y = torch.empty((max(nf, 1), C), dtype=torch.float32, device=dev)
    ch = torch.empty(max(nf, 1), dtype=torch.uint8, device=dev)

    def jac():
        _lib.call("dlp_frontier_jacobi", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(W.data), code(W.data), ptr(f),
                  nf, C, ptr(X), ld(X), ptr(rhs), ld(rhs), ptr(S.diag), 1e-4, ptr(Y), ld(Y), code(X), ptr(ch), None,
                  None, 0, W.nnz / a.n, cur_stream())
    for _ in range(3):
        jac()
    algo = 12 * nf + e_f * (8 + 4 * C) + nf * (12 * C + 5)
    out["frontier_jacobi"] = line("k_frontier_jacobi", algo, timed(jac, 20), rows=nf, entries=e_f)
    # the push from the batch's residual
    s64 = S.astype(torch.float64)
    hmax = solver.hmax or 1.0
    eps = [a.tol / (1.25 * hmax)] * solver.C + [solver.eps_h]
    for name, dt in (("push_fp64", torch.float64), ("push_fp32", torch.float32)):
        sw = S.astype(dt)
        diag = sw.diag.to(dt)
        rhs_d = (s64.rhs_h if dt == torch.float64 else S.rhs_h).to(dt)
        Z0 = solvers.padded_empty(a.n, C, dt, dev)
        R0 = solvers.padded_empty(a.n, C, dt, dev)
        Z0.copy_(Zprev[:, :C])
        R0.copy_(solvers.residual(s64, Zprev, s64.rhs_h))
        Z, R = solvers.padded_empty(a.n, C, dt, dev), solvers.padded_empty(a.n, C, dt, dev)
        eps_d = torch.as_tensor(eps, dtype=torch.float64, device=dev)
        cand = kernels.flatnonzero(kernels.violating(R0, diag, eps_d))
        fp = kernels.FusedPush(W, C)
        res = {}

        def push():
            Z.copy_(Z0)
            R.copy_(R0)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            res["run"] = fp.run(Z, R, diag, eps, cand, 100_000)
            ev1.record()
            ev1.synchronize()
            res["ms"] = ev0.elapsed_time(ev1)
        push()
        ms = []
        for _ in range(5):
            flush.fill_(1.0)
            push()
            ms.append(res["ms"])
        rounds, ok, edges = res["run"]
        _, frows, trows, _ = fp.counts()
        sz = 8 if dt == torch.float64 else 4
        algo = frows * (12 + 4 * C * sz + 4) + edges * (8 + 4 + 2 * C * sz) + trows * (8 + C * sz + sz)
        out[name] = line("k_push_scatter + k_push_sift (whole dlp_fused_push call)", algo, float(np.median(ms)),
                         rounds=rounds, converged=ok, candidates=int(cand.numel()), frontier_rows=frows,
                         touched_rows=trows, entries=edges)
    del ct
    _line(a, "row kernels on the headline graph: achieved HBM GB/s per kernel (CUDA events, after an L2 flush)",
          out["spmm"]["achieved_after_l2_flush"], "GB/s", out["spmm"]["ms_per_launch_after_l2_flush"],
          {"workload": workload_name(a), "frontier": "the changed rows of one batch of %d updates" % a.batch},
          kernels=out)


def main(argv=None):
    a = parse(argv)
    if a.no_graphs:
        from dynlplus_b200 import solvers
        solvers.GRAPHS = False
    if a.impl == "reference":
        return reference_arm(a)
    if a.workload != "edge-stream":
        return {"static": wl_static, "amg": wl_amg, "batched": wl_batched, "serving": wl_serving,
                "kernels": wl_kernels}[a.workload](a) or 0
    return ours(a)


if __name__ == "__main__":
    sys.exit(main())

"""Times the REFERENCE's own code on the host cores for the edge-stream workload (MEASUREMENT
INFRASTRUCTURE, not product code).

    python oracle/time_reference.py --reference <reference checkout> [--n 1000000 --batches 3]

The reference (shishir9159/DynLPlus) is pure Python over CuPy; tests/golden/cupy_shim.py maps CuPy
onto NumPy/SciPy so its modules run unchanged on the CPU. The reference has no edge-update API, so
per batch of edge updates this script

1. patches the adjacency with the oracle's edge patch (ref_np.apply_edges; timed apart),
2. runs the reference's `Stream._build` on the updated graph (dynlp/stream.py:142-177: the
   grounding by connected components and the U x U system), and
3. runs the reference's `DynLPPlus.solve` (dynlp/solvers.py:301-343, Jacobi-PCG, float32 sweeps with
   float64 certification) warm-started from the previous batch's scores, at the certified
   tolerance `--tol`,

then reports the reference's time per batch, the relative residual its answer reaches in fp64
(max_c ||rhs_c - A F_c|| / ||rhs_c||), and, on the same batches, the oracle port that bench.py's CPU
legs run (oracle/edge_cpu.py, fp64 Jacobi-PCG to the relative residual target). It needs the
reference checkout, so it runs where the reference is, not on a machine that only has this
repository. Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _relres(W, diag, rhs, F):
    R = rhs - (diag[:, None] * F - W @ F)
    rn = np.sqrt((rhs * rhs).sum(axis=0))
    return float((np.sqrt((R * R).sum(axis=0)) / np.where(rn > 0, rn, 1.0)).max())


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--reference", default=os.environ.get("DLP_REFERENCE"),
                    help="the reference checkout (default: $DLP_REFERENCE)")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--deg", type=float, default=10.0)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--label-frac", type=float, default=0.005)
    ap.add_argument("--batch", type=int, default=10_000)
    ap.add_argument("--batches", type=int, default=3)
    ap.add_argument("--tol", type=float, nargs="+", default=[1e-3, 1e-6],
                    help="certified tolerances of the reference's DynLPPlus (one run each)")
    ap.add_argument("--target-relres", type=float, default=1e-6, help="the oracle port's stop rule")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--no-port", action="store_true")
    a = ap.parse_args(argv)
    if not a.reference:
        ap.error("--reference (or DLP_REFERENCE) names the reference checkout")

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import cupy_shim  # noqa: E402
    from dynlplus_b200 import graphs  # noqa: E402  (workload generators, CPU tensors)
    from oracle import edge_cpu  # noqa: E402
    from oracle import ref_np as O  # noqa: E402

    sys.modules.pop("dynlp", None)  # this repository's alias package must not shadow the reference
    cupy_shim.install(a.reference)
    import dynlp.graphs as RG  # noqa: E402
    import dynlp.solvers as RS  # noqa: E402
    import dynlp.stream as RST  # noqa: E402

    ds = graphs.er_graph(a.n, a.deg, a.k, seed=a.seed, device="cpu")
    lab = graphs.label_mask(a.n, a.label_frac, seed=a.seed, device="cpu").numpy()
    y = ds.y.numpy().astype(np.int32)
    A0 = ds.A.to_scipy().astype(np.float64).tocsr()
    up = graphs.EdgeUpdates(ds.A, seed=a.seed)
    batches = [up.next(a.batch) for _ in range(a.batches)]
    n, K = a.n, a.k

    def ref_stream(A32):
        """A reference Stream over a fixed graph: the attributes Stream._build reads
        (dynlp/stream.py:89-128 sets them; the schedule is not needed for an edge batch)."""
        S = object.__new__(RST.Stream)
        S.ds = RG.Dataset("er", A32, y, K, np.arange(n, dtype=np.int64))
        S.dtype, S.labeled, S.y = "float32", lab, y
        S.rows = RG.csr_rows(A32)
        S.tau, S.wmax = float(A32.data.mean()), float(A32.data.max())
        S.eta = 0.0
        S.prior = np.full(1 if K == 2 else K, 0.5 if K == 2 else 1.0 / K, dtype="float32")
        return S

    def as32(A):
        A32 = A.astype(np.float32).tocsr()
        A32.indices = A32.indices.astype(np.int32)
        A32.indptr = A32.indptr.astype(np.int32)
        return A32

    none = np.zeros(0, dtype=np.int64)
    active = np.ones(n, dtype=bool)
    runs = []
    for tol in a.tol:
        solver = RS.DynLPPlus(n, K, "float32", method="pcg", tol=tol)
        A = A0
        t = time.perf_counter()
        sys0 = ref_stream(as32(A))._build(0, active, np.zeros(n, dtype=bool), none, none)
        solver.solve(sys0)
        t_static = time.perf_counter() - t
        prevU = np.zeros(n, dtype=bool)
        prevU[sys0.U] = True
        per, rels, iters, patch = [], [], [], []
        for i, b in enumerate(batches):
            t = time.perf_counter()
            A = O.apply_edges(A, b["ins_u"], b["ins_v"], b["ins_w"].astype(np.float64), b["del_u"], b["del_v"])
            A32 = as32(A)
            patch.append(time.perf_counter() - t)
            t = time.perf_counter()
            s = ref_stream(A32)._build(i + 1, active, prevU, none, none)
            st = solver.solve(s)
            per.append(time.perf_counter() - t)
            prevU = np.zeros(n, dtype=bool)
            prevU[s.U] = True
            s64 = s.astype(np.float64)
            F = solver.scores(s).astype(np.float64)
            rels.append(_relres(s64.W, s64.diag, s64.rhs, F))
            iters.append(int(st.iters))
        runs.append({"tol": tol, "static_s": t_static, "s_per_batch": per, "patch_s_per_batch": patch,
                     "edge_updates_per_s": a.batch * len(per) / sum(per), "relres": rels, "iterations": iters})

    port = None
    if not a.no_port:
        Z0 = edge_cpu.static_solve(A0, y, lab, K, a.target_relres)
        es = edge_cpu.EdgeSolverCPU(A0, y, lab, K, Z0, target_relres=a.target_relres)
        per = []
        for b in batches:
            t = time.perf_counter()
            es.step(b)
            per.append(time.perf_counter() - t)
        port = {"s_per_batch": per, "edge_updates_per_s": a.batch * len(per) / sum(per),
                "target_relres": a.target_relres}
    out = {"workload": f"er-n{n}-d{a.deg:g}-k{K}-lab{a.label_frac:g}, {a.batches} batches of {a.batch} updates",
           "cores": 1, "reference_dynlpplus_pcg": runs, "oracle_port": port}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Streaming benchmark with the reference's reporting (mirrors dynlp/bench.py): run solvers over a
vertex-arrival batch stream, score them against the fp64 reference solution F*, and write the
reference's CSV rows (same FIELDS, same meaning) plus a JSON sidecar with the arguments and the
environment, so B200 runs compare row for row with the reference's results files.

  python -m dynlplus_b200.bench --dataset er --n 1000000 --deg 5 --init-frac 1 --batches 0 \\
      --solvers itlp,dynlp,dynlp+pcg,dynlp+amg,dynlp+auto --out results/er1m.csv
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import os
import platform
import sys as _sys
import time

import torch

from . import graphs
from .backend import Timer, mem_used_gb, sync
from .solvers import SOLVERS, Reference, make, predict, residual, rho_cols
from .stream import IncrementalStream, Stream

# (flag, type, default, help); type None = a switch. The reference's flags (dynlp/bench.py:22-33).
ARGS = [
    ("--dataset", str, "sbm", "sbm | er | synth2 | synth10 | path/to/graph.npz (imdb is not built here)"),
    ("--n", int, 100_000, "sbm/er size"), ("--classes", int, 2, "sbm/er classes"), ("--deg", float, 10.0, None),
    ("--p-in", float, 0.85, "SBM: fraction of intra-class edges"),
    ("--data-dir", str, graphs.DATA_DIR, "graph caches (synthN); default: $DATA_DIR or ./data"),
    ("--label-frac", float, 0.01, None), ("--init-frac", float, 0.1, None), ("--batches", int, 10, None),
    ("--del-frac", float, 0.1, None), ("--eta-rel", float, 0.0, "grounding regulariser (x mean degree)"),
    ("--incremental", None, False, "keep the batch system resident (needed by dynlp+inc)"),
    ("--solvers", str, "dynlp,dynlp-fh,dynlp+auto", ",".join(SOLVERS)),
    ("--delta", float, 1e-4, "DynLP/ItLP change threshold"), ("--tol", float, 1e-3, "certified max error"),
    ("--group", str, "auto", "lanes per row for the frontier kernels (1..32)"),
    ("--dtype", str, "float32", None), ("--max-iter", int, None, None),
    ("--no-reference", None, False, "skip F* (no error columns)"), ("--seed", int, 0, None),
    ("--out", str, None, "CSV output (a .json config is written next to it)"), ("--tag", str, "", "label for this run"),
    ("--no-warmup", None, False, "skip the warm-up stream"),
]
# the reference's CSV columns (dynlp/bench.py:36-38), in its order
FIELDS = ["tag", "dataset", "K", "batch", "solver", "n_active", "n_u", "nnz", "inserted", "deleted", "iters", "edges",
          "sweeps", "ms", "setup_ms", "path", "err_max", "cert_self", "cert_post", "hmax", "hmax_ref", "agree",
          "acc_true", "build_ms", "ref_ms", "run_s", "delta", "tol", "dtype", "group"]


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    for flag, typ, default, hlp in ARGS:
        if typ is None:
            ap.add_argument(flag, action="store_true", help=hlp)
        else:
            ap.add_argument(flag, type=typ, default=default, help=hlp)
    return ap.parse_args(argv)


def env_info():
    p = torch.cuda.get_device_properties(0)
    return {"python": platform.python_version(), "gpu": p.name, "cc": f"{p.major}.{p.minor}",
            "mem_gb": round(p.total_memory / 1e9, 1), "sms": p.multi_processor_count, "torch": torch.__version__,
            "cuda": torch.version.cuda}


def metrics(sys, sys64, Fall, Fstar, hmax, y_u, K, pick):
    """Accuracy against the true labels, and with F*: max error, label agreement and the posterior
    certificate rho * hmax of the scores' own fp64 residual (dynlp/bench.py:49-61)."""
    nan, F = float("nan"), pick(Fall)
    pred, known = predict(F, K), y_u >= 0
    acc = float((pred[known] == y_u[known]).double().mean().item()) if bool(known.any()) else nan
    if Fstar is None or not sys.n_solved:
        return acc, nan, nan, nan
    Fa = Fall.to(torch.float64).contiguous()
    if sys.solved is not None:
        Fa[~sys.solved] = 0  # inert rows hold 0 in the exact solution
    R = residual(sys64, Fa, sys64.rhs)
    err = float((F.to(torch.float64) - Fstar.to(torch.float64)).abs().max().item())
    agree = float((pred == predict(Fstar, K)).double().mean().item())
    return acc, err, agree, float(rho_cols(sys64, R).max().item()) * hmax


def warmup(names, K, a):
    """Run every solver on a small stream first (graph capture, workspaces, the library load)."""
    ds = graphs.sbm(3000, K, 8.0, seed=123, dtype=a.dtype)
    st = (IncrementalStream if a.incremental else Stream)(ds, init_frac=0.9, n_batches=3, dtype=a.dtype,
                                                          label_frac=0.02)
    solvers = [make(nm, ds.n, K, dtype=a.dtype, delta=a.delta, tol=a.tol, group=a.group) for nm in names]
    for S in st.batches():
        for s in ([] if a.no_reference else [Reference(ds.n, K)]) + solvers:
            s.solve(S)
    sync()


def summarize(rows, names, run_s):
    """Per solver over all batches: time, speed-up over dynlp, iterations, worst error and bound,
    mean accuracy (dynlp/bench.py:143-157)."""
    fin = lambda v: [x for x in v if not math.isnan(x)]  # noqa: E731
    tot = {nm: sum(r["ms"] for r in rows if r["solver"] == nm) for nm in names}
    base, nan = tot.get("dynlp"), float("nan")
    hdr = f"{'solver':<11} {'time s':>8} {'x dynlp':>8} {'iters':>8} {'max err':>9} {'max bound':>10} {'acc':>7}"
    print(f"\nsummary ({run_s:.0f}s wall)\n{hdr}\n{'-' * len(hdr)}")
    for nm in names:
        rs = [r for r in rows if r["solver"] == nm]
        err, bnd, acc = (fin([r[k] for r in rs]) for k in ("err_max", "cert_post", "acc_true"))
        print(f"{nm:<11} {tot[nm] / 1e3:8.2f} {base / tot[nm] if base and tot[nm] else nan:8.2f} "
              f"{sum(r['iters'] for r in rs):8d} {max(err, default=nan):9.2e} {max(bnd, default=nan):10.2e} "
              f"{sum(acc) / len(acc) if acc else nan:7.4f}")


def main(argv=None):
    a, t_run = parse(argv), time.perf_counter()
    info = env_info()
    print("[env]", json.dumps(info), flush=True)
    ds = graphs.load(a.dataset, n=a.n, K=a.classes, deg=a.deg, p_in=a.p_in, seed=a.seed, dtype=a.dtype,
                     data_dir=a.data_dir)
    sync()
    print(f"[data] {ds.name}: n={ds.n:,} nnz={ds.nnz:,} K={ds.K} ({time.perf_counter() - t_run:.1f}s, "
          f"gpu mem {mem_used_gb():.1f} GB)", flush=True)
    stream = (IncrementalStream if a.incremental else Stream)(
        ds, label_frac=a.label_frac, init_frac=a.init_frac, n_batches=a.batches, del_frac=a.del_frac,
        eta_rel=a.eta_rel, seed=a.seed, dtype=a.dtype)
    names = [s.strip() for s in a.solvers.split(",") if s.strip()]
    if "dynlp+inc" in names and not a.incremental:
        raise SystemExit("dynlp+inc needs --incremental")
    if not a.no_warmup:
        warmup(names, ds.K, a)
    solvers = [make(nm, ds.n, ds.K, dtype=a.dtype, delta=a.delta, tol=a.tol, group=a.group, max_iter=a.max_iter)
               for nm in names]
    ref, rows, it = None if a.no_reference else Reference(ds.n, ds.K), [], stream.batches()
    for _ in range(len(stream)):
        with Timer() as tb:
            sys = next(it)
        ref_ms, Fstar, hmax, sys64 = float("nan"), None, None, None
        pick = (lambda v: v) if sys.solved is None else (lambda v: v[sys.solved])  # noqa: E731
        if ref is not None:
            with Timer() as tr:
                Fstar, hmax, _ = ref.solve(sys)
            ref_ms, sys64, Fstar = tr.ms, sys.astype(torch.float64), pick(Fstar)
        y_u = pick(ds.y[sys.U.long()])
        tau_nc = sys.comps["tau"][1] if "tau" in sys.comps else 0
        fh_nc = sys.comps["fh"][1] if "fh" in sys.comps else 0
        print(f"[batch {sys.t:>3}] active={sys.n_active:,} |U|={sys.n_solved:,} +{sys.n_inserted:,} "
              f"-{sys.n_deleted:,} comps tau/fh={tau_nc:,}/{fh_nc:,} build={tb.ms:.0f}ms ref={ref_ms:.0f}ms"
              + (f" max(h)={hmax:.3g}" if hmax is not None else ""), flush=True)
        for s in solvers:
            st = s.solve(sys)
            acc, err, agree, cert = metrics(sys, sys64, s.scores(sys), Fstar, hmax, y_u, ds.K, pick)
            row = dict(tag=a.tag or ds.name, dataset=ds.name, K=ds.K, batch=sys.t, solver=s.name,
                       n_active=sys.n_active, n_u=sys.n_solved, nnz=sys.nnz, inserted=sys.n_inserted,
                       deleted=sys.n_deleted, iters=st.iters, edges=st.edges, sweeps=st.edges / max(sys.nnz, 1),
                       ms=st.ms, setup_ms=st.setup_ms, path=st.path, err_max=err, cert_self=st.cert, cert_post=cert,
                       hmax=st.hmax, hmax_ref=float("nan") if hmax is None else hmax, agree=agree, acc_true=acc,
                       build_ms=tb.ms, ref_ms=ref_ms, delta=a.delta, tol=a.tol, dtype=a.dtype, group=a.group)
            rows.append(row)
            print(f"    {s.name:<11} {st.ms:9.1f} ms  iters={st.iters:<7} err={err:.2e} bound={cert:.2e} "
                  f"acc={acc:.4f} {st.path}", flush=True)
    run_s = time.perf_counter() - t_run
    for r in rows:
        r["run_s"] = run_s
    summarize(rows, names, run_s)
    if a.out:
        os.makedirs(os.path.dirname(a.out) or ".", exist_ok=True)
        new = not os.path.exists(a.out)
        with open(a.out, "a", newline="") as fh:
            w = csv.DictWriter(fh, fieldnames=FIELDS)
            if new:
                w.writeheader()
            w.writerows(rows)
        with open(os.path.splitext(a.out)[0] + ".json", "w") as fh:
            json.dump({"args": vars(a), "env": info, "argv": _sys.argv, "run_s": run_s}, fh, indent=2)
        print(f"[out] {len(rows)} rows -> {a.out}")
    return rows


if __name__ == "__main__":
    main()

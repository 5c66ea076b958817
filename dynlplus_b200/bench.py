"""Streaming benchmark in the reference's reporting format: solvers run over a vertex-arrival batch
stream, each batch is scored against the fp64 solution F*, and the rows are written with the
reference's CSV columns (`FIELDS`, dynlp/bench.py:36-38) plus a JSON sidecar with the arguments and
the device, so B200 runs compare row for row with the reference's results files (and feed
`python -m dynlplus_b200.matrix`).

  python -m dynlplus_b200.bench --dataset er --n 1000000 --deg 5 --init-frac 1 --batches 0 \\
      --solvers itlp,dynlp,dynlp+pcg,dynlp+amg,dynlp+auto --out results/er1m.csv

Structure: `Scorer` holds one batch's reference solution and scores any solver's scores against it;
`stream_rows` is a generator of CSV rows; the end-of-run summary is the results matrix's own
aggregation (`matrix.aggregate`) printed through a column specification.
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import os
import platform
import sys
import time

import torch

from . import graphs, matrix
from .backend import Timer, mem_used_gb, sync
from .solvers import SOLVERS, Reference, make, predict, residual, rho_cols
from .stream import IncrementalStream, Stream

# The command line, as data: (flag, type, default, help); type None = a switch. The reference's
# flags and defaults (dynlp/bench.py:22-33), except --dataset, whose reference default is the IMDB
# graph (downloads; not built here).
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
    ("--no-warmup", None, False, "skip the warm-up solves"),
]
# The CSV columns, in the reference's order (dynlp/bench.py:36-38).
FIELDS = ["tag", "dataset", "K", "batch", "solver", "n_active", "n_u", "nnz", "inserted", "deleted", "iters", "edges",
          "sweeps", "ms", "setup_ms", "path", "err_max", "cert_self", "cert_post", "hmax", "hmax_ref", "agree",
          "acc_true", "build_ms", "ref_ms", "run_s", "delta", "tol", "dtype", "group"]
NAN = float("nan")


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    for flag, typ, default, hlp in ARGS:
        kw = {"action": "store_true"} if typ is None else {"type": typ, "default": default}
        ap.add_argument(flag, help=hlp, **kw)
    return ap.parse_args(argv)


def device_info():
    """The run's device and software (the JSON sidecar's env record)."""
    p = torch.cuda.get_device_properties(0)
    return {"python": platform.python_version(), "gpu": p.name, "cc": f"{p.major}.{p.minor}",
            "mem_gb": round(p.total_memory / 1e9, 1), "sms": p.multi_processor_count, "torch": torch.__version__,
            "cuda": torch.version.cuda}


class Scorer:
    """One batch's yardstick. The quality columns keep the reference's definitions
    (dynlp/bench.py:58-70): acc_true = label accuracy on the rows with a true label; with F*:
    err_max = max |F - F*| over the solved rows, agree = share of rows whose predicted label equals
    F*'s, cert_post = rho(fp64 residual of F) * hmax(F*)."""

    def __init__(self, ds, sys, ref):
        self.sys, self.K = sys, ds.K
        self.solved = sys.solved  # global-index systems (the resident stream) carry inert rows
        self.truth = self._rows(ds.y[sys.U.long()])
        self.ref_ms, self.Fstar, self.hmax, self.sys64 = NAN, None, None, None
        if ref is not None:
            with Timer() as t:
                Fstar, self.hmax, _ = ref.solve(sys)
            self.ref_ms, self.Fstar, self.sys64 = t.ms, self._rows(Fstar), sys.astype(torch.float64)

    def _rows(self, X):
        return X if self.solved is None else X[self.solved]

    def score(self, F_all):
        F = self._rows(F_all)
        pred = predict(F, self.K)
        has_truth = self.truth >= 0
        acc = float((pred[has_truth] == self.truth[has_truth]).double().mean()) if bool(has_truth.any()) else NAN
        if self.Fstar is None or not self.sys.n_solved:
            return {"acc_true": acc, "err_max": NAN, "agree": NAN, "cert_post": NAN}
        F64 = F_all.to(torch.float64).contiguous()
        if self.solved is not None:
            F64[~self.solved] = 0  # the exact solution of an inert row is 0
        rho = float(rho_cols(self.sys64, residual(self.sys64, F64, self.sys64.rhs)).max())
        return {"acc_true": acc,
                "err_max": float((F.double() - self.Fstar.double()).abs().max()),
                "agree": float((pred == predict(self.Fstar, self.K)).double().mean()),
                "cert_post": rho * self.hmax}


def solver_names(a):
    names = [s.strip() for s in a.solvers.split(",") if s.strip()]
    if "dynlp+inc" in names and not a.incremental:
        raise SystemExit("dynlp+inc needs --incremental")
    return names


def prime(names, K, a):
    """Warm-up: every solver (and the reference) solves the initial system of a small SBM stream, so
    CUDA graphs, workspaces and the library are in place before the timed batches."""
    ds = graphs.sbm(3000, K, 8.0, seed=123, dtype=a.dtype)
    kind = IncrementalStream if a.incremental else Stream
    sys0 = next(iter(kind(ds, init_frac=0.9, n_batches=0, dtype=a.dtype, label_frac=0.02).batches()))
    for s in ([] if a.no_reference else [Reference(ds.n, K)]) + \
            [make(nm, ds.n, K, dtype=a.dtype, delta=a.delta, tol=a.tol, group=a.group) for nm in names]:
        s.solve(sys0)
    sync()


def stream_rows(a, ds, names, log=print):
    """Yield one CSV row per (batch, solver) over the vertex-arrival stream of `ds`."""
    kind = IncrementalStream if a.incremental else Stream
    st = kind(ds, label_frac=a.label_frac, init_frac=a.init_frac, n_batches=a.batches, del_frac=a.del_frac,
              eta_rel=a.eta_rel, seed=a.seed, dtype=a.dtype)
    solvers = [make(nm, ds.n, ds.K, dtype=a.dtype, delta=a.delta, tol=a.tol, group=a.group, max_iter=a.max_iter)
               for nm in names]
    ref = None if a.no_reference else Reference(ds.n, ds.K)
    batches = st.batches()
    for _ in range(len(st)):
        with Timer() as tb:
            sys = next(batches)
        sc = Scorer(ds, sys, ref)
        ncomp = {k: v[1] for k, v in sys.comps.items()}
        log(f"batch {sys.t}: {sys.n_active:,} active, {sys.n_solved:,} solved, +{sys.n_inserted:,} "
            f"-{sys.n_deleted:,} vertices, new components {ncomp or '-'}, assembly {tb.ms:.0f} ms, "
            f"F* {sc.ref_ms:.0f} ms" + (f", hmax {sc.hmax:.3g}" if sc.hmax is not None else ""))
        common = dict(tag=a.tag or ds.name, dataset=ds.name, K=ds.K, batch=sys.t, n_active=sys.n_active,
                      n_u=sys.n_solved, nnz=sys.nnz, inserted=sys.n_inserted, deleted=sys.n_deleted,
                      build_ms=tb.ms, ref_ms=sc.ref_ms, hmax_ref=NAN if sc.hmax is None else sc.hmax,
                      delta=a.delta, tol=a.tol, dtype=a.dtype, group=a.group)
        for s in solvers:
            stats = s.solve(sys)
            q = sc.score(s.scores(sys))
            log(f"  {s.name:<11} {stats.ms:9.1f} ms, {stats.iters} iterations, path {stats.path}, "
                f"error {q['err_max']:.2e} (bound {q['cert_post']:.2e}), accuracy {q['acc_true']:.4f}")
            yield {**common, **q, "solver": s.name, "iters": stats.iters, "edges": stats.edges,
                   "sweeps": stats.edges / max(sys.nnz, 1), "ms": stats.ms, "setup_ms": stats.setup_ms,
                   "path": stats.path, "cert_self": stats.cert, "hmax": stats.hmax}


# the end-of-run summary: (header, width, cell of a matrix aggregate)
SUMMARY = [("solver", 11, lambda g: g["solver"]), ("time s", 8, lambda g: f"{g['time_s']:.2f}"),
           ("x dynlp", 8, lambda g: f"{g['x_dynlp']:.2f}"), ("iters", 8, lambda g: str(g["iters"])),
           ("max err", 9, lambda g: f"{g['err']:.2e}"), ("max bound", 10, lambda g: f"{g['bound']:.2e}"),
           ("acc", 7, lambda g: f"{g['acc']:.4f}")]


def summary(rows, run_s):
    """Per solver over all batches, from the results matrix's aggregation."""
    fmt = lambda cells: " ".join(c.ljust(w) if i == 0 else c.rjust(w)  # noqa: E731
                                 for i, ((_, w, _), c) in enumerate(zip(SUMMARY, cells)))
    head = fmt([h for h, _, _ in SUMMARY])
    lines = [f"summary over {len({r['batch'] for r in rows})} batches ({run_s:.0f} s wall)", head, "-" * len(head)]
    lines += [fmt([f(g) for _, _, f in SUMMARY]) for g in matrix.aggregate(rows)]
    return "\n".join(lines)


def write(rows, path, a, info, run_s):
    """Append the rows to the CSV (header on a new file) and write the JSON sidecar beside it."""
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    fresh = not os.path.exists(path)
    with open(path, "a", newline="") as fh:
        w = csv.DictWriter(fh, fieldnames=FIELDS)
        if fresh:
            w.writeheader()
        w.writerows(rows)
    with open(os.path.splitext(path)[0] + ".json", "w") as fh:
        json.dump({"args": vars(a), "env": info, "argv": sys.argv, "run_s": run_s}, fh, indent=2)


def main(argv=None):
    a = parse(argv)
    t0 = time.perf_counter()
    info = device_info()
    print("device", json.dumps(info), flush=True)
    ds = graphs.load(a.dataset, n=a.n, K=a.classes, deg=a.deg, p_in=a.p_in, seed=a.seed, dtype=a.dtype,
                     data_dir=a.data_dir)
    sync()
    print(f"graph {ds.name}: n={ds.n:,} nnz={ds.nnz:,} K={ds.K}, loaded in {time.perf_counter() - t0:.1f} s, "
          f"{mem_used_gb():.1f} GB on the device", flush=True)
    names = solver_names(a)
    if not a.no_warmup:
        prime(names, ds.K, a)
    rows = list(stream_rows(a, ds, names, log=lambda m: print(m, flush=True)))
    run_s = time.perf_counter() - t0
    for r in rows:
        r["run_s"] = run_s
    print(summary(rows, run_s))
    if a.out:
        write(rows, a.out, a, info, run_s)
        print(f"{len(rows)} rows written to {a.out}")
    return rows


if __name__ == "__main__":
    main()

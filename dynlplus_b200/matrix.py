"""Method matrix of a results directory (the reference's scripts/matrix.py, same files and layout):
the streaming benchmark's CSV rows grouped by (tag, solver) into total solve time, iterations,
sweeps, worst error and bound, mean accuracy, the run's wall time and the usual path, with each
solver's speed relative to dynlp; written as matrix.csv and as a markdown summary matrix.md.

  python -m dynlplus_b200.matrix results/sanity
"""
from __future__ import annotations

import glob
import os
import sys

import pandas as pd

# the solvers in the reference's order (dynlp/solvers.py:461); others sort after them
ORDER = ["itlp", "dynlp", "dynlp-fh", "dynlp+pcg", "dynlp+amg", "dynlp+auto", "dynlp+inc"]


def _md_table(head, rows):
    lines = ["| " + " | ".join(head) + " |", "|" + "---|" * len(head)]
    return "\n".join(lines + ["| " + " | ".join(r) + " |" for r in rows])


def _fmt(v, spec):
    return "–" if pd.isna(v) else format(v, spec)


def summarize(d):
    """(per-(tag, solver) frame, batch-assembly seconds per tag, all rows) of the CSVs in d."""
    files = [f for f in sorted(glob.glob(os.path.join(d, "*.csv"))) if not f.endswith("matrix.csv")]
    frames = [x for x in (pd.read_csv(f) for f in files) if "solver" in x.columns]
    rows = pd.concat(frames, ignore_index=True)
    g = rows.groupby(["tag", "solver"]).agg(
        time_s=("ms", lambda v: v.sum() / 1e3), iters=("iters", "sum"), sweeps=("sweeps", "sum"),
        err=("err_max", "max"), bound=("cert_post", "max"), acc=("acc_true", "mean"), run_s=("run_s", "max"),
        path=("path", lambda v: v.mode().iat[0])).reset_index()
    build_s = rows.drop_duplicates(["tag", "batch"]).groupby("tag").build_ms.sum() / 1e3
    ref_time = g[g.solver == "dynlp"].set_index("tag").time_s
    g["x_dynlp"] = g.tag.map(ref_time) / g.time_s
    rank = {s: i for i, s in enumerate(ORDER)}
    g["order"] = g.solver.map(rank).fillna(len(ORDER))
    g = g.sort_values(["tag", "order"]).drop(columns="order")
    return g, build_s, rows


def main(d):
    g, build_s, rows = summarize(d)
    g.to_csv(os.path.join(d, "matrix.csv"), index=False)
    rank = {s: i for i, s in enumerate(ORDER)}
    tags = list(dict.fromkeys(g.tag))
    solvers = list(dict.fromkeys(g.sort_values("solver", key=lambda s: s.map(rank).fillna(99)).solver))
    cell = {(r.tag, r.solver): r for r in g.itertuples()}
    lines = [f"# Method matrix: `{d}`", "",
             f"δ = {rows.delta.iat[0]:g} (DynLP/ItLP), tol = {rows.tol.iat[0]:g} (DynLP+). Cell: solve time / accuracy.",
             "",
             _md_table(["method"] + tags,
                       [[s] + [f"{_fmt(c.time_s, '.2f')} s / {_fmt(c.acc, '.3f')}" if (c := cell.get((t, s))) else ""
                               for t in tags] for s in solvers])]
    for t in tags:
        rs = [cell[(t, s)] for s in solvers if (t, s) in cell]
        lines += ["", f"## {t}", f"wall {rs[0].run_s:.0f} s per run, batch assembly {build_s[t]:.2f} s", "",
                  _md_table(["method", "time s", "× dynlp", "iters", "sweeps", "max err", "bound", "acc", "path"],
                            [[r.solver, _fmt(r.time_s, ".2f"), _fmt(r.x_dynlp, ".2f"), str(r.iters),
                              _fmt(r.sweeps, ".0f"), _fmt(r.err, ".1e"), _fmt(r.bound, ".1e"), _fmt(r.acc, ".4f"),
                              r.path] for r in rs])]
    text = "\n".join(lines) + "\n"
    with open(os.path.join(d, "matrix.md"), "w", encoding="utf-8") as fh:
        fh.write(text)
    print(text, end="")
    return g


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "results/sanity")

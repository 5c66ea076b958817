"""Method matrix of a results directory: the streaming benchmark's CSV rows per (tag, solver), written
as matrix.csv and as a markdown report matrix.md in the layout of the reference's scripts/matrix.py
(same files, columns and lines, so B200 results compare with the reference's).

  python -m dynlplus_b200.matrix results/sanity

The aggregation is plain Python over csv rows (`aggregate`), shared with the streaming benchmark's
end-of-run summary; the two markdown tables are driven by column specifications.
"""
from __future__ import annotations

import csv
import glob
import math
import os
import sys
from collections import Counter, OrderedDict

# the solvers in the reference's order (dynlp/solvers.py:461); others sort after them
ORDER = ["itlp", "dynlp", "dynlp-fh", "dynlp+pcg", "dynlp+amg", "dynlp+auto", "dynlp+inc"]
# matrix.csv columns, in order
CSV_COLUMNS = ["tag", "solver", "time_s", "iters", "sweeps", "err", "bound", "acc", "run_s", "path", "x_dynlp"]


def _num(v):
    """A CSV cell as a float (empty or 'nan' -> NaN)."""
    try:
        return float(v)
    except (TypeError, ValueError):
        return math.nan


def _max(xs):
    xs = [x for x in xs if not math.isnan(x)]
    return max(xs) if xs else math.nan


def _mean(xs):
    xs = [x for x in xs if not math.isnan(x)]
    return sum(xs) / len(xs) if xs else math.nan


def _usual(paths):
    """The most frequent path (ties: the first in sorted order)."""
    c = Counter(paths)
    top = max(c.values())
    return min(p for p, k in c.items() if k == top)


def _rank(solver):
    return ORDER.index(solver) if solver in ORDER else len(ORDER)


def aggregate(rows):
    """Per (tag, solver) over the benchmark rows (dicts of CSV cells or numbers): total solve seconds,
    iterations, sweeps, worst error and bound, mean accuracy against the true labels, the run's wall
    seconds, the usual path and the speed relative to dynlp on the same tag. Sorted by tag, then
    solver in the reference's order."""
    groups = OrderedDict()
    for r in rows:
        groups.setdefault((str(r["tag"]), str(r["solver"])), []).append(r)
    out = []
    for (tag, solver), rs in groups.items():
        out.append({
            "tag": tag, "solver": solver,
            "time_s": sum(_num(r["ms"]) for r in rs) / 1e3,
            "iters": sum(int(_num(r["iters"])) for r in rs),
            "sweeps": sum(_num(r["sweeps"]) for r in rs),
            "err": _max(_num(r["err_max"]) for r in rs),
            "bound": _max(_num(r["cert_post"]) for r in rs),
            "acc": _mean(_num(r["acc_true"]) for r in rs),
            "run_s": _max(_num(r["run_s"]) for r in rs),
            "path": _usual(str(r["path"]) for r in rs),
        })
    base = {g["tag"]: g["time_s"] for g in out if g["solver"] == "dynlp"}
    for g in out:
        b = base.get(g["tag"])
        g["x_dynlp"] = b / g["time_s"] if b is not None and g["time_s"] else math.nan
    out.sort(key=lambda g: (g["tag"], _rank(g["solver"])))
    return out


def assembly_seconds(rows):
    """Batch assembly seconds per tag: each (tag, batch) counted once (its first row)."""
    seen, tot = set(), OrderedDict()
    for r in rows:
        key = (str(r["tag"]), str(r["batch"]))
        if key in seen:
            continue
        seen.add(key)
        tot[key[0]] = tot.get(key[0], 0.0) + _num(r["build_ms"]) / 1e3
    return tot


def read_rows(d):
    """All benchmark rows of the CSVs in d (matrix.csv itself excluded)."""
    rows = []
    for f in sorted(glob.glob(os.path.join(d, "*.csv"))):
        if f.endswith("matrix.csv"):
            continue
        with open(f, newline="") as fh:
            rd = csv.DictReader(fh)
            if rd.fieldnames and "solver" in rd.fieldnames:
                rows.extend(rd)
    return rows


def _cell(v):
    """A matrix.csv cell: floats in full (repr), NaN as an empty cell."""
    if isinstance(v, float):
        return "" if math.isnan(v) else repr(v)
    return v


def _fmt(v, spec):
    return "–" if isinstance(v, float) and math.isnan(v) else format(v, spec)


def _md(head, body):
    lines = ["| " + " | ".join(head) + " |", "|" + "---|" * len(head)]
    return lines + ["| " + " | ".join(r) + " |" for r in body]


# the per-tag table: (header, cell of one aggregate)
TAG_TABLE = [
    ("method", lambda g: g["solver"]),
    ("time s", lambda g: _fmt(g["time_s"], ".2f")),
    ("× dynlp", lambda g: _fmt(g["x_dynlp"], ".2f")),
    ("iters", lambda g: str(g["iters"])),
    ("sweeps", lambda g: _fmt(g["sweeps"], ".0f")),
    ("max err", lambda g: _fmt(g["err"], ".1e")),
    ("bound", lambda g: _fmt(g["bound"], ".1e")),
    ("acc", lambda g: _fmt(g["acc"], ".4f")),
    ("path", lambda g: g["path"]),
]


def report(d, agg, rows):
    """The markdown report: the solve time / accuracy matrix, then one table per tag."""
    tags = list(OrderedDict.fromkeys(g["tag"] for g in agg))
    solvers = sorted(OrderedDict.fromkeys(g["solver"] for g in sorted(agg, key=lambda g: g["solver"])),
                     key=lambda s: ORDER.index(s) if s in ORDER else 99)
    cell = {(g["tag"], g["solver"]): g for g in agg}
    build = assembly_seconds(rows)
    out = [f"# Method matrix: `{d}`", "",
           f"δ = {_num(rows[0]['delta']):g} (DynLP/ItLP), tol = {_num(rows[0]['tol']):g} (DynLP+). "
           "Cell: solve time / accuracy.", ""]
    body = []
    for s in solvers:
        line = [s]
        for t in tags:
            g = cell.get((t, s))
            line.append(f"{_fmt(g['time_s'], '.2f')} s / {_fmt(g['acc'], '.3f')}" if g else "")
        body.append(line)
    out += _md(["method"] + tags, body)
    for t in tags:
        gs = [cell[(t, s)] for s in solvers if (t, s) in cell]
        out += ["", f"## {t}", f"wall {gs[0]['run_s']:.0f} s per run, batch assembly {build[t]:.2f} s", ""]
        out += _md([h for h, _ in TAG_TABLE], [[f(g) for _, f in TAG_TABLE] for g in gs])
    return "\n".join(out) + "\n"


def main(d):
    rows = read_rows(d)
    agg = aggregate(rows)
    with open(os.path.join(d, "matrix.csv"), "w", newline="") as fh:
        w = csv.writer(fh)
        w.writerow(CSV_COLUMNS)
        for g in agg:
            w.writerow([_cell(g[c]) for c in CSV_COLUMNS])
    text = report(d, agg, rows)
    with open(os.path.join(d, "matrix.md"), "w", encoding="utf-8") as fh:
        fh.write(text)
    print(text, end="")
    return agg


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "results/sanity")

"""Kernel micro-benchmark over all rows (the reference's dynlp/kernelbench.py: same flags, same CSV
columns): the library sparse product (torch CSR @ dense, cuSPARSE) against the row-major SpMM, and
the frontier Jacobi kernel at each lane count, for several column counts. Times are ms per call
(CUDA events over `--reps` calls after one untimed call); GB/s are of the gather model
nnz * (4 + s_w + C s_x) bytes, as the reference counts them.

  python -m dynlplus_b200.kernelbench --dataset er --n 1000000 --cols 2,9,16,32,64 --out kernels.csv
"""
from __future__ import annotations

import argparse
import csv
import os

import numpy as np
import torch

from . import graphs
from .kernels import FrontierOps, spmm_axpy

# (flag, type, default): the reference's flags (dynlp/kernelbench.py:21-24)
ARGS = [("--dataset", str, "sbm"), ("--n", int, 1_000_000), ("--deg", float, 10.0), ("--dtype", str, "float32"),
        ("--cols", str, "2,16,32,64"), ("--groups", str, "8,32,128,cols"), ("--reps", int, 10), ("--seed", int, 0),
        ("--data-dir", str, graphs.DATA_DIR), ("--out", str, None)]
FIELDS = ["dataset", "n", "nnz", "C", "dtype", "kernel", "ms", "gb_s"]


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    for flag, typ, default in ARGS:
        ap.add_argument(flag, type=typ, default=default)
    return ap.parse_args(argv)


def kernel_name(g):
    """The reference's row labels: `cols` (class-parallel), lanesG (G lanes per row), blockG."""
    return g if g == "cols" else f"lanes{g}" if int(g) <= 32 else f"block{g}"


def main(argv=None):
    a = parse(argv)
    dev = torch.device("cuda")
    ds = graphs.load(a.dataset, n=a.n, deg=a.deg, seed=a.seed, dtype=a.dtype, data_dir=a.data_dir, device=dev)
    W, n = ds.A, ds.A.shape[0]
    dt = W.data.dtype
    real = torch.tensor([], dtype=dt).element_size()
    print(f"[data] {ds.name}: n={n:,} nnz={W.nnz:,} mean deg={W.nnz / n:.1f}")
    Wt = torch.sparse_csr_tensor(W.indptr, W.indices, W.data, (n, n))  # the library product
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timeit(fn):
        fn()
        t0.record()
        for _ in range(a.reps):
            fn()
        t1.record()
        t1.synchronize()
        return t0.elapsed_time(t1) / a.reps

    rs, rows = np.random.RandomState(a.seed), []
    allrows = torch.arange(n, dtype=torch.int32, device=dev)
    for C in [int(c) for c in a.cols.split(",")]:
        X, rhs = (torch.as_tensor(rs.random_sample((n, C)), device=dev).to(dt).contiguous() for _ in range(2))
        diag = (Wt @ torch.ones((n, 1), dtype=dt, device=dev))[:, 0] + 1
        res = [("cusparse", timeit(lambda: Wt @ X)), ("rowmajor", timeit(lambda: spmm_axpy(W, X)))]
        for g in a.groups.split(","):
            if g != "cols" and int(g) > 32:
                print(f"[skip] {kernel_name(g)}: the frontier kernels take at most 32 lanes per row")
                continue
            ops = FrontierOps(W, C, mapping="cols") if g == "cols" else FrontierOps(W, C, int(g), mapping="rows")
            res.append((kernel_name(g), timeit(lambda: ops.jacobi(allrows, X, rhs, diag, 1e-4))))
        best = min(ms for _, ms in res)
        mb = W.nnz * (4 + real + C * real) / 1e6
        print(f"\nC={C}\n{'kernel':>9} {'ms':>9} {'GB/s':>7} {'vs best':>8}")
        for k, ms in res:
            print(f"{k:>9} {ms:9.3f} {mb / ms:7.0f} {ms / best:7.1f}x")
            rows.append(dict(dataset=ds.name, n=n, nnz=W.nnz, C=C, dtype=a.dtype, kernel=k, ms=ms, gb_s=mb / ms))
        del X, rhs
        torch.cuda.empty_cache()  # keep the peak to one column count
    if a.out:
        os.makedirs(os.path.dirname(a.out) or ".", exist_ok=True)
        with open(a.out, "w", newline="") as fh:
            w = csv.DictWriter(fh, fieldnames=FIELDS)
            w.writeheader()
            w.writerows(rows)
        print(f"[out] {a.out}")
    return rows


if __name__ == "__main__":
    main()

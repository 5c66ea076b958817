"""Frontier kernels and row-major SpMM behind the reference's kernels API.

Mirrors dynlp/kernels.py: `spmm_axpy` (:377-393), `FrontierOps` (:436-492), `FusedPush`
(:396-433) and `auto_group` (:365-370). Compute runs in libdlp.so (hand-written sm_100a kernels);
the classes here only hold buffers and launch. Unlike the reference, the kernels take a row-range
pair (rbeg, rend) so the same code serves plain CSR and the slack-padded resident graph, and
leading dimensions so score matrices may be padded for 16-byte vector gathers.
"""
from __future__ import annotations

import torch

from . import _lib
from .backend import CSR, code, ld, ptr, stream, workspace

MAX_KERNEL_COLS = 256  # widest score matrix every layout takes (scalar path: 32 lanes x 8 columns)
COLS_MIN = 17


def auto_group(avg_deg: float) -> int:
    """Power-of-two lanes per row close to the mean degree, in [2, 32] (dynlp/kernels.py:365-370)."""
    g = 2
    while g < 32 and g * 2 <= max(avg_deg, 1.0):
        g *= 2
    return g


def _group(W, group) -> int:
    if group == "auto" or group is None:
        return 0
    return min(int(group), 32)


def gather_view(X: torch.Tensor) -> torch.Tensor:
    """X itself when its storage covers n * ld elements (the vector gathers may read the padding
    columns of every row, the last one included), else a contiguous copy."""
    if X.dim() == 2 and X.stride(0) > X.shape[1]:
        need = (X.storage_offset() + X.shape[0] * X.stride(0)) * X.element_size()
        if X.untyped_storage().nbytes() < need:
            return X.contiguous()
    return X


def _rows_of(W):
    if isinstance(W, CSR):
        return W.rbeg, W.rend
    return W.rbeg, W.rend  # any object with rbeg/rend/indices/data/shape (the resident graph)


def spmm_axpy(W, X, a=None, b=1.0, group="auto", *, rhs=None, cr=1.0, alpha=1.0, rows=None, out=None,
              compact=False, out_dtype=None):
    """a * X + b * (W @ X) for row-major X (n x C) in one pass (dynlp/kernels.py:377-393).

    Extensions used by the solvers: `rhs` adds cr * rhs (residual form), `alpha` scales the a-term,
    `rows` restricts the output to a row subset (written in place unless `compact`).
    """
    n = W.shape[0]
    if X.dim() != 2:
        raise ValueError("X must be 2-D (n x C)")
    C = X.shape[1]
    if out is None:
        odt = out_dtype or (torch.float32 if X.dtype == torch.bfloat16 else X.dtype)
        nout = int(rows.numel()) if (rows is not None and compact) else n
        out = torch.empty((nout, C), dtype=odt, device=X.device)
    rbeg, rend = _rows_of(W)
    X = gather_view(X)
    nrows = int(rows.numel()) if rows is not None else n
    if a is not None and a.dtype != (torch.float32 if out.dtype == torch.bfloat16 else out.dtype):
        a = a.to(torch.float32 if out.dtype == torch.bfloat16 else out.dtype)
    if rhs is not None and rhs.dtype != (torch.float32 if out.dtype == torch.bfloat16 else out.dtype):
        rhs = rhs.to(torch.float32 if out.dtype == torch.bfloat16 else out.dtype)
    _lib.call("dlp_spmm", ptr(rbeg), ptr(rend), ptr(W.indices), ptr(W.data), code(W.data), nrows,
              ptr(rows), C, ptr(X), ld(X), code(X), ptr(a), float(alpha), float(b), ptr(rhs),
              ld(rhs) if rhs is not None else C, float(cr), ptr(out), ld(out), code(out), int(bool(compact)),
              _group(W, group), W.nnz / max(n, 1), stream())
    return out


class FusedPush:
    """Asynchronous residual push with device-resident frontiers (dynlp/kernels.py:396-433).

    Takes the residual of every violating vertex (|r_u| > eps_c * diag_u), adds r_u / diag_u to z_u
    and scatters it to the neighbours, keeping r exact; converges for this M-matrix despite the
    asynchrony (chaotic relaxation). C <= 33."""

    def __init__(self, W, C, group="auto", threads=256, blocks_per_sm=8):
        if C > 33:
            raise ValueError("FusedPush takes at most 33 columns")
        self.W, self.C = W, C
        self.edges = 0

    def run(self, Z, R, diag, eps, cand, max_rounds, check_every=8, use_graph=True):
        """Push until no vertex violates; returns (rounds, converged, edge visits) (:415-433)."""
        import ctypes as ct
        W, n, C = self.W, self.W.shape[0], self.C
        cand = cand.to(torch.int32).contiguous()
        eps_h = (ct.c_double * C)(*[float(e) for e in (eps.tolist() if torch.is_tensor(eps) else eps)])
        ws = workspace("fused_push").get(_lib.lib().dlp_fused_push_workspace_bytes(n, C))
        rounds, ok, edges = ct.c_int32(0), ct.c_int32(0), ct.c_ulonglong(0)
        # a run cut short by max_rounds reports converged=False, as the reference's does (:424-433)
        _lib.call("dlp_fused_push", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(W.data), code(W.data), n, C,
                  ptr(diag.to(Z.dtype).contiguous()), ptr(Z), ld(Z), ptr(R), ld(R), code(Z), eps_h, ptr(cand),
                  int(cand.numel()), int(max_rounds), int(check_every), int(bool(use_graph)), ptr(ws), ws.numel(),
                  ct.byref(rounds), ct.byref(ok), ct.byref(edges), stream(), allow=(_lib.DLP_ERR_CAP,))
        self.edges = int(edges.value)
        self._ws = ws
        return int(rounds.value), bool(ok.value), int(edges.value)

    def counts(self):
        """(rounds, frontier rows, touched rows, edge visits) summed over the last run's rounds."""
        import ctypes as ct
        out = (ct.c_ulonglong * 4)()
        _lib.call("dlp_fused_push_counts", ptr(self._ws), out, stream())
        return tuple(int(x) for x in out)


class FrontierOps:
    """Frontier primitives bound to one sparse matrix and column count (dynlp/kernels.py:436-492)."""

    def __init__(self, W, C, group="auto", threads=256, mapping="auto"):
        self.W, self.C, self.threads, self.mapping = W, C, threads, mapping
        self.gs = _group(W, group)
        self.real = torch.float64 if W.data.dtype == torch.float64 else torch.float32
        self.use_kernel = True  # there is no fallback: the kernels are the implementation
        self.edges = torch.zeros((), dtype=torch.int64, device=W.indices.device)  # device edge-visit counter

    def _rows(self, rows):
        rbeg, rend = _rows_of(self.W)
        rows = rows.to(torch.int32)
        if rows.numel():
            self.edges += (rend.index_select(0, rows) - rbeg.index_select(0, rows)).sum(dtype=torch.int64)
        return rows

    def jacobi(self, frontier, X, rhs, diag, delta, out_list=None, out_count=None):
        """New values for frontier rows and a changed-by-more-than-delta flag (:464-474)."""
        W = self.W
        f = self._rows(frontier)
        nf = int(f.numel())
        Y = torch.empty((nf, self.C), dtype=X.dtype, device=X.device)
        ch = torch.empty(nf, dtype=torch.uint8, device=X.device)
        rbeg, rend = _rows_of(W)
        X = gather_view(X)
        diag = diag.to(X.dtype)
        rhs = rhs.to(X.dtype)
        _lib.call("dlp_frontier_jacobi", ptr(rbeg), ptr(rend), ptr(W.indices), ptr(W.data), code(W.data), ptr(f),
                  nf, self.C, ptr(X), ld(X), ptr(rhs), ld(rhs), ptr(diag), float(delta), ptr(Y), ld(Y), code(X),
                  ptr(ch), ptr(out_list), ptr(out_count), self.gs, W.nnz / max(W.shape[0], 1), stream())
        return Y, ch.bool()

    def push(self, frontier, D, R, mark):
        """R += W[:, frontier] @ D (W symmetric) and mark touched vertices (:476-486)."""
        W = self.W
        f = self._rows(frontier)
        rbeg, rend = _rows_of(W)
        D = D.to(R.dtype).contiguous()
        _lib.call("dlp_push_scatter", ptr(rbeg), ptr(rend), ptr(W.indices), ptr(W.data), code(W.data), ptr(f),
                  int(f.numel()), self.C, ptr(D), ld(D), ptr(R), ld(R), code(R), ptr(mark), self.gs,
                  W.nnz / max(W.shape[0], 1), stream())

    def mark_neighbors(self, rows, mark):
        r = self._rows(rows)
        rbeg, rend = _rows_of(self.W)
        _lib.call("dlp_mark_neighbors", ptr(rbeg), ptr(rend), ptr(self.W.indices), ptr(r), int(r.numel()),
                  ptr(mark), stream())


def flatnonzero(flag: torch.Tensor, idx: torch.Tensor | None = None, out: torch.Tensor | None = None,
                count: torch.Tensor | None = None, sync: bool = True):
    """Ascending indices of the non-zero uint8 flags (numpy.flatnonzero), mapped through idx.

    With sync=False the result buffer and a device count are returned without a host read.
    """
    n = int(flag.numel())
    if out is None:
        out = torch.empty(max(n, 1), dtype=torch.int32, device=flag.device)
    if count is None:
        count = torch.empty(1, dtype=torch.int32, device=flag.device)
    ws = workspace("compact").get(_lib.lib().dlp_compact_workspace_bytes(n))
    _lib.call("dlp_compact", ptr(flag), ptr(idx), n, ptr(out), ptr(count), ptr(ws), ws.numel(), stream())
    if not sync:
        return out, count
    return out[: int(count.item())]


def colreduce(kind: int, X, Y=None, diag=None, mask=None, out=None):
    """Column reductions in fp64: 0 max|X|/diag, 1 sum X*Y, 2 sum X^2, 3 max|X| (device double[C])."""
    n, C = X.shape
    if out is None:
        out = torch.empty(C, dtype=torch.float64, device=X.device)
    if diag is not None:
        diag = diag.to(X.dtype)
    if Y is not None:
        Y = Y.to(X.dtype)
    ws = workspace("colreduce").get(_lib.lib().dlp_colreduce_workspace_bytes(C))
    _lib.call("dlp_colreduce", kind, n, C, ptr(X), ld(X), ptr(Y), ld(Y) if Y is not None else C, ptr(diag),
              code(X), ptr(mask), ptr(out), ptr(ws), ws.numel(), stream())
    return out


def violating(R, diag, eps_d, idx=None, clear_mark=None, out=None):
    """uint8 flag per row (or per idx entry): any_c |R[r,c]| > eps_c * diag[r] (dynlp/solvers.py:105)."""
    n = int(idx.numel()) if idx is not None else R.shape[0]
    if out is None:
        out = torch.empty(max(n, 1), dtype=torch.uint8, device=R.device)
    eps64 = eps_d.to(torch.float64)
    _lib.call("dlp_violating", ptr(idx), n, R.shape[1], ptr(R), ld(R), ptr(diag.to(R.dtype)), code(R), ptr(eps64),
              ptr(out), ptr(clear_mark), stream())
    return out[:n]


def push_take(cand, Z, R, diag, D, mark=None):
    """D = R[cand] / diag[cand]; Z[cand] += D; R[cand] = 0; mark[cand] = 1 (dynlp/solvers.py:109-113)."""
    _lib.call("dlp_push_take", ptr(cand), int(cand.numel()), Z.shape[1], ptr(Z), ld(Z), ptr(R), ld(R),
              ptr(diag.to(Z.dtype)), ptr(D), ld(D), code(Z), ptr(mark), stream())

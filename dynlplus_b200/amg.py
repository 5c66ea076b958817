"""Aggregation-based algebraic multigrid for grounded graph Laplacians (mirrors dynlp/amg.py).

The operator is A = diag(s + rowsum(W)) - W with grounding s > 0. Aggregates come from
heavy-edge handshake matching; two matching passes per level coarsen by about 4x. The coarse
operator keeps the (W_c, s_c) form: W_c sums the inter-aggregate weights and s_c the grounding
(dynlp/amg.py:1-10). Setup and cycle run in libdlp's kernels (csrc/amg.cu); the coarsest level is
inverted once in fp64 (the dense coarse solve) and applied by a dense fp64 kernel per cycle.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib, kernels
from .backend import CSR, DTYPES, code, ld, ptr, stream, workspace


def code_of(dt):
    return DTYPES[dt]


@dataclass
class Level:
    W: CSR
    s: torch.Tensor      # fp64 grounding
    diag: torch.Tensor   # fp64 s + rowsum(W)
    agg: torch.Tensor = None      # fine -> coarse map (int32)
    off: torch.Tensor = None      # members of aggregate a: members[off[a]:off[a+1]]
    members: torch.Tensor = None

    def apply(self, X):
        return kernels.spmm_axpy(self.W, X, a=self.diag.to(X.dtype), b=-1.0)


def _rowsum(W: CSR) -> torch.Tensor:
    n = W.shape[0]
    ones = torch.ones((n, 1), dtype=torch.float64, device=W.indices.device)
    return kernels.spmm_axpy(W, ones)[:, 0] if n else torch.zeros(0, dtype=torch.float64, device=W.indices.device)


def handshake(W: CSR, rounds=3):
    """Heavy-edge handshake matching (dynlp/amg.py:32-64): (agg int32, number of aggregates)."""
    n = W.shape[0]
    dev = W.indices.device
    agg = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    nagg = torch.empty(1, dtype=torch.int32, device=dev)
    ws = workspace("amg_match").get(_lib.lib().dlp_amg_match_workspace_bytes(n))
    _lib.call("dlp_amg_match", n, ptr(W.indptr), ptr(W.indices), ptr(W.data.float().contiguous()), int(rounds),
              ptr(agg), ptr(nagg), ptr(ws), ws.numel(), stream())
    return agg[:n], int(nagg.item())


def members(agg, nc):
    n = int(agg.numel())
    dev = agg.device
    off = torch.empty(nc + 1, dtype=torch.int32, device=dev)
    mem = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    ws = workspace("amg_members").get(_lib.lib().dlp_amg_members_workspace_bytes(nc))
    _lib.call("dlp_amg_members", n, nc, ptr(agg), ptr(off), ptr(mem), ptr(ws), ws.numel(), stream())
    return off, mem[:n]


def coarsen(W: CSR, s, agg, nc, off=None, mem=None):
    """(W_c, s_c) of the aggregation (dynlp/amg.py:67-74): sorted CSR rows, fp64 sums in the fine
    CSR order. Every fine entry gets the key (aggregate of its row, aggregate of its column); a
    stable radix sort by key (dlp_sort_pairs) brings each coarse entry's contributions together in
    their original order and one kernel sums the runs (the reference's coalesce)."""
    dev = W.indices.device
    n, m = W.shape[0], int(W.indices.numel())
    if s is not None and off is None:
        off, mem = members(agg, nc)
    key = torch.empty(max(m, 1), dtype=torch.int64, device=dev)
    val = torch.empty(max(m, 1), dtype=torch.float64, device=dev)
    _lib.call("dlp_amg_coarse_keys", n, ptr(W.indptr), ptr(W.indices), ptr(W.data.float().contiguous()),
              ptr(agg.to(torch.int32).contiguous()), nc, ptr(key), ptr(val), stream())
    key, val = key[:m], val[:m]
    if m > 1:  # stable radix sort by coarse entry; the "no entry" marker sorts last
        kt = torch.empty_like(key)
        vt = torch.empty_like(val)
        ws = workspace("amg_sort").get(_lib.lib().dlp_sort_pairs_workspace_bytes(m))
        _lib.call("dlp_sort_pairs", m, nc * nc, ptr(key), ptr(val), ptr(kt), ptr(vt), ptr(ws), ws.numel(), stream())
        del kt, vt
    indptr_c = torch.empty(nc + 1, dtype=torch.int32, device=dev)
    col_c = torch.empty(max(m, 1), dtype=torch.int32, device=dev)
    w_c = torch.empty(max(m, 1), dtype=torch.float32, device=dev)
    nnz = torch.empty(1, dtype=torch.int32, device=dev)
    sc = torch.empty(max(nc, 1), dtype=torch.float64, device=dev) if s is not None else None
    ws = workspace("amg_coarse").get(_lib.lib().dlp_amg_coarse_reduce_workspace_bytes(m, nc))
    _lib.call("dlp_amg_coarse_reduce", m, ptr(key), ptr(val), nc, ptr(off), ptr(mem),
              ptr(s.to(torch.float64).contiguous()) if s is not None else None, ptr(sc), ptr(indptr_c), ptr(col_c),
              ptr(w_c), ptr(nnz), ptr(ws), ws.numel(), stream())
    k = int(nnz.item())
    Wc = CSR(w_c[:k], col_c[:k], indptr_c, (nc, nc))
    return Wc, (sc[:nc] if sc is not None else None)


class AMG:
    """Symmetric V-cycle preconditioner: weighted-Jacobi smoothing, exact fp64 coarse solve
    (dynlp/amg.py:77-134); same options and defaults as the reference."""

    def __init__(self, W, s, *, max_coarse=1500, passes=2, rounds=3, omega=0.7, nu=1, max_levels=25,
                 min_ratio=0.85, coarse_sweeps=20):
        self.omega, self.nu, self.coarse_sweeps = omega, nu, coarse_sweeps
        self.levels: list[Level] = []
        W = CSR(W.data.float().contiguous(), W.indices, W.indptr, W.shape) if isinstance(W, CSR) else W
        n = W.shape[0]
        s64 = s.to(torch.float64).contiguous()
        cur = Level(W, s64, s64 + _rowsum(W))
        dev = W.indices.device
        while n > max_coarse and len(self.levels) < max_levels:
            agg = torch.arange(n, dtype=torch.int32, device=dev)
            nc, Wp = n, cur.W
            for _ in range(passes):
                a2, nc2 = handshake(Wp, rounds)
                agg = a2[agg.long()]
                Wp, _ = coarsen(Wp, None, a2, nc2)
                nc = nc2
            if nc > min_ratio * n:
                break
            off, mem = members(agg, nc)
            Wc, sc = coarsen(cur.W, cur.s, agg, nc, off, mem)
            cur.agg, cur.off, cur.members = agg.contiguous(), off, mem
            self.levels.append(cur)
            cur = Level(Wc, sc, sc + _rowsum(Wc))
            n = nc
        self.coarse = cur
        self.inv = None
        if n <= 4 * max_coarse:
            Ad = torch.zeros((n, n), dtype=torch.float64, device=dev)
            if cur.W.nnz:
                rows = torch.repeat_interleave(torch.arange(n, device=dev), torch.diff(cur.W.indptr.long()))
                Ad[rows, cur.W.indices.long()] = -cur.W.data.double()
            Ad[torch.arange(n, device=dev), torch.arange(n, device=dev)] += cur.diag
            # the dense coarse operator is inverted once at setup (Gauss-Jordan in fp64, in place);
            # each cycle applies the inverse with a libdlp kernel
            if n:
                ws = workspace("amg_inverse").get(_lib.lib().dlp_dense_spd_inverse_workspace_bytes(n))
                _lib.call("dlp_dense_spd_inverse", n, ptr(Ad), ptr(ws), ws.numel(), stream())
            self.inv = Ad
        self.work_per_apply = sum(2 * nu * L.W.nnz + 2 * L.W.shape[0] for L in self.levels)
        self.work_per_apply += n * n if self.inv is not None else coarse_sweeps * cur.W.nnz
        self.sizes = [L.W.shape[0] for L in self.levels] + [n]
        self._buf: dict = {}

    def _b(self, tag, lvl, n, C, dt, dev):
        key = (tag, lvl, C, dt)
        t = self._buf.get(key)
        if t is None:
            t = torch.empty((max(n, 1), C), dtype=dt, device=dev)
            self._buf[key] = t
        return t[:n]

    def _sweep(self, L, X, R, lvl, out_tag):
        """One damped Jacobi sweep X + omega (R - A X) / diag into a fresh buffer."""
        n, C = X.shape
        Y = self._b(out_tag, lvl, n, C, X.dtype, X.device)
        diag = self._diag(L, lvl, X.dtype)
        _lib.call("dlp_amg_jacobi_sweep", n, C, ptr(L.W.indptr), ptr(L.W.indices), ptr(L.W.data), ptr(X), ld(X),
                  ptr(R), ld(R), ptr(diag), float(self.omega), ptr(Y), ld(Y), code(X), stream())
        return Y

    def _diag(self, L, lvl, dt):
        key = ("diag", lvl, 0, dt)
        d = self._buf.get(key)
        if d is None:
            d = L.diag.to(dt).contiguous()
            self._buf[key] = d
        return d

    def _smooth(self, L, X, R, sweeps, lvl):
        tags = ("sa", "sb")
        for i in range(sweeps):
            X = self._sweep(L, X, R, lvl, tags[i % 2] if X.data_ptr() != self._b(tags[i % 2], lvl, *X.shape,
                                                                                   X.dtype, X.device).data_ptr()
                            else tags[(i + 1) % 2])
        return X

    def _cycle(self, lvl, R):
        n, C = R.shape
        dt, dev = R.dtype, R.device
        if lvl == len(self.levels):
            L = self.coarse
            if self.inv is not None:
                Y = self._b("x", lvl, n, C, dt, dev)
                _lib.call("dlp_dense_apply", n, C, ptr(self.inv), ptr(R), ld(R), ptr(Y), ld(Y), code(R), stream())
                return Y
            X = self._b("x", lvl, n, C, dt, dev)
            _lib.call("dlp_amg_scale_rows", n, C, float(self.omega), ptr(R), ld(R), ptr(self._diag(L, lvl, dt)), ptr(X),
                      ld(X), code(R), stream())
            return self._smooth(L, X, R, self.coarse_sweeps - 1, lvl)
        L = self.levels[lvl]
        X = self._b("x", lvl, n, C, dt, dev)
        diag = self._diag(L, lvl, dt)
        _lib.call("dlp_amg_scale_rows", n, C, float(self.omega), ptr(R), ld(R), ptr(diag), ptr(X), ld(X), code(R),
                  stream())
        X = self._smooth(L, X, R, self.nu - 1, lvl)
        # restriction of the residual R - A X
        Rr = self._b("r", lvl, n, C, dt, dev)
        kernels.spmm_axpy(L.W, X, a=diag, alpha=-1.0, b=1.0, rhs=R, out=Rr)
        nc = self.levels[lvl + 1].W.shape[0] if lvl + 1 < len(self.levels) else self.coarse.W.shape[0]
        Rc = self._b("rc", lvl, nc, C, dt, dev)
        _lib.call("dlp_amg_restrict", nc, C, ptr(L.off), ptr(L.members), ptr(Rr), ld(Rr), ptr(Rc), ld(Rc), code(R),
                  stream())
        Xc = self._cycle(lvl + 1, Rc)
        _lib.call("dlp_amg_prolong_add", n, C, ptr(L.agg), ptr(Xc), ld(Xc), ptr(X), ld(X), code(R), stream())
        return self._smooth(L, X, R, self.nu, lvl)

    def levels_desc(self, dt):
        """The hierarchy as the library's level descriptors (dlp_amg_level), diagonals in dt; cached
        per precision together with the tensors it points at."""
        import ctypes as ct
        key = ("desc", dt)
        d = self._buf.get(key)
        if d is None:
            lv = self.levels + [self.coarse]
            arr = (_lib.AmgLevel * len(lv))()
            keep = []
            for i, L in enumerate(lv):
                diag = self._diag(L, i, dt)
                w = L.W.data if L.W.data.dtype == torch.float32 else L.W.data.float().contiguous()
                keep.append(w)
                last = i == len(lv) - 1
                arr[i] = _lib.AmgLevel(int(L.W.shape[0]), int(L.W.nnz), ptr(L.W.indptr), ptr(L.W.indices), ptr(w),
                                       ptr(diag), None if last else ptr(L.agg), None if last else ptr(L.off),
                                       None if last else ptr(L.members))
            d = (arr, len(lv), keep)
            self._buf[key] = d
            del ct
        return d

    def vcycle_workspace(self, C, dt):
        arr, nlev, _ = self.levels_desc(dt)
        return workspace("amg_vcycle").get(_lib.lib().dlp_amg_vcycle_workspace_bytes(arr, nlev, C, code_of(dt)))

    def __call__(self, R):
        """M(R): one V-cycle (dlp_amg_vcycle: every level in one library call); returns a new tensor.
        Inputs wider than 64 columns are cycled 64 columns at a time (the columns are independent)."""
        R = R.contiguous()
        n, C = R.shape
        Y = torch.empty_like(R)
        arr, nlev, _ = self.levels_desc(R.dtype)
        for c0 in range(0, C, 64):
            Rc = R[:, c0:c0 + 64] if C > 64 else R
            Yc = torch.empty_like(Rc.contiguous()) if C > 64 else Y
            Rc = Rc.contiguous()
            cw = Rc.shape[1]
            ws = self.vcycle_workspace(cw, R.dtype)
            _lib.call("dlp_amg_vcycle", arr, nlev, ptr(self.inv), self.nu, float(self.omega), self.coarse_sweeps, cw,
                      code(R), ptr(Rc), ld(Rc), ptr(Yc), ld(Yc), ptr(ws), ws.numel(), stream())
            if C > 64:
                Y[:, c0:c0 + 64] = Yc
        return Y

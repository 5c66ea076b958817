"""Many independent harmonic solves in one launch sequence (no reference counterpart).

`BatchedSystems` concatenates grounded systems with the same column count into one block-
diagonal CSR, cuts the rows into tiles aligned to instance boundaries, and `solve` runs the
batched block PCG of libdlp (`dlp_pcg_batched`): every instance keeps its own CG scalars and stop
state, so its iterates are the ones it would have alone. DynLP+'s h column (A h = diag) rides
along. `autotune` picks the lane group and tile size of the batch by timing the apply kernel.

`solve_many(systems, ...)` groups arbitrary systems by column count and returns each one's
scores; the serving loop uses it to batch fresh-solve requests.
"""
from __future__ import annotations

import ctypes as ct
import time

import numpy as np
import torch

from . import _lib, kernels
from .backend import CSR, code, ld, ptr, stream, workspace
from .solvers import padded_empty

_TUNE: dict = {}


class BatchedSystems:
    def __init__(self, systems, tile_rows=1024, dtype=torch.float64, with_h=True):
        assert systems, "no systems"
        C = systems[0].C
        assert all(s.C == C for s in systems), "one column count per batch"
        self.systems, self.C, self.dtype = systems, C, dtype
        self.Ch = C + (1 if with_h else 0)
        dev = systems[0].diag.device
        self.dev = dev
        sizes = [s.n_u for s in systems]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        N = int(self.offsets[-1])
        self.N = N
        nnzs = [s.W.nnz for s in systems]
        ip = [torch.zeros(1, dtype=torch.int64, device=dev)]
        cols, ws = [], []
        base_nnz = 0
        for s, off in zip(systems, self.offsets[:-1]):
            W = s.W
            ip.append(W.indptr[1:].long() + base_nnz)
            cols.append(W.indices.long() + int(off))
            ws.append(W.data.float())
            base_nnz += W.nnz
        self.indptr = torch.cat(ip).to(torch.int32)
        self.col = torch.cat(cols).to(torch.int32) if cols else torch.zeros(0, dtype=torch.int32, device=dev)
        self.w = torch.cat(ws) if ws else torch.zeros(0, dtype=torch.float32, device=dev)
        self.nnz = int(sum(nnzs))
        s64 = [s.astype(torch.float64) for s in systems]
        self.diag = torch.cat([s.diag for s in s64]).to(dtype).contiguous()
        rhs = torch.cat([torch.cat([s.rhs, s.diag[:, None]], 1) if with_h else s.rhs for s in s64])
        self.rhs = rhs.to(dtype).contiguous()
        self.set_tiles(tile_rows)

    def set_tiles(self, tile_rows):
        self.tile_rows = tile_rows
        tinst, tbeg, tend, toff = [], [], [], [0]
        for i, (a, b) in enumerate(zip(self.offsets[:-1], self.offsets[1:])):
            starts = np.arange(a, b, tile_rows) if b > a else np.zeros(0, dtype=np.int64)
            tinst.append(np.full(starts.shape[0], i, dtype=np.int32))
            tbeg.append(starts)
            tend.append(np.minimum(starts + tile_rows, b))
            toff.append(toff[-1] + starts.shape[0])
        dev = self.dev
        self.tinst = torch.from_numpy(np.concatenate(tinst).astype(np.int32)).to(dev)
        self.tbeg = torch.from_numpy(np.concatenate(tbeg).astype(np.int32)).to(dev)
        self.tend = torch.from_numpy(np.concatenate(tend).astype(np.int32)).to(dev)
        self.toff = torch.tensor(toff, dtype=torch.int32, device=dev)
        self.ntiles = int(self.tinst.numel())

    def csr(self) -> CSR:
        return CSR(self.w, self.col, self.indptr, (self.N, self.N))

    def autotune(self, candidates=((1, 512), (2, 512), (2, 1024), (4, 1024), (2, 2048)), reps=3):
        """Pick (edge lanes per row, tile rows) by timing the batch's SpMM on each candidate; cached
        per (rows, entries, columns)."""
        key = (self.N, self.nnz, self.Ch, self.dtype)
        if key in _TUNE:
            self.group, tr = _TUNE[key]
            self.set_tiles(tr)
            return self.group, tr
        X = padded_empty(self.N, self.Ch, self.dtype, self.dev, 1.0)
        best, arg = float("inf"), (0, self.tile_rows)
        for g, tr in candidates:
            self.set_tiles(tr)
            W = self.csr()
            Y = torch.empty((self.N, self.Ch), dtype=self.dtype, device=self.dev)
            kernels.spmm_axpy(W, X, a=self.diag, b=-1.0, out=Y, group=g)
            torch.cuda.current_stream().synchronize()
            t = time.perf_counter()
            for _ in range(reps):
                kernels.spmm_axpy(W, X, a=self.diag, b=-1.0, out=Y, group=g)
            torch.cuda.current_stream().synchronize()
            dt = (time.perf_counter() - t) / reps
            if dt < best:
                best, arg = dt, (g, tr)
        self.group = arg[0]
        self.set_tiles(arg[1])
        _TUNE[key] = arg
        return arg

    def solve(self, target_relres=1e-6, eps=None, max_iter=100_000, patience=400, check_every=8, use_graph=True,
              group=None, Z0=None, inst_targets=None):
        """Solve every instance; returns (Z (N x Ch), iters, status, relres) with per-instance arrays."""
        B, Ch, N, dev, dt = len(self.systems), self.Ch, self.N, self.dev, self.dtype
        Z = padded_empty(N, Ch, dt, dev)
        if Z0 is not None:
            Z.copy_(Z0)
        else:
            Z.zero_()
        R = torch.empty((N, Ch), dtype=dt, device=dev)
        P = padded_empty(N, Ch, dt, dev, 0.0)
        AP = torch.empty((N, Ch), dtype=dt, device=dev)
        # per-instance column norms of the right-hand side (fp64); the h column only needs a loose solve
        rn = torch.empty((B, Ch), dtype=torch.float64, device=dev)
        for i, (a, b) in enumerate(zip(self.offsets[:-1], self.offsets[1:])):
            rn[i] = kernels.colreduce(2, self.rhs[a:b]).sqrt() if b > a else torch.ones(Ch, dtype=torch.float64,
                                                                                        device=dev)
        if Ch > self.C:
            rn[:, self.C:] *= 1e3
        rn = torch.where(rn > 0, rn, torch.ones_like(rn))
        if inst_targets is not None:  # instance i stops at ||R_c|| <= inst_targets[i] ||rhs_c||
            t = torch.as_tensor(np.asarray(inst_targets, dtype=np.float64) / target_relres, device=dev)
            rn = rn * t[:, None]
        rn = rn.contiguous()
        mode = 2
        epsd = torch.full((B, Ch), 1e300, dtype=torch.float64, device=dev)
        if eps is not None:
            mode = 3
            epsd[:] = torch.as_tensor(eps, dtype=torch.float64, device=dev)
        ws = workspace("batched").get(_lib.lib().dlp_pcg_batched_workspace_bytes(B, self.ntiles, Ch))
        iters = (ct.c_int32 * B)()
        status = (ct.c_int32 * B)()
        rel = (ct.c_double * B)()
        g = self.group if group is None and hasattr(self, "group") else (group or 0)
        _lib.call("dlp_pcg_batched", ptr(self.indptr), ptr(self.col), ptr(self.w), N, Ch, ptr(self.diag), ptr(self.rhs),
                  ld(self.rhs), ptr(Z), ld(Z), ptr(R), ld(R), ptr(P), ld(P), ptr(AP), ld(AP), code(Z), B, self.ntiles,
                  ptr(self.tinst), ptr(self.tbeg), ptr(self.tend), ptr(self.toff), ptr(epsd), ptr(rn),
                  float(target_relres), mode, int(max_iter), int(patience), int(check_every), int(bool(use_graph)),
                  int(g), self.nnz / max(N, 1), ptr(ws), ws.numel(), iters, status, rel, stream())
        return Z, np.array(iters), np.array(status), np.array(rel)

    def split(self, Z):
        """Per-instance score blocks (views)."""
        return [Z[a:b, : self.C] for a, b in zip(self.offsets[:-1], self.offsets[1:])]


def solve_many(systems, target_relres=1e-6, dtype=torch.float64, tile_rows=1024, autotune=False):
    """Solve independent systems in batches grouped by column count; returns F per system (in order)
    and per-system (iterations, status, relative residual)."""
    out = [None] * len(systems)
    info = [None] * len(systems)
    by_c: dict = {}
    for i, s in enumerate(systems):
        by_c.setdefault(s.C, []).append(i)
    for C, idx in by_c.items():
        bs = BatchedSystems([systems[i] for i in idx], tile_rows=tile_rows, dtype=dtype)
        if autotune:
            bs.autotune()
        Z, it, stt, rel = bs.solve(target_relres=target_relres)
        for j, F in zip(idx, bs.split(Z)):
            out[j] = F
        for k, j in enumerate(idx):
            info[j] = (int(it[k]), int(stt[k]), float(rel[k]))
    return out, info


def solve_many_mixed(systems, target_relres=1e-6, tile_rows=1024, rounds=6, autotune=False, inner=1e-4):
    """solve_many in mixed precision: the batched PCG sweeps run in fp32 and the accuracy is won back
    by refinement against the fp64 residual (dynlp/solvers.py:322-337 applied to the batch): after a
    solve from zero, every round computes R = rhs - A Z in fp64 for all instances at once, stops when
    every instance's relative residual meets the target, and otherwise solves A D = R / scale in fp32
    and adds D * scale. The scale (column maxima of R) and the correction's target are each
    instance's own, so an instance's result does not depend on the others in its batch (autotune: the
    rows-per-warp and tile shape of the fp32 sweeps picked by BatchedSystems.autotune; inner: the
    smallest relative residual asked of one fp32 solve). Returns F per system and (iterations,
    status, relative residual) per system."""
    out, info = [None] * len(systems), [None] * len(systems)
    by_c: dict = {}
    for i, s in enumerate(systems):
        by_c.setdefault(s.C, []).append(i)
    for C, idx in by_c.items():
        group = [systems[i] for i in idx]
        bs = BatchedSystems(group, tile_rows=tile_rows, dtype=torch.float32)
        if autotune:
            bs.autotune()
        dev, N, Ch = bs.dev, bs.N, bs.Ch
        s64 = [s.astype(torch.float64) for s in group]
        diag64 = torch.cat([s.diag for s in s64]).contiguous()
        rhs64 = torch.cat([torch.cat([s.rhs, s.diag[:, None]], 1) for s in s64]).contiguous()
        A = CSR(bs.w, bs.col, bs.indptr, (N, N))
        spans = list(zip(bs.offsets[:-1], bs.offsets[1:]))
        ones = torch.ones(C, dtype=torch.float64, device=dev)
        rhs_n = [kernels.colreduce(2, rhs64[a:b, :C]).sqrt() if b > a else ones for a, b in spans]
        Z64 = padded_empty(N, Ch, torch.float64, dev, 0.0)
        # the fp32 solves aim no lower than `inner`: below their precision floor (about 1e-6 of
        # ||rhs|| on these systems, lower for some) a solve only stalls until its patience runs out
        Zf, it, _, _ = bs.solve(target_relres=max(target_relres, inner))
        Z64 += Zf.double()
        iters = it.astype(np.int64)
        rel = np.zeros(len(group))
        for rnd in range(rounds + 1):
            R64 = kernels.spmm_axpy(A, Z64, a=diag64, alpha=-1.0, b=1.0, rhs=rhs64)
            rn = [kernels.colreduce(2, R64[a:b, :C]).sqrt() if b > a else 0 * ones for a, b in spans]
            rel = np.array([float((r / torch.where(h > 0, h, torch.ones_like(h))).max()) for r, h in zip(rn, rhs_n)])
            if (rel <= target_relres).all() or rnd == rounds:
                break
            scales, rhs32 = [], torch.empty((N, Ch), dtype=torch.float32, device=dev)
            for a, b in spans:
                sc = kernels.colreduce(3, R64[a:b]) if b > a else torch.ones(Ch, dtype=torch.float64, device=dev)
                sc = torch.where(sc > 0, sc, torch.ones_like(sc))
                rhs32[a:b] = (R64[a:b] / sc[None, :]).float()
                scales.append(sc)
            bs.rhs = rhs32
            # each instance's correction brings its residual to a fifth of the target, or by `inner`
            # when that is further than one fp32 solve safely resolves (another round follows)
            need = [max(0.2 * target_relres / max(r, 1e-300), inner) for r in rel]
            D, it2, _, _ = bs.solve(target_relres=target_relres, inst_targets=need)
            for k, ((a, b), sc) in enumerate(zip(spans, scales)):
                if rel[k] > target_relres:  # a converged instance keeps its scores (same as alone)
                    Z64[a:b] += D[a:b].double() * sc[None, :]
                    iters[k] += it2[k]
        for k, j in enumerate(idx):
            a, b = spans[k]
            out[j] = Z64[a:b, :C]
            info[j] = (int(iters[k]), 5 if rel[k] <= target_relres else 2, float(rel[k]))
    return out, info

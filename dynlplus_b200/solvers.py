"""Label-propagation solvers (mirrors dynlp/solvers.py).

DynLP+ (certified): A = diag - W is a nonsingular M-matrix, so |r| <= rho * diag implies
|F - F*| <= rho * h with A h = diag (dynlp/solvers.py:10-12); h rides along as one extra column.
The iterations run in libdlp's kernels: Jacobi-PCG is one fused C call (three kernels per
iteration, the iteration loop as a CUDA graph WHILE node, device-side stop rule), push and
frontier Jacobi use the row kernels, and the fp64 refinement (solvers.py:322-337) uses fp64
residual SpMMs.

Extension over the reference: `target_relres` adds a second stop rule, the relative residual
max_c ||rhs_c - A F_c||_2 / ||rhs_c||_2 in fp64, which the certified loops must also meet.
"""
from __future__ import annotations

import ctypes as ct
import threading
from dataclasses import dataclass

import torch

from . import _lib, kernels
from .backend import Timer, code, ld, ptr, stream, workspace
from .kernels import FrontierOps
from .stream import System

F64 = torch.float64


@dataclass
class Stats:
    iters: int = 0
    edges: int = 0              # edge visits: hardware-independent work
    ms: float = 0.0             # init + setup + solve
    setup_ms: float = 0.0       # AMG setup (included in ms)
    path: str = ""
    cert: float = float("nan")  # bound the solver certified itself
    hmax: float = float("nan")
    relres: float = float("nan")  # fp64 relative residual of the F columns at return


def _pad(C, dt):
    q = 16 // torch.tensor([], dtype=dt).element_size()
    return (C + q - 1) // q * q


def padded_empty(n, C, dt, dev, fill=None):
    """n x C view of an n x ld buffer whose rows start on 16-byte boundaries (vector gathers)."""
    buf = torch.empty((n, _pad(C, dt)), dtype=dt, device=dev) if fill is None else \
        torch.full((n, _pad(C, dt)), fill, dtype=dt, device=dev)
    return buf[:, :C]


_SCRATCH: dict = {}
_PINNED = threading.local()


def _read_host(x):
    """A small device array read to the host through a pinned buffer of this thread (one blocking
    copy; a pageable read stages through a driver buffer first). Returns a list."""
    if x.device.type != "cuda":
        return x.tolist()
    key = (x.dtype, x.device.index)
    bufs = getattr(_PINNED, "bufs", None)
    if bufs is None:
        bufs = _PINNED.bufs = {}
    h = bufs.get(key)
    if h is None or h.numel() < x.numel():
        h = bufs[key] = torch.empty(max(x.numel(), 64), dtype=x.dtype, pin_memory=True)
    h[: x.numel()].copy_(x.reshape(-1), non_blocking=True)
    torch.cuda.current_stream(x.device).synchronize()
    return h[: x.numel()].tolist()


def _scratch(tag, n, C, dt, dev, padded=False):
    """n x C scratch matrix: one buffer per (tag, C, dtype, device, stream, padding), zero-filled when
    allocated, grown by at least a quarter when a larger n arrives, and handed out as its first n
    rows (same leading dimension), so systems of changing size (vertex-arrival batches, refinement of
    systems of every size) reuse one allocation instead of keeping one per size. Its contents are
    whatever the last user of the key left."""
    dev = torch.device(dev)
    sid = torch.cuda.current_stream().cuda_stream if dev.type == "cuda" else 0  # per stream, like workspaces
    key = (tag, C, dt, dev, sid, padded)
    buf = _SCRATCH.get(key)
    if buf is None or buf.shape[0] < n:
        rows = n if buf is None else max(n, buf.shape[0] + buf.shape[0] // 4)
        buf = padded_empty(rows, C, dt, dev, 0.0) if padded else torch.zeros((rows, C), dtype=dt, device=dev)
        _SCRATCH[key] = buf
    return buf[:n]


def spmm(W, X):
    """W @ X (dynlp/solvers.py:40-43)."""
    return kernels.spmm_axpy(W, X)


def apply_A(sys: System, X):
    """diag * X - W X (dynlp/solvers.py:46-49)."""
    return kernels.spmm_axpy(sys.W, X, a=sys.diag, b=-1.0)


def residual(sys: System, X, rhs, out=None, rows=None):
    """rhs - A X in one fused pass (fp64 when X is fp64). A full residual it allocates has 16-byte
    aligned padded rows, which the SpMM writes whole."""
    if out is None and rows is None:
        out = padded_empty(X.shape[0], X.shape[1], X.dtype, X.device)
    return kernels.spmm_axpy(sys.W, X, a=sys.diag.to(X.dtype), alpha=-1.0, b=1.0, rhs=rhs, out=out, rows=rows)


def rho_cols(sys: System, R):
    """max_u |R_uc| / diag_u per column (dynlp/solvers.py:52-54), fp64 on the device."""
    if R.shape[0] == 0:
        return torch.zeros(R.shape[1], dtype=F64, device=R.device)
    return kernels.colreduce(0, R, diag=sys.diag.to(R.dtype))


def violation(sys: System, R, eps_d):
    """max |R_uc| / (eps_c diag_u); <= 1 means converged (dynlp/solvers.py:57-59)."""
    if R.shape[0] == 0:
        return 0.0
    return float((rho_cols(sys, R) / torch.as_tensor(eps_d, dtype=F64, device=R.device)).max().item())


def col_norms(X):
    return kernels.colreduce(2, X).sqrt()


def residual_stats(sys: System, R, rhs=None, H=None):
    """The certification check's reductions in one pass and one device-to-host copy: (rho_cols,
    column sums of R^2, column sums of rhs^2 or None, max |H| or None) as host lists / floats
    (dynlp/solvers.py:52-54, :295-301)."""
    n, C = R.shape
    dt = R.dtype
    out = torch.zeros(3 * C + 1, dtype=F64, device=R.device)
    if n:
        if rhs is not None:
            rhs = rhs.to(dt)
        if H is not None:
            H = H.to(dt)
        ws = workspace("resid_stats").get(_lib.lib().dlp_residual_stats_workspace_bytes(C))
        _lib.call("dlp_residual_stats", n, C, ptr(R), ld(R), ptr(rhs), ld(rhs) if rhs is not None else C,
                  ptr(sys.diag.to(dt)), ptr(H), ld(H) if H is not None else 1, code(R), ptr(out), ptr(ws), ws.numel(),
                  stream())
    v = _read_host(out)
    res = _Stats((v[:C], v[C:2 * C], v[2 * C:3 * C] if rhs is not None else None, v[3 * C] if H is not None else None))
    res.dev = out  # the device copy: the refinement scales from it without an upload
    return res


class _Stats(tuple):
    """residual_stats' result: (rho_cols, sums of R^2, sums of rhs^2, max |h|) with `.dev`, the
    device array they were read from."""


class JacobiM:
    """R / diag (dynlp/solvers.py:62-63); recognised by `pcg`, which then runs the fused kernels."""

    def __init__(self, sys):
        self.sys = sys

    def __call__(self, R):
        return R / self.sys.diag.to(R.dtype)[:, None]


def jacobi_M(sys):
    return JacobiM(sys)


def bf16_weights(W):
    """bf16 copy of a sparse operator's weights, cached on the object (the BF16 sweeps)."""
    wb = getattr(W, "_w_bf16", None)
    if wb is None or wb.numel() != W.data.numel():
        wb = W.data.to(torch.bfloat16)
        try:
            W._w_bf16 = wb
        except AttributeError:
            pass
    return wb


# Optional record of fused-PCG calls: when a list, every dlp_pcg call appends (start event, end
# event, iterations, n, C) recorded on the launching stream (a profiler hook; None = off).
PCG_EVENTS = None

# Default of pcg(use_graph=None): run the PCG iteration loop as a CUDA graph (True), or launch its
# kernels one by one (False: the same kernels, for kernel-level profilers that do not follow graph
# control flow).
GRAPHS = True
# fp32 solves with whole-row gathers run the two-kernel iteration (dlp_pcg mode bit 3 off); False
# forces the three-kernel one (for comparisons)
TWO_KERNEL = True


def pcg(sys: System, Z, rhs, eps, M, max_iter, st: Stats, work_M=0, patience=400, *, target_relres=None,
        rhs_norm=None, check_every=8, use_graph=None, lowp=False, zero_start=False, confirm=True):
    """Block PCG (one CG per column) until |r_c| <= eps_c * diag (dynlp/solvers.py:66-97).

    Jacobi-preconditioned solves run as one fused libdlp call. With `target_relres` the relative
    residual ||R_c|| / rhs_norm_c <= target must hold as well (rhs_norm defaults to ||rhs_c||).
    zero_start: the solve starts from Z = 0 whatever Z holds, with rhs as the initial residual.
    confirm=False: a proposed stop is final without the recheck on the true residual (for a caller
    that computes the fp64 residual next; the AMG-preconditioned loops always recheck)."""
    if eps is None and target_relres is None:
        raise ValueError("pcg needs eps and/or target_relres")
    if M is not None and not isinstance(M, JacobiM):
        if zero_start:
            Z.zero_()  # these loops start from the Z they are given
        from .amg import AMG
        if isinstance(M, AMG) and (not lowp or Z.dtype == torch.float32):
            return _pcg_amg(sys, Z, rhs, eps, M, max_iter, st, work_M, patience, target_relres, rhs_norm,
                            check_every, use_graph, lowp)
        return _pcg_generic(sys, Z, rhs, eps, M, max_iter, st, work_M, patience, target_relres, rhs_norm, lowp)
    n, C = Z.shape
    if n == 0:
        return Z
    dt, dev = Z.dtype, Z.device
    diag = sys.diag.to(dt).contiguous()
    W = sys.W
    wdt = W.data.dtype
    if dt == torch.float32 and wdt != torch.float32:
        raise TypeError("fp32 PCG needs fp32 weights")
    R = _scratch("pcg_R", n, C, dt, dev)
    P = _scratch("pcg_P", n, C, dt, dev, padded=True)
    # padded like P: the apply writes whole 16-byte aligned rows (two vector stores per row for
    # fp32 rows of 9-12 columns) instead of one scalar store per column
    AP = _scratch("pcg_AP", n, C, dt, dev, padded=True)
    eps_h = (ct.c_double * C)(*[float(e) for e in eps]) if eps is not None else None
    mode = 1 if eps is not None else 0
    rn = None
    if target_relres is not None:
        mode |= 2
        if rhs_norm is None:
            rhs_norm = col_norms(rhs.to(dt)).cpu().tolist()
        rn = (ct.c_double * C)(*[float(x) for x in rhs_norm])
    if zero_start:
        mode |= 4  # Z == 0 on entry: the initial residual is rhs (no SpMM)
    if not TWO_KERNEL:
        mode |= 8  # the three-kernel iteration even where the two-kernel one applies
    if not confirm:
        mode |= 16  # the caller confirms the stop on its own (fp64) residual
    ws = workspace("pcg").get(_lib.lib().dlp_pcg_workspace_bytes(C))
    it, viol, rel, status = ct.c_int32(0), ct.c_double(0), ct.c_double(0), ct.c_int32(0)
    rhs = rhs.to(dt)
    w_lo = P_lo = None
    if lowp:
        if dt != torch.float32:
            raise TypeError("the BF16 sweeps run inside the fp32 working precision")
        w_lo = bf16_weights(W)
        P_lo = _scratch("pcg_Plo", n, C, torch.bfloat16, dev, padded=True)
    ev = None
    if PCG_EVENTS is not None:
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ev[0].record()
    _lib.call("dlp_pcg", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(W.data), code(W.data), n, C, ptr(diag),
              ptr(rhs), ld(rhs), ptr(Z), ld(Z), ptr(R), ld(R), ptr(P), ld(P), ptr(AP), ld(AP), code(Z), eps_h, rn,
              float(target_relres or 0.0), mode, int(max_iter), int(patience), int(check_every),
              int(bool(GRAPHS if use_graph is None else use_graph)),
              W.nnz / max(n, 1), ptr(ws), ws.numel(), ct.byref(it), ct.byref(viol), ct.byref(rel), ct.byref(status),
              stream(), ptr(w_lo), ptr(P_lo), ld(P_lo) if P_lo is not None else 0,
              allow=(_lib.DLP_ERR_CAP,))  # at the iteration cap the iterate stands, as in the reference
    if ev is not None:
        ev[1].record()
        PCG_EVENTS.append((ev[0], ev[1], it.value, n, C))
    st.iters += it.value
    st.edges += (it.value + 2) * W.nnz + work_M * it.value
    st.relres = rel.value
    if status.value == 4:
        raise FloatingPointError("PCG breakdown: non-finite residual")
    return Z


def _pcg_amg(sys, Z, rhs, eps, M, max_iter, st, work_M, patience, target_relres, rhs_norm, check_every, use_graph,
             lowp=False):
    """PCG with the AMG V-cycle as preconditioner, its loop on the device (dlp_pcg_amg): the
    reference's pcg (dynlp/solvers.py:66-97) with M = amg.AMG, one host read per device-side loop
    and per confirmation of a proposed stop."""
    n, C = Z.shape
    if n == 0:
        return Z
    dt, dev = Z.dtype, Z.device
    W = sys.W
    w32 = W.data if W.data.dtype == torch.float32 else W.data.float().contiguous()
    diag = sys.diag.to(dt).contiguous()
    rhs = rhs.to(dt)
    R = _scratch("amg_R", n, C, dt, dev)
    P = _scratch("amg_P", n, C, dt, dev)
    AP = _scratch("amg_AP", n, C, dt, dev)
    Y = _scratch("amg_Y", n, C, dt, dev)
    arr, nlev, _ = M.levels_desc(dt)
    ws = workspace("pcg_amg").get(_lib.lib().dlp_pcg_amg_workspace_bytes(arr, nlev, C, code(Z)))
    mode = 1 if eps is not None else 0
    eps_h = (ct.c_double * C)(*[float(e) for e in eps]) if eps is not None else None
    rn = None
    if target_relres is not None:
        mode |= 2
        if rhs_norm is None:
            rhs_norm = col_norms(rhs).cpu().tolist()
        rn = (ct.c_double * C)(*[float(x) for x in rhs_norm])
    w_lo = P_lo = None
    if lowp:  # bf16 weights and a bf16 mirror of P in the apply (fp32 accumulation)
        w_lo = bf16_weights(W)
        P_lo = _scratch("amg_Plo", n, C, torch.bfloat16, dev, padded=True)
    it, rel, status = ct.c_int32(0), ct.c_double(0), ct.c_int32(0)
    _lib.call("dlp_pcg_amg", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(w32), n, C, ptr(diag), ptr(rhs), ld(rhs),
              ptr(Z), ld(Z), ptr(R), ld(R), ptr(P), ld(P), ptr(AP), ld(AP), ptr(Y), ld(Y), code(Z), eps_h, rn,
              float(target_relres or 0.0), mode, int(max_iter), int(patience),
              int(bool(GRAPHS if use_graph is None else use_graph)), W.nnz / max(n, 1), arr, nlev, ptr(M.inv),
              int(M.nu), float(M.omega), int(M.coarse_sweeps), ptr(ws), ws.numel(), ct.byref(it), ct.byref(rel),
              ct.byref(status), stream(), ptr(w_lo), ptr(P_lo), ld(P_lo) if P_lo is not None else 0,
              allow=(_lib.DLP_ERR_CAP,))
    st.iters += it.value
    st.edges += (it.value + 2) * W.nnz + work_M * it.value
    st.relres = rel.value
    if status.value == 4:
        raise FloatingPointError("PCG breakdown: non-finite residual")
    return Z


def _apply_lowp(sys, P, W, wb, Pb, ones):
    """A P with the SpMM on bf16 weights and a bf16 mirror of P (fp32 accumulation and diagonal)."""
    n, C = P.shape
    _lib.call("dlp_cols_scale", n, C, ptr(P), ld(P), code(P), ptr(ones), 2, ptr(Pb), ld(Pb), code(Pb), stream())
    AP = torch.empty_like(P)
    _lib.call("dlp_spmm_lowp", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(wb), n, C, ptr(Pb), ld(Pb), ptr(P),
              ld(P), ptr(sys.diag.to(torch.float32).contiguous()), 1.0, -1.0, ptr(AP), ld(AP), 0,
              W.nnz / max(n, 1), stream())
    return AP


def _pcg_generic(sys, Z, rhs, eps, M, max_iter, st, work_M, patience, target_relres, rhs_norm, lowp=False):
    """PCG with a general preconditioner M (the AMG V-cycle): the reference loop
    (dynlp/solvers.py:66-97) over libdlp's SpMM and fp64 column reductions."""
    dt = Z.dtype
    if lowp:
        if dt != torch.float32:
            raise TypeError("the BF16 sweeps run inside the fp32 working precision")
        wb = bf16_weights(sys.W)
        Pb = _scratch("gen_Plo", Z.shape[0], Z.shape[1], torch.bfloat16, Z.device, padded=True)
        ones = torch.ones(Z.shape[1], dtype=F64, device=Z.device)
        applyA = lambda X: _apply_lowp(sys, X.contiguous(), sys.W, wb, Pb, ones)  # noqa: E731
    else:
        applyA = lambda X: apply_A(sys, X)  # noqa: E731
    eps_d = torch.as_tensor(eps, dtype=F64, device=Z.device)
    rn = None
    if target_relres is not None:
        rn = (col_norms(rhs.to(dt)) if rhs_norm is None else torch.as_tensor(rhs_norm, dtype=F64, device=Z.device))

    def stop_metric(R):
        m = (rho_cols(sys, R) / eps_d).max()
        if rn is not None:
            m = torch.maximum(m, (col_norms(R) / torch.where(rn > 0, rn, torch.ones_like(rn))).max() / target_relres)
        return float(m.item())

    R = residual(sys, Z, rhs.to(dt))
    st.edges += sys.nnz
    best = stop_metric(R)
    if best <= 1:
        return Z
    P = Y = M(R)
    rz, stall = kernels.colreduce(1, R, Y=Y), 0
    for _ in range(max_iter):
        AP = applyA(P)
        pAp = kernels.colreduce(1, P, Y=AP)
        alpha = torch.where(pAp > 0, rz / torch.where(pAp > 0, pAp, torch.ones_like(pAp)), torch.zeros_like(pAp))
        Z += alpha.to(dt)[None, :] * P
        R -= alpha.to(dt)[None, :] * AP
        st.iters, st.edges = st.iters + 1, st.edges + sys.nnz + work_M
        v = stop_metric(R)
        if v <= 1:
            R = residual(sys, Z, rhs.to(dt))
            st.edges += sys.nnz
            if (v := stop_metric(R)) <= 1:
                break
        best, stall = (v, 0) if v < 0.9 * best else (best, stall + 1)
        if stall >= patience:
            break
        Y = M(R)
        rz_new = kernels.colreduce(1, R, Y=Y)
        beta = torch.where(rz > 0, rz_new / torch.where(rz > 0, rz, torch.ones_like(rz)), torch.zeros_like(rz))
        P = Y + beta.to(dt)[None, :] * P
        rz = rz_new
    return Z


def push(sys: System, Z, R, eps, ops: FrontierOps, st: Stats, budget_edges=None, max_iter=10**7, record=None):
    """Residual push (Jacobi on the violating set) until |r_c| <= eps_c * diag (solvers.py:100-125).

    One round: D = R[cand]/diag; Z[cand] += D; R[cand] = 0; R[N(cand)] += W D (atomics); the next
    candidates are the touched rows that violate. Sets are compacted in ascending order, so the
    candidate set of every round equals the reference's (up to float ties at the threshold).
    `record`, a list, receives (cand, touched) per round. Returns (Z, R, converged)."""
    n = Z.shape[0]
    dev, dt = Z.device, Z.dtype
    diag = sys.diag.to(dt).contiguous()
    eps_d = torch.as_tensor(eps, dtype=F64, device=dev)
    flags = torch.empty(max(n, 1), dtype=torch.uint8, device=dev)
    mark = torch.zeros(max(n, 1), dtype=torch.uint8, device=dev)
    cand = kernels.flatnonzero(kernels.violating(R, diag, eps_d, out=flags))
    e0, it, best, stall = int(ops.edges), 0, float("inf"), 0
    D = torch.empty((max(n, 1), Z.shape[1]), dtype=dt, device=dev)
    while cand.numel() and it < max_iter:
        kernels.push_take(cand, Z, R, diag, D[: cand.numel()], mark)
        ops.push(cand, D[: cand.numel()], R, mark)
        touched = kernels.flatnonzero(mark)
        viol = kernels.violating(R, diag, eps_d, idx=touched, clear_mark=mark, out=flags)
        if record is not None:
            record.append((cand.clone(), touched.clone()))
        cand = kernels.flatnonzero(viol, idx=touched)
        it += 1
        if it % 32 == 0:
            if budget_edges is not None and int(ops.edges) - e0 > budget_edges:
                break
            v = violation(sys, R, eps_d)
            best, stall = (v, 0) if v < 0.99 * best else (best, stall + 1)
            if stall >= 8:
                break
    st.iters += it
    return Z, R, cand.numel() == 0


def _comp_avg(lab, nc, S_rows, T_rows, fallback):
    """Per component of the new vertices: sum of S over sum of T (T = 0: fallback)
    (dynlp/solvers.py:128-135)."""
    lab = lab.long()
    S = torch.zeros((nc,) + tuple(S_rows.shape[1:]), dtype=S_rows.dtype, device=S_rows.device).index_add_(0, lab, S_rows)
    T = torch.zeros(nc, dtype=S_rows.dtype, device=S_rows.device).index_add_(0, lab, T_rows.to(S_rows.dtype))
    ok = T > 0
    Tn = torch.where(ok, T, torch.ones_like(T))
    fb = torch.as_tensor(fallback, dtype=S_rows.dtype, device=S_rows.device)
    if S.dim() == 2:
        return torch.where(ok[:, None], S / Tn[:, None], fb)
    return torch.where(ok, S / Tn, fb)


def _rows_spmm(sys: System, rows, Y):
    """W[rows] @ Y (rows of the system's operator, compact output)."""
    return kernels.spmm_axpy(sys.W, Y.contiguous(), rows=rows.to(torch.int32).contiguous(), compact=True)


def supernode_init(sys: System, X, known=None, cols=None, comp="tau"):
    """Initialise the new rows per component of the new vertices (DynLP's supernodes,
    dynlp/solvers.py:138-153): with known=None the share of the component's weight to each
    labelled class (DynLP's rule); with a known mask the weighted average over labelled and known
    neighbours. Writes X[new, cols] in place and returns X."""
    new = torch.nonzero(sys.is_new, as_tuple=False).flatten()
    if not new.numel() or comp not in sys.comps:
        return X
    cols = slice(0, sys.C) if cols is None else cols
    B = sys.B.to(X.dtype)
    s_, t = sys.label_cols(B)[new], B[new].sum(dim=1)
    if known is not None:
        kf = known.to(X.dtype)
        s_ = s_ + _rows_spmm(sys, new, X[:, cols] * kf[:, None])
        t = t + _rows_spmm(sys, new, kf[:, None])[:, 0]
    lab, nc = sys.comps[comp]
    X[new, cols] = _comp_avg(lab, nc, s_, t, sys.prior.to(X.dtype)[None, :])[lab.long()]
    return X


def init_h(sys: System, H, known, fallback, comp="fh"):
    """New rows: h = 1 + the component's weighted average h over known neighbours, labelled ones
    counting with h = 0 (dynlp/solvers.py:156-163). Writes H[new, 0] in place and returns H."""
    new = torch.nonzero(sys.is_new, as_tuple=False).flatten()
    if new.numel() and comp in sys.comps:
        kf = known.to(H.dtype)
        lab, nc = sys.comps[comp]
        a = _rows_spmm(sys, new, (H[:, 0] * kf)[:, None])[:, 0]
        b = sys.B.to(H.dtype)[new].sum(dim=1) + _rows_spmm(sys, new, kf[:, None])[:, 0]
        H[new, 0] = (_comp_avg(lab, nc, a, b, fallback - 1) + 1)[lab.long()]
    return H


def predict(F, K):
    """dynlp/solvers.py:166-167."""
    return (F[:, 0] > 0.5).to(torch.int32) if K == 2 else F.argmax(dim=1).to(torch.int32)


class Solver:
    name = "base"

    def __init__(self, n_total, K, dtype="float32", store_dtype=None):
        from .backend import to_dtype
        self.n_total, self.K, self.dtype = n_total, K, to_dtype(dtype)
        self.store_dtype, self.C, self.F = to_dtype(store_dtype or dtype), 1 if K == 2 else K, None

    def _warm(self, sys: System):
        if self.F is None:
            self.F = torch.empty((self.n_total, self.C), dtype=self.store_dtype, device=sys.diag.device)
            self.F[:] = sys.prior.to(self.store_dtype)
        return self.F[sys.U].to(self.dtype)

    def _store(self, sys: System, X):
        self.F[sys.U] = X.to(self.store_dtype)

    def scores(self, sys: System):
        return self.F[sys.U]


class ItLP(Solver):
    """Plain Jacobi label propagation from the prior (dynlp/solvers.py:188-210): X = (rhs + W X) /
    diag over all rows until no entry moves by more than delta, one frontier-Jacobi launch over
    every row per sweep (its change flags are the stop test)."""
    name = "itlp"

    def __init__(self, n_total, K, dtype="float32", delta=1e-4, max_iter=200_000):
        super().__init__(n_total, K, dtype)
        self.delta, self.max_iter = delta, max_iter

    def solve(self, sys):
        st, sys = Stats(path="jacobi"), sys.astype(self.dtype)
        with Timer() as tm:
            X = self._warm(sys).contiguous()
            X[:] = sys.prior
            n = X.shape[0]
            if n:
                ops = FrontierOps(sys.W, self.C)
                rows = torch.arange(n, dtype=torch.int32, device=X.device)
                for _ in range(self.max_iter):
                    Y, ch = ops.jacobi(rows, X, sys.rhs, sys.diag, self.delta)
                    X, st.iters, st.edges = Y, st.iters + 1, st.edges + sys.nnz
                    if not bool(ch.any()):
                        break
            self._store(sys, X)
        st.ms = tm.ms
        return st


class DynLP(Solver):
    """DynLP's frontier Jacobi (Algorithm 2, dynlp/solvers.py:213-241) on the frontier kernels: the
    new rows start at their component's label share (supernode_init, the paper's tau components or
    the adaptive ones with comp="fh"), the frontier starts at the seed rows; each round updates
    the rows that changed by more than delta and the next frontier is their neighbourhood."""

    def __init__(self, n_total, K, dtype="float32", delta=1e-4, group="auto", comp="tau", max_iter=10**7):
        super().__init__(n_total, K, dtype)
        self.delta, self.group, self.comp, self.max_iter = delta, group, comp, max_iter
        self.name = "dynlp" if comp == "tau" else f"dynlp-{comp}"

    def solve(self, sys, record=None):
        st, sys = Stats(path="frontier-jacobi"), sys.astype(self.dtype)
        with Timer() as tm:
            X = supernode_init(sys, self._warm(sys).contiguous(), comp=self.comp)
            ops = FrontierOps(sys.W, self.C, self.group)
            n = X.shape[0]
            frontier = kernels.flatnonzero(sys.seed.to(torch.uint8))
            mark = torch.zeros(max(n, 1), dtype=torch.uint8, device=X.device)
            while frontier.numel() and st.iters < self.max_iter:
                if record is not None:
                    record.append(frontier.clone())
                Y, ch = ops.jacobi(frontier, X, sys.rhs, sys.diag, self.delta)
                st.iters += 1
                chu = ch.to(torch.uint8)
                upd = kernels.flatnonzero(chu, idx=frontier)
                if not upd.numel():
                    break
                X[upd.long()] = Y[ch]
                mark.zero_()
                mark[upd.long()] = 1
                ops.mark_neighbors(upd, mark)
                frontier = kernels.flatnonzero(mark)
            self._store(sys, X)
        st.edges, st.ms = int(ops.edges), tm.ms
        return st


class DynLPPlus(Solver):
    """Certified DynLP+: guarantees ||F - F*||_inf <= tol on every batch (dynlp/solvers.py:244-343)."""

    def __init__(self, n_total, K, dtype="float32", method="auto", tol=1e-3, eps_h=0.05, group="auto",
                 push_frac=0.05, push_budget=30.0, amg_hmax=2000.0, max_iter=100_000, amg_opts=None,
                 target_relres=None, lowp=False, class_sum=False, refine_share=0.2):
        super().__init__(n_total, K, dtype, store_dtype="float64")  # float64 master copy of F and h
        self.method, self.tol, self.eps_h, self.group = method, tol, eps_h, group
        self.push_frac, self.push_budget, self.amg_hmax = push_frac, push_budget, amg_hmax
        self.max_iter, self.amg_opts = max_iter, amg_opts or {}
        self.target_relres = target_relres
        # share of the relative-residual target a correction round aims for (the rest absorbs the
        # working-precision rounding between the PCG's own residual and the fp64 one); the fp64
        # residual after the round decides whether another one runs
        self.refine_share = refine_share
        self.lowp = lowp  # SpMM sweeps on bf16 weights and scores (fp32 accumulation)
        # refinement corrections solve K - 1 class columns and derive the last (_correct_class_sum)
        self.class_sum = class_sum
        self.name, self.H, self.hmax = f"dynlp+{method}", None, None

    def _use_amg(self):
        return self.method == "amg" or (self.method == "auto" and (self.hmax or float("inf")) > self.amg_hmax)

    def _precond(self, sys, st, amg_box):
        if not self._use_amg():
            return jacobi_M(sys), 0
        if amg_box[0] is None:
            from .amg import AMG
            with Timer() as t:
                amg_box[0] = AMG(sys.W, sys.s, **self.amg_opts)
            st.setup_ms += t.ms
            st.edges += 10 * sys.nnz
        return amg_box[0], amg_box[0].work_per_apply

    def _global(self, sys, Z, rhs, eps, st, amg_box, **kw):
        M, wm = self._precond(sys, st, amg_box)
        return pcg(sys, Z, rhs, eps, M, self.max_iter, st, wm, lowp=self.lowp and Z.dtype == torch.float32, **kw)

    def _run(self, sys, Z, rhs, eps, ops, st, amg_box, zero_start=False, **kw):
        """auto: push when few rows violate, else PCG/AMG (dynlp/solvers.py:272-288). With
        zero_start the solve starts from Z = 0 (Z's incoming values are ignored) and the residual is
        rhs itself."""
        if self.method != "auto":
            st.path = self.method
            return self._global(sys, Z, rhs, eps, st, amg_box, zero_start=zero_start, **kw)
        if zero_start:
            R = rhs
        else:
            R = residual(sys, Z, rhs)
            st.edges += sys.nnz
        n = Z.shape[0]
        eps_d = torch.as_tensor(eps, dtype=F64, device=Z.device)
        frac = int(kernels.violating(R, sys.diag, eps_d).sum().item()) / max(n, 1)
        if n and frac > self.push_frac:
            st.path = "amg" if self._use_amg() else "pcg"
            return self._global(sys, Z, rhs, eps, st, amg_box, zero_start=zero_start, **kw)
        if zero_start:
            Z.zero_()
            R = rhs.clone()  # push updates R in place
        Z, R, ok = push(sys, Z, R, eps, ops, st, self.push_budget * max(sys.nnz, 1))
        st.path = "push"
        if ok and not kw.get("target_relres"):
            return Z
        st.path = "push+amg" if self._use_amg() else "push+pcg"
        return self._global(sys, Z, rhs, eps, st, amg_box, **kw)

    def _floor(self, scale=1.0):
        """Smallest residual ratio the working precision resolves (dynlp/solvers.py:290-293)."""
        u = 1e-7 if self.dtype == torch.float32 else 2e-16
        return min(0.5, max(20 * u, 10 * u * scale))

    def _bound(self, rc, h_est):
        """(hmax, bound) from the column residual ratios (dynlp/solvers.py:295-301)."""
        C = self.C
        if rc[C] > self.eps_h:
            return h_est, float("inf")
        hmax = h_est / (1 - float(rc[C]))
        return hmax, float(max(rc[:C])) * hmax

    def _relres_ok(self, ss, rhs_norm):
        """max_c ||R_c|| / ||rhs_c|| over the label columns, from the column sums of squares."""
        if self.target_relres is None:
            return True, float("nan")
        rel = max((ss[c] ** 0.5) / rhs_norm[c] if rhs_norm[c] > 0 else ss[c] ** 0.5 for c in range(self.C))
        return rel <= self.target_relres, rel

    def _refine(self, sw, s64, Z64, rhs64, ops, st, amg_box, rounds, rhs_norm, R64=None, stats=None):
        """fp64 certification and refinement (dynlp/solvers.py:322-337): R64 = rhs - A Z64; if the
        certificate (or the relative residual) falls short, solve A D = R64 / scale in the working
        precision and add D * scale. `stats` (residual_stats of R64) may come with R64. Returns
        (Z64, R64, hmax, bound, relres)."""
        C = self.C
        hmax, bound, rel = self.hmax, float("inf"), float("nan")
        dev = Z64.device
        for _ in range(rounds):
            if R64 is None:
                R64 = residual(s64, Z64, rhs64)
                st.edges += s64.nnz
                stats = None
            if stats is None:
                stats = residual_stats(s64, R64, H=Z64[:, C:])
            rc, ss, _, h_est = stats
            hmax, bound = self._bound(rc, h_est)
            ok_rel, rel = self._relres_ok(ss, rhs_norm)
            if bound <= self.tol and ok_rel:
                break
            scale = [r if r > 0 else 1.0 for r in rc]
            dv = getattr(stats, "dev", None)
            if dv is not None and dv.device == dev and dv.numel() >= C + 1:
                sc = torch.where(dv[: C + 1] > 0, dv[: C + 1], torch.ones_like(dv[: C + 1]))  # = scale, on device
            else:
                sc = torch.tensor(scale, dtype=F64, device=dev)
            eps_c = [min(max(e / s, self._floor(h_est)), 1.0) for e, s in
                     zip([self.tol / (1.25 * hmax)] * C + [self.eps_h], scale)]
            kw = {}
            if self.target_relres is not None:
                # the correction must bring the fp64 residual of every F column under the target, or
                # as far as the working precision resolves in one round (the next round continues)
                rnR = [ss[c] ** 0.5 for c in range(C)]
                # what one round can resolve: bf16 gathers ~2e-3, fp32 sweeps ~3e-6, fp64 ~1e-13
                fl = (2e-3 if self.lowp else 3e-6) if self.dtype == torch.float32 else 1e-13
                allowed = [max(self.refine_share * self.target_relres * float(rhs_norm[c]), fl * rnR[c], 1e-300) /
                           scale[c] for c in range(C)]
                # the fp64 residual computed next confirms the correction's stop, so the solve skips
                # its own recheck on the working-precision residual
                kw = dict(target_relres=1.0, rhs_norm=allowed + [1e300], confirm=False)
            if kw and self.dtype == torch.float32 and self._class_sum_applies(s64, C):
                self._correct_class_sum(sw, s64, Z64, R64, sc, scale, eps_c, allowed, kw, ops, st, amg_box)
            else:
                Rs = _scratch("ref_Rs", Z64.shape[0], C + 1, self.dtype, dev)
                _lib.call("dlp_cols_scale", Z64.shape[0], C + 1, ptr(R64), ld(R64), code(R64), ptr(sc), 0, ptr(Rs),
                          ld(Rs), code(Rs), stream())
                D = _scratch("ref_D", Z64.shape[0], C + 1, self.dtype, dev, padded=True)  # zeroed by the zero start
                D = self._run(sw, D, Rs, eps_c, ops, st, amg_box, zero_start=True, **kw)
                _lib.call("dlp_cols_scale", Z64.shape[0], C + 1, ptr(D), ld(D), code(D), ptr(sc), 1, ptr(Z64),
                          ld(Z64), code(Z64), stream())
            R64, stats = None, None
        if R64 is None:
            R64 = residual(s64, Z64, rhs64)
            st.edges += s64.nnz
            rc, ss, _, h_est = residual_stats(s64, R64, H=Z64[:, C:])
            hmax, bound = self._bound(rc, h_est)
            _, rel = self._relres_ok(ss, rhs_norm)
        return Z64, R64, hmax, bound, rel

    def _class_sum_applies(self, s64, C):
        """class_sum: more than one class column, and the system's right-hand sides sum to its
        grounding on every solved row (sum_c rhs_c = s = A 1, so the scores sum to one there). The
        identity holds by construction of the systems (stream.build_system, EdgeStream); it is
        checked once, on the first system the solver corrects, and trusted afterwards."""
        if not (self.class_sum and C > 2):
            return False
        key = "checked"
        if getattr(self, "_cs_key", None) != key:
            d = (s64.rhs.sum(dim=1) - s64.s).abs()
            if s64.solved is not None:
                d = torch.where(s64.solved, d, torch.zeros_like(d))
            self._cs_ok = bool(d.max() <= 1e-9 * max(float(s64.s.abs().max()), 1e-300)) if d.numel() else False
            self._cs_key = key
        return self._cs_ok

    def _correct_class_sum(self, sw, s64, Z64, R64, sc, scale, eps_c, allowed, kw, ops, st, amg_box):
        """The refinement's correction with the last class column eliminated: the scores of a grounded
        row sum to one, so the PCG solves the first C - 1 class columns and h (C columns: 32-byte rows
        for C = 8), and the last class is set to one minus the others. Its residual is minus the sum
        of theirs, so each solved class column aims at the last one's target over sqrt(C - 1) (the
        fp64 residual of every column, the derived one included, decides the next round)."""
        C, n, dev = self.C, Z64.shape[0], Z64.device
        absA = [allowed[c] * scale[c] for c in range(C)]
        lim = absA[C - 1] / (C - 1) ** 0.5
        allowed_e = [min(absA[c], lim) / scale[c] for c in range(C - 1)]
        kw = dict(kw, rhs_norm=allowed_e + [1e300])
        eps_e = list(eps_c[: C - 1]) + [eps_c[C]]
        Re = _scratch("ref_Re", n, C, torch.float32, dev)
        _lib.call("dlp_class_sum_rhs", n, C, ptr(R64), ld(R64), ptr(sc), ptr(Re), ld(Re), stream())
        De = _scratch("ref_De", n, C, torch.float32, dev, padded=True)  # zeroed by the zero start
        De = self._run(sw, De, Re, eps_e, ops, st, amg_box, zero_start=True, **kw)
        sol = None
        if s64.solved is not None:
            sol = s64.solved.view(torch.uint8) if s64.solved.dtype == torch.bool else s64.solved.to(torch.uint8)
        _lib.call("dlp_class_sum_update", n, C, ptr(De), ld(De), ptr(sc), ptr(Z64), ld(Z64), ptr(sol), stream())

    def _rhs_h(self, sys):
        if sys.rhs_h is not None:
            return sys.rhs_h
        return torch.cat([sys.rhs, sys.diag[:, None]], dim=1).contiguous()

    def solve(self, sys):
        st, C, tol = Stats(), self.C, self.tol
        sw, s64 = sys.astype(self.dtype), sys.astype(F64)
        with Timer() as tm:
            dev = sw.diag.device
            n = sys.n_u
            if self.H is None:
                self.H = torch.zeros((self.n_total, 1), dtype=self.store_dtype, device=dev)
            known = ~sw.is_new
            X = supernode_init(sw, self._warm(sw), known, comp="fh")
            Hc = init_h(sw, self.H[sw.U].to(self.dtype), known, self.hmax or 1.0)
            Z = padded_empty(n, C + 1, self.dtype, dev)
            Z[:, :C] = X
            Z[:, C:] = Hc
            rhs = self._rhs_h(sw)
            ops, amg_box, hmax = FrontierOps(sw.W, C + 1, self.group), [None], self.hmax
            if hmax is None and n:  # first batch: get h before choosing the label tolerance
                M, wm = self._precond(sw, st, amg_box) if self.method == "amg" else (jacobi_M(sw), 0)
                Zh = padded_empty(n, 1, self.dtype, dev)
                Zh.copy_(Z[:, C:])
                Zh = pcg(sw, Zh, rhs[:, C:].contiguous(), [self.eps_h], M, self.max_iter, st, wm)
                Z[:, C:] = Zh
                hmax = float(Zh.max().item()) / (1 - self.eps_h)
            self.hmax = hmax = hmax or 1.0
            eps = [max(tol / (1.25 * hmax), self._floor())] * C + [max(self.eps_h, self._floor(hmax))]
            rhs64 = self._rhs_h(s64)
            rn = col_norms(rhs64[:, :C]).cpu().tolist() if self.target_relres is not None else None
            kw = {}
            if self.target_relres is not None:
                kw = dict(target_relres=self.target_relres, rhs_norm=rn + [1e300])
            Z = self._run(sw, Z, rhs, eps, ops, st, amg_box, **kw)
            Z64 = padded_empty(n, C + 1, F64, dev)
            Z64.copy_(Z)
            if n:
                Z64, R64, hmax, bound, rel = self._refine(sw, s64, Z64, rhs64, ops, st, amg_box,
                                                          10 if self.dtype == torch.float32 else 2, rn)
            else:
                R64, bound, rel = None, 0.0, 0.0
            st.cert, st.hmax, self.hmax, st.relres = bound, hmax, hmax, rel
            self._store(sw, Z64[:, :C])
            self.H[sw.U] = Z64[:, C:]
            self._Z64, self._R64 = Z64, R64
        st.edges += int(ops.edges)
        st.ms = tm.ms
        return st


class IncrementalLP(DynLPPlus):
    """Certified DynLP+ with resident state on a global-index system (dynlp/solvers.py:346-434).

    Keeps Z = [F, h] and its fp64 residual R between batches; a batch refreshes R on its changed
    rows only (one fused SpMM over those rows), small changes are repaired by push and larger ones
    by the working-precision PCG correction with fp64 refinement; R is recomputed in full every
    `full_every` batches to bound drift."""

    def __init__(self, n_total, K, dtype="float32", tol=1e-3, full_every=16, max_rounds=50_000, method="auto",
                 class_sum="auto", **kw):
        # auto: where dropping a class column shortens the rows to a whole number of 16-byte vectors
        # of at most 12 floats (K = 4, 8, 12: one load fewer per gathered row); measured on B200 at
        # K = 8 (18.6 iterations at 0.156 ms against 17.65 at 0.216) and, at K = 32 with no whole-row
        # layout either way, slower than solving every column
        if class_sum == "auto":
            class_sum = K % 4 == 0 and K <= 12
        super().__init__(n_total, K, dtype, method=method, tol=tol, class_sum=class_sum, **kw)
        self.name, self.full_every, self.max_rounds = "dynlp+inc", full_every, max_rounds
        self.Z = self.R = None
        self.since_full = 0

    def _full_residual(self, s64, st):
        self.R = residual(s64, self.Z, self._rhs_h(s64), out=self.R)
        st.edges += s64.nnz
        self.since_full = 0

    def _push(self, s64, eps, st):
        """Repair the violating rows of R (dynlp/solvers.py:375-389): the fused asynchronous push
        for up to 33 columns, the synchronous vectorised push beyond."""
        Z, R = self.Z, self.R
        eps_d = torch.as_tensor(eps, dtype=F64, device=Z.device)
        if Z.shape[1] <= 33:
            if getattr(self, "_fused", None) is None or self._fused.W is not s64.W:
                self._fused = kernels.FusedPush(s64.W, Z.shape[1], self.group)
            cand = kernels.flatnonzero(kernels.violating(R, s64.diag, eps_d))
            rounds, ok, edges = self._fused.run(Z, R, s64.diag, eps_d, cand, self.max_rounds)
            st.iters, st.edges = st.iters + rounds, st.edges + edges
            return ok
        ops = FrontierOps(s64.W, Z.shape[1], self.group)
        ok = push(s64, Z, R, eps, ops, st, max_iter=self.max_rounds)[2]
        st.edges += int(ops.edges)
        return ok

    def _park(self, s64, rows):
        if rows is not None and rows.numel():
            h0 = float(self.hmax or 1.0)
            sol = s64.solved.view(torch.uint8) if s64.solved.dtype == torch.bool else s64.solved.to(torch.uint8)
            _lib.call("dlp_park_rows", ptr(rows), int(rows.numel()), ptr(sol), self.C, 1,
                      ptr(s64.prior.to(F64).contiguous()), h0, ptr(self.Z), ld(self.Z), ptr(self.R), ld(self.R),
                      stream())

    def solve(self, sys):
        if sys.solved is None:
            raise ValueError("dynlp+inc needs a global-index system (EdgeStream)")
        s64, C, tol, st = sys.astype(F64), self.C, self.tol, Stats(path="inc-push")
        sw = sys.astype(self.dtype)
        with Timer() as tm:
            rhs64 = self._rhs_h(s64)
            if self.Z is None:
                inner = DynLPPlus.solve(self, sys)
                st.iters, st.edges, st.setup_ms, st.path = inner.iters, inner.edges, inner.setup_ms, "inc-" + inner.path
                self.Z, self.R = self._Z64, self._R64
                st.cert, st.hmax, st.relres = inner.cert, inner.hmax, inner.relres
                self.since_full = 0
            else:
                self._park(s64, sys.moved)
                if s64.comps:  # vertex arrivals: new rows start at their component's average
                    known = s64.solved & ~s64.is_new
                    supernode_init(s64, self.Z[:, :C], known, comp="fh")
                    init_h(s64, self.Z[:, C:], known, self.hmax or 1.0)
                Q = sys.changed
                if Q is not None and Q.numel():
                    residual(s64, self.Z, rhs64, out=self.R, rows=Q)
                    st.edges += int(Q.numel()) * max(int(s64.nnz / max(s64.n_u, 1)), 1)
                self.since_full += 1
                if self.since_full >= self.full_every:
                    self._full_residual(s64, st)
                amg_box = [None]
                ops = FrontierOps(sw.W, C + 1, self.group)
                # one pass: rho_cols, ||R_c||^2, ||rhs_c||^2 and max h
                stats = residual_stats(s64, self.R, rhs=rhs64 if self.target_relres is not None else None,
                                       H=self.Z[:, C:])
                rc, ss, bb, h_est = stats
                rn = [b ** 0.5 for b in bb[:C]] if bb is not None else None
                hmax, bound = self._bound(rc, h_est)
                ok_rel, rel = self._relres_ok(ss, rn)
                st.path = "inc-none"
                if not (bound <= tol and ok_rel):
                    small = False
                    if self.target_relres is None and self.method in ("auto", "push"):
                        eps = [tol / (1.25 * (self.hmax or 1.0))] * C + [self.eps_h]
                        eps_d = torch.as_tensor(eps, dtype=F64, device=self.Z.device)
                        nviol = int(kernels.violating(self.R, s64.diag, eps_d).sum().item())
                        small = nviol / max(s64.n_solved, 1) <= self.push_frac
                    if small:
                        st.path = "inc-push"
                        for _ in range(4):
                            ok = self._push(s64, eps, st)
                            rc2, _, _, h2 = residual_stats(s64, self.R, H=self.Z[:, C:])
                            hmax, bound = self._bound(rc2, h2)
                            if ok and bound <= tol:
                                break
                            eps = [tol / (1.25 * hmax)] * C + [self.eps_h]
                        rel = float("nan")
                        stats = None
                    if not (bound <= tol and small):
                        st.path = "inc-" + ("pcg" if self.method in ("auto", "pcg", "push") else self.method)
                        self.Z, self.R, hmax, bound, rel = self._refine(sw, s64, self.Z, rhs64, ops, st, amg_box, 10,
                                                                        rn, R64=self.R, stats=stats)
                st.cert, st.hmax, self.hmax, st.relres = bound, hmax, hmax, rel
            self.F, self.H = self.Z[:, :C], self.Z[:, C:]
        st.ms = tm.ms
        return st


    def relabel(self, sys):
        """Labels after the last solve (predict, dynlp/solvers.py:166-167) on every row of the
        global-index system (-1 outside the solved set), and the rows whose label changed since the
        previous call. Returns device tensors (labels, changed rows, their labels, count[1]); the
        first `count` entries of the two lists are valid. No host read."""
        Z = self.Z
        n, dev = Z.shape[0], Z.device
        if getattr(self, "_labels", None) is None or self._labels.numel() != max(n, 1):
            self._labels = torch.full((max(n, 1),), -2, dtype=torch.int32, device=dev)
            self._chg = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
            self._chg_lab = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
            self._nchg = torch.zeros(1, dtype=torch.int32, device=dev)
        sol = sys.solved.view(torch.uint8) if sys.solved.dtype == torch.bool else sys.solved.to(torch.uint8)
        ws = workspace("predict").get(_lib.lib().dlp_predict_workspace_bytes(n))
        _lib.call("dlp_predict", n, self.C, ptr(Z), ld(Z), code(Z), int(self.K == 2), ptr(sol), ptr(self._labels),
                  ptr(self._chg), ptr(self._chg_lab), ptr(self._nchg), ptr(ws), ws.numel(), stream())
        return self._labels[:n], self._chg, self._chg_lab, self._nchg


class PlainFP32LP(Solver):
    """The plain FP32 path the serving loop is measured against: scores kept in fp32 on the global-index
    system and every batch solved by fp32 Jacobi-PCG from the previous scores until the fp32 relative
    residual meets the target -- no fp64 residual, no refinement (the reference's solver run in one
    precision, dynlp/solvers.py:66-97). `relres` is still reported against the fp64 system."""

    name = "plain-fp32"

    def __init__(self, n_total, K, target_relres=1e-6, max_iter=100_000):
        super().__init__(n_total, K, "float32")
        self.target_relres, self.max_iter = target_relres, max_iter
        self.Z = None

    def solve(self, sys):
        st = Stats(path="plain-fp32")
        sw = sys.astype(torch.float32)
        with Timer() as tm:
            n, C = sw.rhs.shape[0], self.C
            if self.Z is None:
                self.Z = padded_empty(n, C, torch.float32, sw.diag.device, fill=0.0)
                self.Z[:] = torch.where(sw.solved[:, None], sw.prior.to(torch.float32)[None, :], torch.zeros_like(self.Z))
            if sys.moved is not None and sys.moved.numel():  # rows entering U start at the prior, rows leaving at 0
                mv = sys.moved.long()
                self.Z[mv] = torch.where(sys.solved[mv, None], sw.prior.to(torch.float32)[None, :],
                                         torch.zeros_like(self.Z[mv]))
            rhs = sw.rhs.contiguous()
            pcg(sw, self.Z, rhs, None, jacobi_M(sw), self.max_iter, st, target_relres=self.target_relres)
            s64 = sys.astype(F64)
            R = residual(s64, self.Z.double(), s64.rhs.contiguous())
            st.relres = float((col_norms(R) / torch.clamp(col_norms(s64.rhs), min=1e-300)).max())
        st.ms = tm.ms
        self.F = self.Z
        return st

    def relabel(self, sys):
        """Labels of every row (-1 outside the solved set) and the rows whose label changed."""
        return IncrementalLP.relabel(self, sys)


class Reference:
    """High-accuracy float64 solution F* and absorption bound (dynlp/solvers.py:437-445)."""

    def __init__(self, n_total, K, tol=1e-8, method="pcg"):
        self.inner = DynLPPlus(n_total, K, "float64", method=method, tol=tol, eps_h=1e-6, max_iter=100_000)

    def solve(self, sys):
        st = self.inner.solve(sys)
        return self.inner.scores(sys), self.inner.hmax, st


def make(name, n_total, K, *, dtype, delta, tol, group, max_iter=None):
    """dynlp/solvers.py:448-458."""
    kw = {} if max_iter is None else {"max_iter": max_iter}
    if name == "itlp":
        return ItLP(n_total, K, dtype, delta, **kw)
    if name in ("dynlp", "dynlp-fh"):
        return DynLP(n_total, K, dtype, delta, group, comp="fh" if name == "dynlp-fh" else "tau", **kw)
    if name == "dynlp+inc":
        return IncrementalLP(n_total, K, dtype, tol=tol, group=group, **kw)
    if name.startswith("dynlp+"):
        return DynLPPlus(n_total, K, dtype, method=name.split("+", 1)[1], tol=tol, group=group, **kw)
    raise ValueError(f"unknown solver {name!r}")


SOLVERS = ["itlp", "dynlp", "dynlp-fh", "dynlp+pcg", "dynlp+amg", "dynlp+auto", "dynlp+inc"]

"""The per-batch linear system and the edge-update stream (mirrors dynlp/stream.py).

Per batch, the harmonic system on the active unlabelled set U (dynlp/stream.py:1-6):
    (diag - W_UU) F_U = rhs,   diag = s + rowsum(W_UU),   s = w(u, L) + eta
Binary problems solve one column (class 1); K classes solve K columns.

* `System`: the reference's dataclass (stream.py:17-58) with torch tensors.
* `build_system`: `Stream._build` (stream.py:142-177) on the device: grounding by connected
  components with the labelled vertices as a sink, U x U filter in CSR order, B = A @ onehot.
* `ResidentGraph`: the graph kept on the device with per-row slack so edges can be inserted in
  place; it is accepted as `W` by every row kernel.
* `EdgeStream`: the resident global-index system (the `IncrementalStream` form, stream.py:180-346:
  inert rows have diag 1, rhs 0 and no live entries) updated by edge batches through
  `apply_edges`, the new entry point of the edge-update workload.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np
import torch

from . import _lib, cc, kernels
from .backend import CSR, code, ld, ptr, stream, to_dtype, workspace
from .graphs import Dataset, csr_rows


@dataclass
class System:
    t: int
    U: torch.Tensor          # global ids of the rows (sorted)
    W: object                # CSR U x U (or the resident graph for global-index systems)
    s: torch.Tensor          # grounding
    diag: torch.Tensor       # s + rowsum(W)
    B: torch.Tensor          # (n_u, K) weight to labelled neighbours per class
    rhs: torch.Tensor        # (n_u, C)
    prior: torch.Tensor      # (C,)
    is_new: torch.Tensor     # rows not in U at the previous batch
    seed: torch.Tensor       # rows whose equation changed (DynLP's affected set)
    comps: dict
    K: int
    C: int
    eta: float
    n_inserted: int
    n_deleted: int
    n_active: int
    n_ungrounded: int = 0
    solved: object = None    # global-index systems: rows really solved (others inert)
    changed: object = None   # global-index systems: rows whose equation changed
    moved: object = None     # global-index systems: rows that entered or left U this batch
    rhs_h: object = None     # (n, C+1) [rhs | diag], the DynLP+ right-hand side with the h column
    _conv: dict = field(default_factory=dict, repr=False, compare=False)

    n_u = property(lambda self: int(self.U.numel()))
    nnz = property(lambda self: int(self.W.nnz))

    @property
    def n_solved(self) -> int:
        return self.n_u if self.solved is None else int(self.solved.sum().item())

    def label_cols(self, M):
        """Columns of a (., K) class matrix that are solved (class 1 if binary)."""
        return M[:, 1:2] if self.K == 2 else M

    def astype(self, dtype) -> "System":
        """Same system in another precision (cached; index arrays shared) (stream.py:49-58)."""
        dt = to_dtype(dtype)
        if dt == self.diag.dtype:
            return self
        if dt not in self._conv:
            cast = {k: getattr(self, k).to(dt) for k in ("s", "diag", "B", "rhs", "prior")}
            W = self.W.astype(dt) if isinstance(self.W, CSR) and dt != torch.float64 else self.W
            rh = self.rhs_h.to(dt) if self.rhs_h is not None else None
            self._conv[dt] = replace(self, W=W, rhs_h=rh, _conv={}, **cast)
        return self._conv[dt]


def _onehot_labels(y, lab_mask, K, dev):
    n = y.numel()
    X = torch.zeros((n, K), dtype=torch.float64, device=dev)
    li = torch.nonzero(lab_mask, as_tuple=False).flatten()
    X[li, y[li].long()] = 1.0
    return X


def _range_positions(beg, end):
    """Slot positions of the ranges [beg[i], end[i]) and each one's range index, in range order."""
    counts = (end.long() - beg.long()).clamp(min=0)
    seg = torch.repeat_interleave(torch.arange(beg.numel(), device=beg.device), counts)
    if not seg.numel():
        return torch.zeros(0, dtype=torch.int64, device=beg.device), seg
    excl = torch.cumsum(counts, 0) - counts
    return beg.long()[seg] + (torch.arange(seg.numel(), device=beg.device) - excl[seg]), seg


def new_components(m, lr, lc, w, tau, wmax, ground):
    """DynLP step 1 for m new vertices with the reference's arguments (dynlp/stream.py:67-81): every
    stored entry lr -> lc of their rows with its weight w (lc = -1 where the neighbour is not new).
    Each vertex's mean dissimilarity s over its live entries (w > 0) is summed in fp64 and rounded
    to fp32; the components are those over the live entries heavier than tau between new vertices
    ("tau") and the adaptive FH ones on 1 - w/wmax scaled by sqrt(s_u s_v) ("fh"); ground is each
    vertex's label weight. Returns {"tau": (labels, count), "fh": (labels, count)}."""
    dev = w.device if torch.is_tensor(w) else None
    lr = torch.as_tensor(lr, device=dev).long()
    lc = torch.as_tensor(lc, device=dev).long()
    w = torch.as_tensor(w, device=dev)
    dev = w.device
    if m == 0:
        z = torch.zeros(0, dtype=torch.int32, device=dev)
        return {"tau": (z, 0), "fh": (z, 0)}
    on = w > 0
    dis = torch.where(on, 1 - w.double() / wmax, torch.zeros((), dtype=torch.float64, device=dev))
    s = torch.zeros(m, dtype=torch.float64, device=dev).index_add_(0, lr, dis)
    cnt = torch.zeros(m, dtype=torch.float64, device=dev).index_add_(0, lr, on.double())
    s = (s / cnt.clamp(min=1)).float() + 1e-6
    e = on & (lc >= 0)
    r, c, we = lr[e], lc[e], w[e]
    heavy = we > tau
    gr = torch.as_tensor(ground, device=dev).to(torch.float32)
    return {"tau": cc.connected_components(m, r[heavy].to(torch.int32), c[heavy].to(torch.int32)),
            "fh": cc.adaptive_components(m, r, c, we, s[r], s[c], wmax, gr)}


def new_components_rows(rows, rbeg, rend, col, w, nl, tau, wmax, ground):
    """new_components over the rows of a CSR (the form the streams call), on the device:
    each one's mean dissimilarity s over its live entries (`dlp_new_dissim`, row order), then the
    components over edges heavier than tau between new vertices ("tau", the paper's) and the
    adaptive FH components on 1 - w/wmax scaled by sqrt(s_u s_v) ("fh"). `nl` maps a column id to
    its new-vertex index (-1: not new); `ground` is each new vertex's label weight."""
    m = int(rows.numel())
    dev = rows.device
    if m == 0:
        z = torch.zeros(0, dtype=torch.int32, device=dev)
        return {"tau": (z, 0), "fh": (z, 0)}
    rows = rows.to(torch.int32).contiguous()
    s = torch.empty(m, dtype=torch.float32, device=dev)
    _lib.call("dlp_new_dissim", ptr(rows), m, ptr(rbeg), ptr(rend), ptr(w), code(w), float(wmax), ptr(s), stream())
    pos, seg = _range_positions(rbeg[rows.long()], rend[rows.long()])
    wv = w[pos]
    c = nl[col[pos].long()]
    e = (wv > 0) & (c >= 0)
    r, c, we = seg[e], c[e].long(), wv[e]
    heavy = we > tau
    tau_c = cc.connected_components(m, r[heavy].to(torch.int32), c[heavy].to(torch.int32))
    fh_c = cc.adaptive_components(m, r, c, we, s[r], s[c], wmax, ground.to(torch.float32))
    return {"tau": tau_c, "fh": fh_c}


def build_system(ds: Dataset, active, labeled, *, eta=0.0, dtype="float32", t=0, prev_U=None, ins=0, dele=0,
                 ins_ids=None, del_ids=None, tau=None, wmax=None):
    """The grounded system of one batch (Stream._build, dynlp/stream.py:142-177), on the device.

    U = active unlabelled vertices whose component (within the active unlabelled subgraph) holds
    label weight; W = A[U, U] in CSR order; B = A @ onehot(y_L); s = sum(B) + eta; diag = s +
    rowsum(W); rhs = B (class 1 when K == 2) + eta * prior. With the batch's inserted / deleted
    vertex ids, DynLP's seed is the new rows plus the neighbours of those vertices; with tau and
    wmax the new vertices' components (tau and FH) are built too (dynlp/stream.py:170-175)."""
    A, K = ds.A, ds.K
    dev = A.indices.device
    n = A.shape[0]
    dt = to_dtype(dtype)
    active = active.to(torch.bool)
    labeled = labeled.to(torch.bool)
    al = active & labeled
    Bfull = kernels.spmm_axpy(A, _onehot_labels(ds.y, al, K, dev))  # fp64 (fp32 weights x fp64 onehot)
    vmask = (active & ~labeled).to(torch.uint8)
    parent, err = cc.graph_components(A, vmask, al.to(torch.uint8))
    root = parent[n]
    Um = vmask.bool() & (parent[:n] == root)
    n_ungrounded = int((vmask.bool() & ~Um).sum().item())
    U = torch.nonzero(Um, as_tuple=False).flatten()
    n_u = int(U.numel())
    loc = torch.full((n,), -1, dtype=torch.int64, device=dev)
    loc[U] = torch.arange(n_u, device=dev)
    rows = csr_rows(A).long()
    cols = A.indices.long()
    keep = Um[rows] & Um[cols]
    indptr = torch.zeros(n_u + 1, dtype=torch.int64, device=dev)
    indptr[1:] = torch.cumsum(torch.bincount(loc[rows[keep]], minlength=n_u), 0)
    W = CSR(A.data[keep].to(dt), loc[cols[keep]].to(torch.int32), indptr.to(torch.int32), (n_u, n_u))
    Bm = Bfull[U]
    s = Bm.sum(dim=1) + eta
    ones = torch.ones((n_u, 1), dtype=torch.float64, device=dev)
    rowsum = kernels.spmm_axpy(W if dt != torch.bfloat16 else W.astype(torch.float32), ones)[:, 0] if n_u else \
        torch.zeros(0, dtype=torch.float64, device=dev)
    diag = s + rowsum
    prior = torch.full((1 if K == 2 else K,), 0.5 if K == 2 else 1.0 / K, dtype=torch.float64, device=dev)
    rhs = (Bm[:, 1:2] if K == 2 else Bm) + eta * prior[None, :]
    is_new = torch.ones(n_u, dtype=torch.bool, device=dev) if prev_U is None else ~prev_U[U]
    seed = is_new.clone()
    if ins_ids is not None or del_ids is not None:
        touch = torch.zeros((n, 1), dtype=torch.float64, device=dev)
        for ids in (ins_ids, del_ids):
            if ids is not None and ids.numel():
                touch[ids.long(), 0] = 1.0
        seed |= kernels.spmm_axpy(A, touch)[U, 0] > 0
        ins, dele = (int(ins_ids.numel()) if ins_ids is not None else ins), \
            (int(del_ids.numel()) if del_ids is not None else dele)
    comps = {}
    if tau is not None:
        new = torch.nonzero(is_new, as_tuple=False).flatten()
        nl = torch.full((n_u,), -1, dtype=torch.int64, device=dev)
        nl[new] = torch.arange(new.numel(), device=dev)
        Wd = W.data.to(dt)
        comps = new_components_rows(new, W.indptr[:-1], W.indptr[1:], W.indices, Wd, nl, tau, wmax,
                               Bm[new].to(dt).sum(dim=1))
    sysd = dict(t=t, U=U, W=W, s=s.to(dt), diag=diag.to(dt), B=Bm.to(dt), rhs=rhs.to(dt).contiguous(),
                prior=prior.to(dt), is_new=is_new, seed=seed, comps=comps, K=K, C=1 if K == 2 else K, eta=eta,
                n_inserted=ins, n_deleted=dele, n_active=int(active.sum().item()), n_ungrounded=n_ungrounded)
    sysd["rhs_h"] = torch.cat([sysd["rhs"], sysd["diag"][:, None]], dim=1).contiguous()
    S = System(**sysd)
    if dt != torch.float64:
        S._conv[torch.float64] = System(**{**sysd, "W": CSR(W.data.to(torch.float32), W.indices, W.indptr, W.shape),
                                           "s": s, "diag": diag, "B": Bm, "rhs": rhs.contiguous(),
                                           "prior": prior, "rhs_h": torch.cat([rhs, diag[:, None]], 1).contiguous()})
    return S


class ResidentGraph:
    """Slack-padded rows on the device. Row r owns slots [rbeg[r], rcap[r]); [rbeg[r], rend[r]) are
    stored entries. `aw` = edge weights (0 = deleted), `data` = the solver operator W_UU."""

    def __init__(self, A: CSR, slack_frac=0.25, slack_min=8):
        self._build_from(A.indptr, A.indices, A.data.to(torch.float32), A.shape[0], slack_frac, slack_min)

    def _build_from(self, indptr, indices, aw, n, slack_frac, slack_min):
        dev = indices.device
        indptr = indptr.long()
        deg = torch.diff(indptr)
        cap = deg + torch.clamp((deg.double() * slack_frac).ceil().long(), min=slack_min)
        rbeg = torch.zeros(n, dtype=torch.int64, device=dev)
        if n > 1:
            rbeg[1:] = torch.cumsum(cap, 0)[:-1]
        total = int(cap.sum().item()) if n else 0
        if total >= 2**31:
            raise ValueError("graph too large for int32 slot offsets")
        rows = torch.repeat_interleave(torch.arange(n, device=dev), deg)
        pos = rbeg[rows] + (torch.arange(indices.numel(), device=dev) - indptr[rows])
        self.indices = torch.full((max(total, 1),), -1, dtype=torch.int32, device=dev)
        self.aw = torch.zeros(max(total, 1), dtype=torch.float32, device=dev)
        self.indices[pos] = indices.to(torch.int32)
        self.aw[pos] = aw
        self.data = torch.zeros_like(self.aw)
        self.rbeg = rbeg.to(torch.int32)
        self.rend = (rbeg + deg).to(torch.int32)
        self.rcap = (rbeg + cap).to(torch.int32)
        self.shape = (n, n)
        self.slack_frac, self.slack_min = slack_frac, slack_min
        self._slot_rows = None

    @property
    def nnz(self) -> int:
        return int((self.rend - self.rbeg).sum().item())

    @property
    def dtype(self):
        return self.data.dtype

    def astype(self, dtype):
        return self

    def slot_rows(self):
        """Row of every slot (for setup-time masking)."""
        cap = (self.rcap - self.rbeg).long()
        return torch.repeat_interleave(torch.arange(self.shape[0], device=self.rbeg.device), cap)

    def rebuild(self, grow=2.0):
        """Repack with more slack (after a row overflowed); tombstones are dropped."""
        n = self.shape[0]
        slots = self.slot_rows()
        rbeg_l = self.rbeg.long()[slots]
        j = torch.arange(slots.numel(), device=slots.device)
        live = (j < self.rend.long()[slots]) & (self.aw[: slots.numel()] != 0)
        rows = slots[live]
        deg = torch.bincount(rows, minlength=n)
        indptr = torch.zeros(n + 1, dtype=torch.int64, device=slots.device)
        indptr[1:] = torch.cumsum(deg, 0)
        del rbeg_l
        w_live = self.data[: slots.numel()][live]
        self._build_from(indptr, self.indices[: slots.numel()][live], self.aw[: slots.numel()][live], n,
                         self.slack_frac * grow + 0.25, max(self.slack_min * 2, 4))
        slots = self.slot_rows()
        j = torch.arange(slots.numel(), device=slots.device)
        live_new = j < self.rend.long()[slots]
        self.data[: slots.numel()][live_new] = w_live

    def to_csr(self, which="aw", drop_zero=True) -> CSR:
        """Compact CSR of the stored entries (column order within rows as stored)."""
        n = self.shape[0]
        slots = self.slot_rows()
        j = torch.arange(slots.numel(), device=slots.device)
        vals = (self.aw if which == "aw" else self.data)[: slots.numel()]
        live = j < self.rend.long()[slots]
        if drop_zero:
            live &= vals != 0
        rows = slots[live]
        indptr = torch.zeros(n + 1, dtype=torch.int64, device=slots.device)
        indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n), 0)
        return CSR(vals[live].clone(), self.indices[: slots.numel()][live].clone(), indptr.to(torch.int32), (n, n))


class EdgeStream:
    """The resident grounded system under edge-update batches (global vertex ids).

    Mirrors IncrementalStream (dynlp/stream.py:180-346) for an edge stream: every vertex keeps its
    global id, rows outside U (labelled or in a component without labels) are inert (diag 1, rhs 0,
    no live solver entries), and each batch is applied in place on the device:
      1. deletions, then insertions, into the resident graph (weights, row sums, label weights);
      2. connected components of the unlabelled subgraph with the labelled vertices as a sink: the
         vertices whose component holds no label leave U, newly grounded ones enter it;
      3. the equations (s, diag, rhs and the h column's rhs) of every changed row are rebuilt.
    `system` is a System whose arrays stay live until the next batch; `changed` lists the rows whose
    equation changed and `moved` the rows that entered or left U.
    """

    def __init__(self, ds: Dataset, labeled, *, eta_rel=0.0, dtype="float32", with_h=True, slack_frac=0.25, slack_min=8,
                 active=None, components=False):
        A, K = ds.A, ds.K
        self.ds, self.K, self.dtype = ds, K, to_dtype(dtype)
        self.C = 1 if K == 2 else K
        self.col0 = 1 if K == 2 else 0
        self.with_h = with_h
        n = A.shape[0]
        dev = A.indices.device
        self.n, self.dev = n, dev
        self.G = ResidentGraph(A, slack_frac=slack_frac, slack_min=slack_min)
        labeled = labeled.to(torch.bool)
        active = torch.ones(n, dtype=torch.bool, device=dev) if active is None else active.to(torch.bool)
        self.active, self.labeled_all = active.clone(), labeled.clone()
        self.labeled = (labeled & active).to(torch.uint8)
        self.vmask = (active & ~labeled).to(torch.uint8)
        self.y = ds.y.to(torch.int32).contiguous()
        self.eta = float(eta_rel * float(A.data.double().sum().item()) / max(n, 1))
        self.prior64 = torch.full((self.C,), 0.5 if K == 2 else 1.0 / K, dtype=torch.float64, device=dev)
        # label weights B = A @ onehot(y_L) (fp64)
        self.B = kernels.spmm_axpy(A, _onehot_labels(self.y, self.labeled.bool(), K, dev)).contiguous()
        # grounding and the masked operator
        self.umask = torch.zeros(n, dtype=torch.uint8, device=dev)
        self.in_t = torch.zeros(n, dtype=torch.uint8, device=dev)
        self.changed = torch.zeros(n, dtype=torch.uint8, device=dev)
        self._squeeze = torch.zeros(n, dtype=torch.uint8, device=dev)  # rows to squeeze after deletions
        self._stat = torch.zeros(8, dtype=torch.int32, device=dev)
        self.counters = {"rebuilds": 0, "ground_changes": 0, "applied": 0, "ground_sweeps": 0, "ground_fallbacks": 0}
        self._ground()
        sr = self.G.slot_rows()
        um = self.umask.bool()
        colv = self.G.indices[: sr.numel()].long().clamp(min=0)
        self.G.data[: sr.numel()] = torch.where(um[sr] & um[colv], self.G.aw[: sr.numel()],
                                                torch.zeros_like(self.G.aw[: sr.numel()]))
        self.rowsum = torch.zeros(n, dtype=torch.float64, device=dev)
        _lib.call("dlp_graph_rowsum", ptr(self.G.rbeg), ptr(self.G.rend), ptr(self.G.data), None, n,
                  ptr(self.rowsum), stream())
        ch = self.C + (1 if with_h else 0)
        self.ld64 = ch + (ch & 1)
        self.ld32 = (ch + 3) // 4 * 4
        self.diag64 = torch.empty(n, dtype=torch.float64, device=dev)
        self.rhs64 = torch.zeros((n, self.ld64), dtype=torch.float64, device=dev)
        self.diag32 = torch.empty(n, dtype=torch.float32, device=dev)
        self.rhs32 = torch.zeros((n, self.ld32), dtype=torch.float32, device=dev)
        self._system_rows(None, n)
        self.t = 0
        # connected components of the active unlabelled subgraph after every batch (the reference
        # labels them in Stream._build, dynlp/stream.py:150-153): computed on a side stream that
        # overlaps the solve; the next batch's patch waits for it
        self.with_components = bool(components)
        self._cc_done = None
        if self.with_components:
            self._cc_stream = torch.cuda.Stream(device=dev)
            self._cc_parent = torch.empty(n + 1, dtype=torch.int32, device=dev)
            self._cc_label = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
            self._cc_counts = torch.zeros(3, dtype=torch.int32, device=dev)  # n_comp, n_masked, error
            # the warm labelling's state between batches (its search seed): zeroed once
            self._cc_ws = torch.zeros(int(_lib.lib().dlp_cc_graph_warm_workspace_bytes(n)), dtype=torch.uint8,
                                      device=dev)
            self._components_launch()
        self.last_changed = torch.arange(n, dtype=torch.int32, device=dev)
        self.last_moved = torch.zeros(0, dtype=torch.int32, device=dev)
        self.n_ins = self.n_del = 0

    # -- helpers -------------------------------------------------------------------------------
    def _ground(self):
        """umask = grounded unlabelled vertices; in_t flags membership changes; returns #changes.

        The grounding check of dynlp/stream.py:150-159 (components of the unlabelled subgraph with
        the labelled vertices as a sink) as reachability from the sink: the same set without a full
        labelling of the components."""
        changes, sweeps = cc.ground_reach(self.G, self.vmask, self.labeled, self.umask, self.in_t, w=self.G.aw)
        self.counters["ground_sweeps"] += abs(sweeps)
        self.counters["ground_fallbacks"] += sweeps < 0
        self._stat[4].fill_(changes)
        return changes

    def _components_launch(self):
        """Queue the component labelling of the current graph on the side stream."""
        G, n = self.G, self.n
        main = torch.cuda.current_stream(self.dev)
        side = self._cc_stream
        side.wait_stream(main)
        with torch.cuda.stream(side):
            _lib.call("dlp_cc_graph_warm", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.aw), code(G.aw),
                      ptr(self.vmask), ptr(self._cc_parent), ptr(self._cc_counts[2:3]), ptr(self._cc_ws),
                      self._cc_ws.numel(), stream())
            wl = workspace("cc_labels").get(_lib.lib().dlp_cc_mask_labels_workspace_bytes(n))
            _lib.call("dlp_cc_mask_labels", n, ptr(self._cc_parent), ptr(self.vmask), ptr(self._cc_label),
                      ptr(self._cc_counts[0:1]), ptr(self._cc_counts[1:2]), ptr(wl), wl.numel(), stream())
            self._cc_done = torch.cuda.Event()
            self._cc_done.record(side)

    def join_components(self):
        """Make the current stream wait for this batch's component labelling (no host wait)."""
        if self._cc_done is not None:
            torch.cuda.current_stream(self.dev).wait_event(self._cc_done)

    def components(self):
        """(labels, n_comp) of the active unlabelled subgraph after the last batch, numbered as the
        reference's connected_components numbers them over its local ids (dynlp/stream.py:150-153,
        dynlp/cc.py:22): labels[i] belongs to the i-th active unlabelled vertex in ascending id order.
        Device int32 labels; one host read for the counts."""
        if not self.with_components:
            raise RuntimeError("EdgeStream(..., components=True) computes the component labels")
        self.join_components()
        n_comp, n_masked, err = self._cc_counts.tolist()
        if err:
            raise RuntimeError("component labelling: entry column outside [0, n)")
        return self._cc_label[:n_masked], n_comp

    def _system_rows(self, rows, nr):
        ch = self.C + (1 if self.with_h else 0)
        _lib.call("dlp_system_rows", ptr(rows), nr, ptr(self.umask), ptr(self.B), self.K, ptr(self.rowsum),
                  self.eta, ptr(self.prior64), self.C, self.col0, int(self.with_h), ptr(self.diag64),
                  ptr(self.rhs64), self.ld64, ptr(self.diag32), ptr(self.rhs32), self.ld32, stream())
        del ch

    def _upload(self, x, dt):
        if x is None:
            return None
        if torch.is_tensor(x):
            return x.to(device=self.dev, dtype=dt, non_blocking=True).contiguous()
        t = torch.from_numpy(np.ascontiguousarray(x)).to(dt)
        if torch.cuda.is_available():
            t = t.pin_memory()
        return t.to(self.dev, non_blocking=True)

    # -- the batch -----------------------------------------------------------------------------
    def apply_edges(self, ins_u=None, ins_v=None, ins_w=None, del_u=None, del_v=None, keep_pending=False) -> System:
        """Apply one edge batch (deletions, then insertions) and return the updated system.

        keep_pending: the previous batch has not been solved yet (several batches patched before one
        solve): its changed and moved rows stay in this batch's lists, so the solve refreshes the
        equations and residuals of every row any of the batches touched."""
        G, n = self.G, self.n
        self._vertex_batch = None
        for name, x in (("ins_u", ins_u), ("ins_v", ins_v), ("del_u", del_u), ("del_v", del_v)):
            if x is not None and not torch.is_tensor(x) and len(x) and (np.min(x) < 0 or np.max(x) >= n):
                raise ValueError(f"edge batch rejected: {name} has vertex ids outside [0, {n})")
        du, dv = self._upload(del_u, torch.int32), self._upload(del_v, torch.int32)
        iu, iv = self._upload(ins_u, torch.int32), self._upload(ins_v, torch.int32)
        iw = self._upload(ins_w, torch.float32)
        nd = int(du.numel()) if du is not None else 0
        ni = int(iu.numel()) if iu is not None else 0
        self.join_components()  # the previous batch's labelling reads the graph this batch patches
        prev_moved = self.last_moved if keep_pending else None
        if not keep_pending:
            self.changed.zero_()
        self._stat.zero_()
        st = self._stat  # [error, overflow, deleted, inserted, ground changes, ground error, changed rows, -]
        s = stream()
        if nd:
            _lib.call("dlp_graph_delete", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.aw), ptr(G.data), ptr(du),
                      ptr(dv), nd, ptr(self.umask), ptr(self.labeled), ptr(self.y), self.K, ptr(self.rowsum),
                      ptr(self.B), ptr(self.changed), ptr(st[2:3]), ptr(st[0:1]), ptr(self._squeeze), s)
        # Everything below is queued in dependency order before one host read of every flag and
        # count: the insertion, the grounding (its sweeps synchronise internally), the membership
        # toggle of the rows it flagged, the changed rows and the solver CSR. An overflow (rare)
        # undoes the toggle, repacks and redoes the rest.
        for attempt in range(4):
            if ni:
                self._insert(iu, iv, iw, ni)
            if self.with_components:
                self._components_launch()
            self._ground_launch()
            self._toggle_flagged()
            mv, _ = kernels.flatnonzero(self.in_t, count=st[7:8], sync=False)
            Qb, _ = kernels.flatnonzero(self.changed, count=st[6:7], sync=False)
            self._csr_launch()
            self._queue_counts()
            flags = self._read_counts()
            if flags["overflow"] == 0:
                break
            self.join_components()
            # back to the batch's start membership: umask before the grounding, then the same rows
            # toggled again put their weights and their neighbours' row sums back
            self.umask.bitwise_xor_(self.in_t)
            self._toggle_flagged()
            G.rebuild()  # a row ran out of slack: repack with more and apply the insertions again
            self.counters["rebuilds"] += 1
            st[1].zero_()
            st[3:8].zero_()  # counts the next attempt makes again
        else:
            raise RuntimeError("edge insertion kept overflowing after repacking")
        if flags["error"]:
            raise ValueError(f"edge batch rejected: {_lib.STATUS.get(flags['error'])} (vertex id out of range?)")
        if flags["ground_error"]:
            raise ValueError("grounding: entry column outside [0, n)")
        nmoved = flags["moved"]
        self.counters["ground_sweeps"] += abs(self._sweeps.value)
        self.counters["ground_fallbacks"] += self._sweeps.value < 0
        moved = mv[:nmoved]
        if nmoved:
            self.counters["ground_changes"] += nmoved
        self._counts = [flags["active"], flags["ungrounded"]]
        nq, nnz = flags["changed"], flags["nnz"]
        self.t += 1
        self._csr_set(nnz)
        Q = Qb[:nq]
        self._system_rows(Q, nq)
        if prev_moved is not None and prev_moved.numel():
            moved = torch.cat([prev_moved, moved])  # parked again by the solve: idempotent
        self.last_changed, self.last_moved = Q, moved
        self.n_ins, self.n_del = ni, nd
        self.counters["applied"] += flags["deleted"] + flags["inserted"]
        return self.system

    def _insert(self, iu, iv, iw, ni):
        G, st = self.G, self._stat
        ws = workspace("insert").get(_lib.lib().dlp_graph_insert_workspace_bytes(ni))
        _lib.call("dlp_graph_insert", self.n, ptr(G.rbeg), ptr(G.rend), ptr(G.rcap), ptr(G.indices), ptr(G.aw),
                  ptr(G.data), ptr(iu), ptr(iv), ptr(iw), ni, ptr(self.umask), ptr(self.labeled), ptr(self.y),
                  self.K, ptr(self.rowsum), ptr(self.B), ptr(self.changed), ptr(st[1:2]), ptr(st[3:4]),
                  ptr(st[0:1]), ptr(ws), ws.numel(), stream())

    def _ground_launch(self):
        """The grounding check (reachability from the labelled vertices through unlabelled ones,
        dynlp/stream.py:150-159): umask and in_t updated, the number of membership changes counted
        into the batch's stat word 4 (its sweeps synchronise the stream internally)."""
        import ctypes as ct
        G, n, st = self.G, self.n, self._stat
        self._sweeps = ct.c_int32(0)
        ws = workspace("ground_reach").get(_lib.lib().dlp_ground_reach_workspace_bytes(n))
        _lib.call("dlp_ground_reach", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.aw), code(G.aw),
                  ptr(self.vmask), ptr(self.labeled), ptr(self.umask), ptr(self.in_t), ptr(st[4:5]), ptr(st[5:6]),
                  ct.addressof(self._sweeps), ptr(ws), ws.numel(), stream())

    def _toggle_flagged(self):
        """Membership change of every row the grounding flagged in in_t (dlp_graph_toggle without a
        list; nothing to do when no row moved)."""
        G = self.G
        _lib.call("dlp_graph_toggle", ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.aw), ptr(G.data), None, self.n,
                  ptr(self.in_t), ptr(self.umask), ptr(self.rowsum), ptr(self.changed), stream())

    def _queue_counts(self):
        """Queue the active and ungrounded vertex counts of the batch's final membership on the
        device (no host read: they come back with the batch's flags in _read_counts)."""
        um = self.umask.view(torch.bool)
        if getattr(self, "_cnt_dev", None) is None:
            self._cnt_dev = torch.zeros(2, dtype=torch.int64, device=self.dev)
        self._cnt_dev[0] = self.vmask.sum() + self.labeled.sum()
        self._cnt_dev[1] = (self.vmask.view(torch.bool) & ~um).sum()

    def _read_counts(self):
        """One host read of the batch's flags and counts (the solver CSR's entry count, and the
        active and ungrounded counts when queued)."""
        if getattr(self, "_h_stat", None) is None:
            self._h_stat = torch.zeros(9, dtype=torch.int32, pin_memory=torch.cuda.is_available())
            self._h_cnt = torch.zeros(2, dtype=torch.int64, pin_memory=torch.cuda.is_available())
        h = self._h_stat
        h[0:8].copy_(self._stat, non_blocking=True)
        h[8:9].copy_(self._csr_ptr[self.n:self.n + 1], non_blocking=True)
        cnt = getattr(self, "_cnt_dev", None)
        if cnt is not None:
            self._h_cnt.copy_(cnt, non_blocking=True)
        torch.cuda.current_stream(self.dev).synchronize()
        v = h.tolist()
        out = {"error": v[0], "overflow": v[1], "deleted": v[2], "inserted": v[3], "moved": v[7],
               "ground_error": v[5], "changed": v[6], "nnz": v[8]}
        if cnt is not None:
            out["active"], out["ungrounded"] = self._h_cnt.tolist()
        return out

    def apply_vertices(self, ins, dele, tau=None, wmax=None) -> System:
        """One vertex-arrival batch (IncrementalStream.batches, dynlp/stream.py:300-346): the
        vertices `dele` leave the active set, then `ins` join it (labelled ones move their label
        weight onto their neighbours' B rows, dynlp/stream.py:230-235); the grounded set is
        re-checked, membership changes toggle the solver weights (:206-228) and every changed
        row's equation is rebuilt. The system carries the new rows (in U now, not at the previous
        batch), DynLP's seed (new rows and the neighbours of the batch's vertices, within U) and,
        with tau / wmax, the new vertices' components over the masked weights (:336-339)."""
        G, n, dev, s = self.G, self.n, self.dev, stream()
        ins = ins.to(device=dev, dtype=torch.int64)
        dele = dele.to(device=dev, dtype=torch.int64)
        prev_u = self.umask.bool().clone()
        self._vertex_batch = None
        self.join_components()
        self.changed.zero_()
        lab_all = self.labeled_all
        for ids, on in ((dele, False), (ins, True)):
            if not ids.numel():
                continue
            self.active[ids] = on
            L = ids[lab_all[ids]].to(torch.int32).contiguous()
            V = ids[~lab_all[ids]]
            self.vmask[V] = 1 if on else 0
            if L.numel():
                self.labeled[L.long()] = 1 if on else 0
                _lib.call("dlp_label_update", ptr(L), int(L.numel()), 1.0 if on else -1.0, ptr(G.rbeg), ptr(G.rend),
                          ptr(G.indices), ptr(G.aw), ptr(self.y), self.K, ptr(self.B), ptr(self.umask),
                          ptr(self.changed), s)
        if self.with_components:
            self._components_launch()
        nmoved = self._ground()
        moved = torch.zeros(0, dtype=torch.int32, device=dev)
        if nmoved:
            moved = kernels.flatnonzero(self.in_t)
            _lib.call("dlp_graph_toggle", ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.aw), ptr(G.data), ptr(moved),
                      int(moved.numel()), ptr(self.in_t), ptr(self.umask), ptr(self.rowsum), ptr(self.changed), s)
            self.counters["ground_changes"] += nmoved
        Q = kernels.flatnonzero(self.changed)
        self._system_rows(Q, int(Q.numel()))
        self.t += 1
        self.last_changed, self.last_moved = Q, moved
        self.n_ins, self.n_del = int(ins.numel()), int(dele.numel())
        um = self.umask.bool()
        is_new = um & ~prev_u
        mark = torch.zeros(n, dtype=torch.uint8, device=dev)
        touched = torch.cat([ins, dele]).to(torch.int32).contiguous()
        if touched.numel():
            _lib.call("dlp_mark_neighbors", ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(touched),
                      int(touched.numel()), ptr(mark), s)
        seed = (mark.bool() | is_new) & um
        comps = {}
        if tau is not None:
            new = torch.nonzero(is_new, as_tuple=False).flatten()
            nl = torch.full((n,), -1, dtype=torch.int64, device=dev)
            nl[new] = torch.arange(new.numel(), device=dev)
            wd = G.data if self.dtype == torch.float32 else G.data.to(self.dtype)
            comps = new_components_rows(new, G.rbeg, G.rend, G.indices, wd, nl, tau, wmax, self.B[new].sum(dim=1))
        self._vertex_batch = {"is_new": is_new, "seed": seed, "comps": comps}
        self._counts = None
        return self.system

    def solver_csr(self) -> CSR:
        """Compact CSR of W_UU (live solver entries only) for the current batch (cached)."""
        if getattr(self, "_csr_t", None) == (self.t, id(self.G.indices)):
            return self._csr
        self._csr_launch()
        self._csr_set(int(self._csr_ptr[self.n].item()))
        return self._csr

    def _csr_launch(self):
        """Queue the compact CSR build of the current slots (no host read)."""
        n, G = self.n, self.G
        cap = int(G.indices.numel())
        if getattr(self, "_csr_cap", 0) < cap:
            self._csr_col = torch.empty(cap, dtype=torch.int32, device=self.dev)
            self._csr_w = torch.empty(cap, dtype=torch.float32, device=self.dev)
            self._csr_ptr = torch.empty(n + 1, dtype=torch.int32, device=self.dev)
            self._csr_cap = cap
        ws = workspace("to_csr").get(_lib.lib().dlp_graph_to_csr_workspace_bytes(n))
        _lib.call("dlp_graph_to_csr", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.data), ptr(self._csr_ptr),
                  ptr(self._csr_col), ptr(self._csr_w), ptr(ws), ws.numel(), stream())

    def _csr_set(self, nnz):
        """The CSR of the build just queued, given its entry count."""
        n, G = self.n, self.G
        self._csr = CSR(self._csr_w[:nnz], self._csr_col[:nnz], self._csr_ptr, (n, n))
        self._csr_t = (self.t, id(G.indices))
        return self._csr

    @property
    def system(self) -> System:
        """Global-index system of the current batch (arrays live until the next batch)."""
        n, C, dev = self.n, self.C, self.dev
        um = self.umask.view(torch.bool)  # 0/1 bytes: a view, no conversion kernel
        if getattr(self, "_s64", None) is None:
            self._s64 = torch.empty(n, dtype=torch.float64, device=dev)
            self._ids = torch.arange(n, device=dev)
            self._no_new = torch.zeros(n, dtype=torch.bool, device=dev)
        s64 = torch.sub(self.diag64, self.rowsum, out=self._s64)
        # active and ungrounded counts change only with vertex batches or membership changes
        if getattr(self, "_counts", None) is None:
            self._counts = torch.stack([self.vmask.sum() + self.labeled.sum(), (self.vmask.bool() & ~um).sum()]).tolist()
        n_active, n_ungrounded = self._counts
        vx = getattr(self, "_vertex_batch", None)
        common = dict(t=self.t, U=self._ids, W=self.solver_csr(),
                      is_new=vx["is_new"] if vx else self._no_new,
                      seed=vx["seed"] if vx else self.changed.view(torch.bool), comps=vx["comps"] if vx else {}, K=self.K,
                      C=C,
                      eta=self.eta,
                      n_inserted=self.n_ins, n_deleted=self.n_del, n_active=int(n_active),
                      n_ungrounded=int(n_ungrounded), solved=um,
                      changed=self.last_changed, moved=self.last_moved)
        ch = C + (1 if self.with_h else 0)
        # the grounding stays fp64 in every precision (its one reader, the AMG setup, works in fp64)
        S = System(s=s64, diag=self.diag32 if self.dtype == torch.float32 else self.diag64.to(self.dtype),
                   B=self.B, rhs=self.rhs32[:, :C] if self.dtype == torch.float32 else self.rhs64[:, :C].to(self.dtype),
                   prior=self.prior64.to(self.dtype), rhs_h=self.rhs32[:, :ch] if self.dtype == torch.float32 else None,
                   **common)
        S._conv[torch.float64] = System(s=s64, diag=self.diag64, B=self.B, rhs=self.rhs64[:, :C], prior=self.prior64,
                                        rhs_h=self.rhs64[:, :ch], **common)
        return S


# ---------------------------------------------------------------------------------------------
# the vertex-arrival stream (dynlp/stream.py:84-177) and its resident form (:180-346)
# ---------------------------------------------------------------------------------------------
class Stream:
    """Reveals a dataset in batches (dynlp/stream.py:84-128): an initial snapshot, then batches of
    new vertices, with a label_frac share of all vertices carrying ground truth, and deletions of
    del_frac x batch-size random active unlabelled vertices. The whole schedule is drawn up front
    on the host with a NumPy RandomState(seed + 7), the same draws in the same order as the
    reference, so a run reproduces the reference's schedule on NumPy exactly. `batches()` yields
    the grounded system of every batch (Stream._build) built on the device."""

    def __init__(self, ds: Dataset, *, label_frac=0.01, init_frac=0.1, n_batches=10, del_frac=0.1, eta_rel=0.0,
                 seed=0, dtype="float32"):
        self.ds, self.dtype, self.del_frac = ds, dtype, del_frac
        n, K = ds.n, ds.K
        dev = ds.A.indices.device
        y = ds.y.cpu().numpy()
        rs = np.random.RandomState(seed + 7)
        cand = np.flatnonzero(y >= 0)
        lab = np.zeros(n, dtype=bool)
        lab[cand[rs.permutation(cand.shape[0])[: max(K, int(label_frac * n))]]] = True
        order = ds.order.cpu().numpy().astype(np.int64).copy()
        n0 = max(int(init_frac * n), 2 * K)
        pos = np.empty(n, dtype=np.int64)
        pos[order] = np.arange(n)
        for c in range(K):  # the initial snapshot needs a labelled vertex of every class
            lc = np.flatnonzero(lab & (y == c))
            if not lc.shape[0]:
                lc = np.flatnonzero(y == c)[:1]
                lab[lc] = True
            if lc.shape[0] and int(pos[lc].min()) >= n0:
                free = np.flatnonzero(~lab[order[:n0]])
                v, j = int(lc[0]), int(free[int(rs.randint(0, free.shape[0]))])
                a, pv = int(order[j]), int(pos[v])
                order[j], order[pv], pos[v], pos[a] = v, a, j, pv
        self.n0 = n0
        self.labeled = torch.as_tensor(lab, device=dev)
        self.order = torch.as_tensor(order, device=dev)
        chunks = np.array_split(order[n0:], n_batches) if n_batches > 0 else []
        data = ds.A.data.cpu().numpy()
        # the component threshold and scale, as the reference takes them (NumPy reductions)
        self.tau, self.wmax = float(data.mean()), float(data.max())
        self.eta = float(eta_rel * data.sum() / n)
        self.prior = torch.full((1 if K == 2 else K,), 0.5 if K == 2 else 1.0 / K, dtype=to_dtype(dtype), device=dev)
        active = np.zeros(n, dtype=bool)
        sched = []
        for t in range(1 + len(chunks)):
            ins, dele = (order[:n0] if t == 0 else chunks[t - 1]), np.zeros(0, dtype=np.int64)
            if t:
                pool = np.flatnonzero(active & ~lab)
                nd = min(int(del_frac * ins.shape[0]), max(pool.shape[0] - 1, 0))
                if nd > 0:
                    dele = pool[rs.permutation(pool.shape[0])[:nd]]
            active[ins], active[dele] = True, False
            sched.append((torch.as_tensor(ins.astype(np.int64), device=dev),
                          torch.as_tensor(dele.astype(np.int64), device=dev)))
        self.schedule = sched

    def __len__(self):
        return len(self.schedule)

    def batches(self):
        n, dev = self.ds.n, self.ds.A.indices.device
        active = torch.zeros(n, dtype=torch.bool, device=dev)
        prev_u = torch.zeros(n, dtype=torch.bool, device=dev)
        for t, (ins, dele) in enumerate(self.schedule):
            active[ins] = True
            active[dele] = False
            S = self._build(t, active, prev_u, ins, dele)
            prev_u = torch.zeros(n, dtype=torch.bool, device=dev)
            prev_u[S.U] = True
            yield S

    def _build(self, t, active, prev_u, ins, dele) -> System:
        return build_system(self.ds, active, self.labeled, eta=self.eta, dtype=self.dtype, t=t, prev_U=prev_u,
                            ins_ids=ins, del_ids=dele, tau=self.tau, wmax=self.wmax)


class IncrementalStream(Stream):
    """The same stream with the batch system resident and updated in place (dynlp/stream.py:180-346):
    global vertex ids, inert rows outside U, solver weights masked in place, label weights moved
    by the batch's labelled vertices, and the grounded set re-checked on the device (by
    reachability from the labelled vertices, which gives the reference's ball-check-or-CC result).
    Systems are live until the next batch. `ball_hops` is accepted for the reference's signature;
    the reachability check needs no ball."""

    def __init__(self, ds: Dataset, *, ball_hops=3, slack_frac=0.25, **kw):
        super().__init__(ds, **kw)
        self.ball_hops = ball_hops
        self.slack_frac = slack_frac
        self.counters = {"ground_sweeps": 0, "ground_fallbacks": 0}
        self.resident = None

    def batches(self):
        n, dev = self.ds.n, self.ds.A.indices.device
        es = EdgeStream(self.ds, self.labeled, eta_rel=0.0, dtype=self.dtype, slack_frac=self.slack_frac,
                        active=torch.zeros(n, dtype=torch.bool, device=dev))
        es.eta = self.eta
        self.resident = es
        for ins, dele in self.schedule:
            S = es.apply_vertices(ins, dele, tau=self.tau, wmax=self.wmax)
            self.counters.update(ground_sweeps=es.counters["ground_sweeps"],
                                 ground_fallbacks=es.counters["ground_fallbacks"])
            yield S

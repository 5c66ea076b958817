"""Continuous-batching serving loop over a resident graph (no reference counterpart; the closest
is the reference's batch loop, dynlp/bench.py:93-118).

The server keeps the resident system (graph, scores, residual) on the device and answers three
request kinds as they arrive:

* `EdgeUpdate`: edge insertions/deletions. Queued updates are patched into the resident graph in
  arrival order (so the final graph is the sequential one), then ONE certified solve brings the
  scores back to the target relative residual for all of them. The result carries the rows whose
  label changed and their new labels. Updates that arrive while a solve runs take the next slot.
* `LabelQuery`: labels of the given vertices (-1 outside the solved set), read from the label
  snapshot published after the last completed update (queries never see scores being solved).
* `FreshSolve`: the harmonic solve of a new graph. Pending fresh solves are solved together in one
  batched launch (per-instance CG, so every result equals what it would be alone).

Admission. Every request has a device-memory cost (its staged inputs and working buffers; a fresh
solve its whole system). One HBM budget is shared by all kinds: a worker takes the queued requests
of its kind, in arrival order, while they fit its slot (edges per update solve, ids per query
batch, instances per fresh batch) and the memory the budget has free, reserves that memory, and
returns it when the batch completes; a request that does not fit waits for the next slot. A
request larger than the whole budget is refused. Each kind has its own worker thread and CUDA
stream, so their device work overlaps (updates and queries on high-priority streams, fresh solves on a
normal one); libdlp calls release the GIL.

Precision. The continuous loop is mixed precision: FP32 (or BF16, lowp=True) sweeps with refinement
against an FP64 residual. mode="sequential" serves one request at a time in arrival order; by
default in plain FP32, the path the loop is measured against (every update solved alone by FP32 PCG
without an FP64 residual, every fresh solve launched alone in FP32), and with precision="mixed" the
loop's own solvers one request at a time (which isolates what batching buys). Every request records
its submit and completion times (p50/p99 latency).
"""
from __future__ import annotations

import queue
import sys
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np
import torch

from . import batched, solvers, stream


@dataclass
class EdgeUpdate:
    ins_u: np.ndarray
    ins_v: np.ndarray
    ins_w: np.ndarray | None = None
    del_u: np.ndarray | None = None
    del_v: np.ndarray | None = None

    @property
    def size(self):
        return len(self.ins_u) + (len(self.del_u) if self.del_u is not None else 0)

    def hbm_bytes(self):
        # staged ids and weights (12 B per insertion, 8 per deletion) and the insertion's dedupe
        # table and slot lists (about 28 B per insertion)
        ni = len(self.ins_u)
        nd = len(self.del_u) if self.del_u is not None else 0
        return 40 * ni + 8 * nd + 4096


@dataclass
class LabelQuery:
    ids: np.ndarray

    @property
    def size(self):
        return len(self.ids)

    def hbm_bytes(self):
        return 12 * len(self.ids) + 4096  # staged int64 ids and the int32 labels gathered


@dataclass
class FreshSolve:
    ds: object            # graphs.Dataset
    labeled: torch.Tensor

    @property
    def size(self):
        return 1

    def hbm_bytes(self, C=None):
        n, nnz = self.ds.n, self.ds.nnz
        C = (1 if self.ds.K == 2 else self.ds.K) if C is None else C
        return int(nnz * 12 + n * (C + 1) * 8 * 7 + n * 64)


@dataclass
class _Item:
    req: object
    fut: Future
    t_submit: float
    kind: str
    t_done: float = 0.0
    extra: dict = field(default_factory=dict)


class AdmissionError(RuntimeError):
    """The request cannot fit the HBM budget."""


class HbmBudget:
    """Device memory reserved by the batches in flight, against a fixed budget."""

    def __init__(self, total):
        self.total, self.used = int(total), 0
        self._cv = threading.Condition()

    def free(self):
        with self._cv:
            return self.total - self.used

    def acquire(self, nbytes, stop=None):
        """Reserve nbytes, waiting while other batches hold the memory (nbytes <= total)."""
        with self._cv:
            while self.used + nbytes > self.total:
                if stop is not None and stop.is_set():
                    raise RuntimeError("server closed")
                self._cv.wait(timeout=0.1)
            self.used += nbytes

    def release(self, nbytes):
        with self._cv:
            self.used -= nbytes
            self._cv.notify_all()


def take_batch(q, first, limit=None, cost=None, budget=None, size=None, slot=None):
    """The requests of one batch: `first`, then queued requests in arrival order while the batch
    holds fewer than `limit` requests (None: no limit), while the summed `size` stays within `slot`
    and, given `cost`, while the summed cost stays within `budget` (`first` is always taken).
    Returns (items, carry): `carry` is the queued request that did not fit, which heads the next
    batch so that arrival order holds, or None. The shutdown sentinel (None) ends the batch and goes
    back on the queue for the worker loop to see."""
    items, carry = [first], None
    used = cost(first) if cost is not None else 0
    filled = size(first) if size is not None else 0
    while limit is None or len(items) < limit:
        try:
            nxt = q.get_nowait()
        except queue.Empty:
            break
        if nxt is None:
            q.put(None)
            break
        need = cost(nxt) if cost is not None else 0
        more = size(nxt) if size is not None else 0
        if (cost is not None and used + need > budget) or (slot is not None and filled + more > slot):
            carry = nxt  # admitted with the next slot
            break
        used += need
        filled += more
        items.append(nxt)
    return items, carry


class Server:
    def __init__(self, ds, labeled, *, dtype="float32", target_relres=1e-6, tol=1e-3, hbm_budget_bytes=None,
                 max_fresh_batch=64, update_slot_edges=200_000, query_slot_ids=4_000_000, mode="continuous",
                 lowp=False, precision=None, switch_interval_s=0.0005):
        """mode="continuous": the continuous-batching loop described above; mode="sequential": one
        request at a time in arrival order. precision="mixed" (the default of the continuous loop):
        FP32 sweeps (lowp: BF16 gathers in the update solves' sweeps) with refinement against the
        FP64 residual; precision="fp32" (the default of the sequential mode): the plain FP32 path. The
        slots cap the edges patched before one update solve and the ids of one query batch.
        switch_interval_s: the interpreter's thread switch interval while the server runs."""
        if mode not in ("continuous", "sequential"):
            raise ValueError(f"unknown serving mode {mode!r}")
        precision = precision or ("mixed" if mode == "continuous" else "fp32")
        if precision not in ("mixed", "fp32"):
            raise ValueError(f"unknown serving precision {precision!r}")
        self.mode, self.precision = mode, precision
        self.target = target_relres
        self.K = ds.K
        self.es = stream.EdgeStream(ds, labeled, dtype=dtype)
        if precision == "mixed":
            self.solver = solvers.IncrementalLP(ds.n, ds.K, dtype, tol=tol, method="pcg",
                                                target_relres=target_relres, full_every=16, lowp=lowp)
        else:
            self.solver = solvers.PlainFP32LP(ds.n, ds.K, target_relres=target_relres)
        self.solver.solve(self.es.system)
        self.labels = self.solver.relabel(self.es.system)[0].clone()
        self.version = 0
        free, total = torch.cuda.mem_get_info()
        self.budget = HbmBudget(hbm_budget_bytes if hbm_budget_bytes is not None else 0.5 * free)
        seq = mode == "sequential"
        self.max_fresh_batch = 1 if seq else max_fresh_batch
        self.slots = {"update": None if seq else update_slot_edges, "query": None if seq else query_slot_ids}
        self._q = {"update": queue.Queue(), "query": queue.Queue(), "fresh": queue.Queue()}
        if seq:  # one queue for every kind: arrival order, one request at a time
            one = queue.Queue()
            self._q = {k: one for k in self._q}
        # updates and queries on high-priority streams: their kernels go ahead of a fresh solve's when
        # both are ready, so a large fresh batch does not hold the resident graph's answers back
        self._streams = {k: torch.cuda.Stream(priority=0 if k == "fresh" else -1) for k in self._q}
        self._stop = threading.Event()
        self._lock = threading.Lock()
        self._carry = {}  # per worker: the queued request that heads its next batch
        self.done: list[_Item] = []
        kinds = ["all"] if seq else list(self._q)
        self._threads = [threading.Thread(target=self._worker, args=(k,), daemon=True) for k in kinds]
        self._dev = torch.cuda.current_device()
        # the workers hand the interpreter lock to each other at every device wait; the default 5 ms
        # switch interval would let a worker busy with host-side bookkeeping hold a waiting one back
        # for that long at each of its host reads (restored by close)
        self._switch = sys.getswitchinterval()
        sys.setswitchinterval(min(self._switch, switch_interval_s))
        for t in self._threads:
            t.start()

    # -- client side ---------------------------------------------------------------------------
    def submit(self, req) -> Future:
        kind = "update" if isinstance(req, EdgeUpdate) else "query" if isinstance(req, LabelQuery) else "fresh"
        fut = Future()
        need = req.hbm_bytes()
        if need > self.budget.total:
            fut.set_exception(AdmissionError(f"{kind} request needs ~{need / 1e9:.2f} GB of device memory, "
                                             f"budget {self.budget.total / 1e9:.2f} GB"))
            return fut
        self._q[kind].put(_Item(req, fut, time.perf_counter(), kind))
        return fut

    def close(self):
        """Stops the workers after their current batch; requests still waiting fail with
        RuntimeError("server closed")."""
        self._stop.set()
        sys.setswitchinterval(self._switch)
        queues = {id(q): q for q in self._q.values()}.values()
        for q in queues:
            q.put(None)
        for t in self._threads:
            t.join(timeout=60)
        left = [it for it in list(self._carry.values()) if it is not None]
        self._carry.clear()
        for q in queues:
            while True:
                try:
                    it = q.get_nowait()
                except queue.Empty:
                    break
                if it is not None:
                    left.append(it)
        for it in left:
            if not it.fut.done():
                it.fut.set_exception(RuntimeError("server closed"))

    def latency(self, kind=None):
        with self._lock:
            lat = [1e3 * (it.t_done - it.t_submit) for it in self.done if kind in (None, it.kind)]
        if not lat:
            return {}
        return {"n": len(lat), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}

    # -- workers -------------------------------------------------------------------------------
    def _finish(self, items, results):
        t = time.perf_counter()
        with self._lock:
            for it in items:
                it.t_done = t
                self.done.append(it)
        for it, r in zip(items, results):
            if isinstance(r, BaseException):
                it.fut.set_exception(r)
            else:
                it.fut.set_result(r)

    def _batch(self, kind, first, limit=None):
        """The batch `first` heads (its kind's slot and the free budget) and the memory it reserves."""
        if self.mode == "sequential":
            items, carry = [first], None
        else:
            items, carry = take_batch(self._q[kind], first, limit=limit, cost=lambda it: it.req.hbm_bytes(),
                                      budget=self.budget.free(), size=lambda it: it.req.size,
                                      slot=self.slots.get(kind))
        nbytes = sum(it.req.hbm_bytes() for it in items)
        self.budget.acquire(nbytes, self._stop)  # waits while other batches hold the memory
        return items, carry, nbytes

    def _worker(self, kind):
        torch.cuda.set_device(self._dev)
        q = self._q["update"] if kind == "all" else self._q[kind]
        with torch.cuda.stream(self._streams["update" if kind == "all" else kind]):
            while not self._stop.is_set():
                first = self._carry.pop(kind, None)
                if first is None:
                    first = q.get()
                if first is None:
                    break
                try:
                    self._carry[kind] = getattr(self, "_do_" + first.kind)(first)
                except BaseException as e:  # a failing batch fails its requests, not the server
                    self._finish([first], [e])

    def _do_update(self, first):
        items, carry, nbytes = self._batch("update", first)
        try:
            for i, it in enumerate(items):  # sequential patch semantics, one solve for all of them
                r = it.req
                self.es.apply_edges(r.ins_u, r.ins_v, r.ins_w, r.del_u, r.del_v, keep_pending=i > 0)
            S = self.es.system
            st = self.solver.solve(S)
            labels, chg, chg_lab, nchg = self.solver.relabel(S)
            k = int(nchg.item())
            rows, labs = chg[:k].cpu().numpy(), chg_lab[:k].cpu().numpy()
            snapshot = labels.clone()
            torch.cuda.current_stream().synchronize()
            with self._lock:
                self.labels, self.version = snapshot, self.version + 1
            res = {"relres": st.relres, "cert": st.cert, "path": st.path, "coalesced": len(items),
                   "version": self.version, "relabelled_rows": rows, "relabelled_labels": labs}
            self._finish(items, [res] * len(items))
        except BaseException as e:
            self._finish(items, [e] * len(items))
        finally:
            self.budget.release(nbytes)
        return carry

    def _do_query(self, first):
        items, carry, nbytes = self._batch("query", first)
        try:
            with self._lock:
                labels = self.labels
            outs = []
            for it in items:
                ids = torch.as_tensor(np.asarray(it.req.ids, dtype=np.int64)).to(labels.device, non_blocking=True)
                outs.append(labels.index_select(0, ids))
            torch.cuda.current_stream().synchronize()
            self._finish(items, [o.cpu().numpy() for o in outs])
        except BaseException as e:
            self._finish(items, [e] * len(items))
        finally:
            self.budget.release(nbytes)
        return carry

    def _do_fresh(self, first):
        """One batched launch of the fresh solves that fit the slot and the budget together."""
        items, carry, nbytes = self._batch("fresh", first, limit=self.max_fresh_batch)
        try:
            systems = []
            for it in items:
                ds = it.req.ds
                systems.append(stream.build_system(ds, torch.ones(ds.n, dtype=torch.bool, device=ds.A.indices.device),
                                                   it.req.labeled, dtype="float32"))
            if self.precision == "mixed":  # FP32 sweeps, refinement against the FP64 residual
                Fs, info = batched.solve_many_mixed(systems, target_relres=self.target)
            else:  # the plain FP32 solve
                Fs, info = batched.solve_many(systems, target_relres=self.target, dtype=torch.float32)
            outs = []
            for S, F, (iters, status, rel) in zip(systems, Fs, info):
                outs.append({"U": S.U, "F": F, "labels": solvers.predict(F, S.K), "iters": iters, "status": status,
                             "relres": rel, "batch": len(items)})
            torch.cuda.current_stream().synchronize()
            self._finish(items, outs)
        except BaseException as e:
            self._finish(items, [e] * len(items))
        finally:
            self.budget.release(nbytes)
        return carry

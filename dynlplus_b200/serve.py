"""Continuous-batching serving loop over a resident graph (no reference counterpart; the closest
is the reference's batch loop, dynlp/bench.py:93-118).

The server keeps the resident system (graph, scores, residual) on the device and answers three
request kinds as they arrive:

* `EdgeUpdate`: edge insertions/deletions. Every queued update is patched into the resident graph
  in arrival order (so the final graph is the sequential one), then ONE certified solve brings the
  scores back to the target relative residual for all of them; the request completes when its
  scores are current. Updates arriving while a solve runs are admitted into the next one.
* `LabelQuery`: argmax labels of the given vertices, read from the label snapshot published after
  the last completed update (queries never see scores that are being solved).
* `FreshSolve`: the harmonic solve of a new graph. Pending fresh solves are admitted while their
  estimated HBM footprint fits the budget and solved together in one batched launch (per-instance
  CG, so every result equals what it would be alone); requests arriving meanwhile wait for the next
  batch. A request larger than the whole budget is refused.

Each kind has its own worker thread and CUDA stream, so their device work overlaps; libdlp calls
release the GIL. Every request records its submit and completion times (p50/p99 latency).
"""
from __future__ import annotations

import queue
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


@dataclass
class LabelQuery:
    ids: np.ndarray


@dataclass
class FreshSolve:
    ds: object            # graphs.Dataset
    labeled: torch.Tensor

    def hbm_bytes(self, C):
        n, nnz = self.ds.n, self.ds.nnz
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


def take_batch(q, first, limit=None, cost=None, budget=None):
    """The requests of one batch: `first`, then queued requests in arrival order while the batch
    holds fewer than `limit` (None: no limit) and, given `cost`, while the summed cost stays within
    `budget` (`first` is always taken). Returns (items, carry): `carry` is the queued request that
    did not fit, which heads the next batch so that arrival order holds, or None. The shutdown
    sentinel (None) ends the batch and goes back on the queue for the worker loop to see."""
    items, carry = [first], None
    used = cost(first) if cost is not None else 0
    while limit is None or len(items) < limit:
        try:
            nxt = q.get_nowait()
        except queue.Empty:
            break
        if nxt is None:
            q.put(None)
            break
        if cost is not None:
            need = cost(nxt)
            if used + need > budget:  # admitted next, once this batch has freed its memory
                carry = nxt
                break
            used += need
        items.append(nxt)
    return items, carry


class Server:
    def __init__(self, ds, labeled, *, dtype="float32", target_relres=1e-6, tol=1e-3, hbm_budget_bytes=None,
                 max_fresh_batch=64, fresh_dtype=torch.float64, mode="continuous", lowp=False):
        """mode="continuous": the loop described above. mode="sequential": the plain path it is
        measured against -- one worker, requests served one at a time in arrival order, every update
        solved on its own and every fresh solve launched alone. lowp: BF16 gathers in the update
        solves' working-precision sweeps (fp64 refinement keeps the target)."""
        if mode not in ("continuous", "sequential"):
            raise ValueError(f"unknown serving mode {mode!r}")
        self.mode = mode
        self.target = target_relres
        self.K = ds.K
        self.fresh_dtype = fresh_dtype
        self.es = stream.EdgeStream(ds, labeled, dtype=dtype)
        self.solver = solvers.IncrementalLP(ds.n, ds.K, dtype, tol=tol, method="pcg", target_relres=target_relres,
                                            full_every=16, lowp=lowp)
        self.solver.solve(self.es.system)
        self.labels = self._snapshot()
        self.version = 0
        free, total = torch.cuda.mem_get_info()
        self.budget = int(hbm_budget_bytes if hbm_budget_bytes is not None else 0.5 * free)
        self.max_fresh_batch = max_fresh_batch if mode == "continuous" else 1
        self._q = {"update": queue.Queue(), "query": queue.Queue(), "fresh": queue.Queue()}
        if mode == "sequential":  # one queue for every kind: arrival order, one request at a time
            one = queue.Queue()
            self._q = {k: one for k in self._q}
        self._streams = {k: torch.cuda.Stream() for k in self._q}
        self._stop = threading.Event()
        self._lock = threading.Lock()
        self._carry = {}  # per worker: the queued request that heads its next batch
        self.done: list[_Item] = []
        kinds = list(self._q) if mode == "continuous" else ["all"]
        self._threads = [threading.Thread(target=self._worker, args=(k,), daemon=True) for k in kinds]
        self._dev = torch.cuda.current_device()
        for t in self._threads:
            t.start()

    # -- client side ---------------------------------------------------------------------------
    def submit(self, req) -> Future:
        kind = "update" if isinstance(req, EdgeUpdate) else "query" if isinstance(req, LabelQuery) else "fresh"
        fut = Future()
        if kind == "fresh":
            C = 1 if req.ds.K == 2 else req.ds.K
            if req.hbm_bytes(C) > self.budget:
                fut.set_exception(AdmissionError(f"fresh solve needs ~{req.hbm_bytes(C) / 1e9:.2f} GB, "
                                                 f"budget {self.budget / 1e9:.2f} GB"))
                return fut
        self._q[kind].put(_Item(req, fut, time.perf_counter(), kind))
        return fut

    def close(self):
        """Stops the workers after their current batch; requests still waiting fail with
        RuntimeError("server closed")."""
        self._stop.set()
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
    def _snapshot(self):
        Z = self.solver.Z
        return solvers.predict(Z[:, : self.solver.C], self.K).clone()

    def _finish(self, items, results):
        t = time.perf_counter()
        with self._lock:
            for it, r in zip(items, results):
                it.t_done = t
                self.done.append(it)
        for it, r in zip(items, results):
            if isinstance(r, BaseException):
                it.fut.set_exception(r)
            else:
                it.fut.set_result(r)

    def _drain(self, kind, first):
        if self.mode == "sequential":
            return [first]
        return take_batch(self._q[kind], first)[0]

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
        items = self._drain("update", first)
        try:
            for i, it in enumerate(items):  # sequential patch semantics, one solve for all of them
                r = it.req
                self.es.apply_edges(r.ins_u, r.ins_v, r.ins_w, r.del_u, r.del_v, keep_pending=i > 0)
            st = self.solver.solve(self.es.system)
            labels = self._snapshot()
            torch.cuda.current_stream().synchronize()
            with self._lock:
                self.labels, self.version = labels, self.version + 1
            res = {"relres": st.relres, "cert": st.cert, "path": st.path, "coalesced": len(items),
                   "version": self.version}
            self._finish(items, [res] * len(items))
        except BaseException as e:
            self._finish(items, [e] * len(items))

    def _do_query(self, first):
        items = self._drain("query", first)
        with self._lock:
            labels = self.labels
        outs = []
        for it in items:
            ids = torch.as_tensor(np.asarray(it.req.ids, dtype=np.int64)).to(labels.device, non_blocking=True)
            outs.append(labels.index_select(0, ids))
        torch.cuda.current_stream().synchronize()
        self._finish(items, [o.cpu().numpy() for o in outs])

    def _do_fresh(self, first):
        """One batched launch of the fresh solves that fit the budget together; returns the queued
        request that did not fit (the worker starts its next batch with it) or None."""
        cost = lambda it: it.req.hbm_bytes(1 if it.req.ds.K == 2 else it.req.ds.K)  # noqa: E731
        items, carry = take_batch(self._q[first.kind], first, self.max_fresh_batch, cost, self.budget)
        try:
            systems = []
            for it in items:
                ds = it.req.ds
                systems.append(stream.build_system(ds, torch.ones(ds.n, dtype=torch.bool, device=ds.A.indices.device),
                                                   it.req.labeled, dtype="float32"))
            Fs, info = batched.solve_many(systems, target_relres=self.target, dtype=self.fresh_dtype)
            outs = []
            for S, F, (iters, status, rel) in zip(systems, Fs, info):
                outs.append({"U": S.U, "F": F, "labels": solvers.predict(F, S.K), "iters": iters, "status": status,
                             "relres": rel, "batch": len(items)})
            torch.cuda.current_stream().synchronize()
            self._finish(items, outs)
        except BaseException as e:
            self._finish(items, [e] * len(items))
        return carry

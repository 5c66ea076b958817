"""Graph datasets and CSR construction (mirrors dynlp/graphs.py).

A dataset is a symmetric, non-negative, loop-free CSR `A` with labels `y` in [0, K) and an arrival
`order` (dynlp/graphs.py:25-33). CSR assembly runs on the device with torch sorts (one-time setup,
not the hot path). Generators:

* `sbm`, `erdos_renyi`: the reference's generators (graphs.py:96-121), same random calls on a
  NumPy RandomState, so they reproduce the reference run on NumPy exactly.
* `planted_partition`, `er_graph`: the benchmark workloads, seeded `numpy.random.default_rng`,
  duplicate pairs kept once (set semantics), self-loops dropped.
* `synth`, `knn_graph`: the reference's synthetic cosine-kNN mixture (graphs.py:78-143), same
  RandomState draws; `build_cached` / `load("synthN")` keep it as an edge-list npz under DATA_DIR.
* `EdgeUpdates`: the edge-update stream (insert uniform non-edges / delete uniform edges).
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass

import numpy as np
import torch

from .backend import CSR, to_dtype

DATA_DIR = os.environ.get("DATA_DIR", "data")  # graph caches (dynlp/graphs.py:21)


def _dev(device=None):
    if device is not None:
        return torch.device(device)
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


@dataclass
class Dataset:
    name: str
    A: CSR
    y: torch.Tensor      # int32 (n,)
    K: int
    order: torch.Tensor  # int64 permutation: arrival order

    n = property(lambda self: self.A.shape[0])
    nnz = property(lambda self: int(self.A.nnz))


def _t(x, dev, dtype=None):
    t = x if torch.is_tensor(x) else torch.as_tensor(np.ascontiguousarray(x))
    t = t.to(dev)
    return t.to(dtype) if dtype is not None else t


def coalesce(rows, cols, vals, n, dtype, device=None) -> CSR:
    """Canonical CSR: duplicates summed, self-loops dropped (dynlp/graphs.py:36-44)."""
    dev = _dev(device) if not torch.is_tensor(rows) else rows.device
    r, c = _t(rows, dev, torch.int64), _t(cols, dev, torch.int64)
    v = _t(vals, dev, torch.float64).to(to_dtype(dtype))  # duplicates summed in the target precision
    keep = r != c
    r, c, v = r[keep], c[keep], v[keep]
    key = r * n + c
    uk, inv = torch.unique(key, sorted=True, return_inverse=True)
    sv = torch.zeros(uk.numel(), dtype=v.dtype, device=dev).index_add_(0, inv, v)
    rr = (uk // n)
    indptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    indptr[1:] = torch.cumsum(torch.bincount(rr, minlength=n), 0)
    return CSR(sv.to(to_dtype(dtype)), (uk % n).to(torch.int32), indptr.to(torch.int32), (n, n))


def symmetric_from_pairs(u, v, w, n, dtype, device=None) -> CSR:
    """dynlp/graphs.py:47-48."""
    dev = _dev(device) if not torch.is_tensor(u) else u.device
    u, v, w = _t(u, dev, torch.int64), _t(v, dev, torch.int64), _t(w, dev, torch.float64)
    return coalesce(torch.cat([u, v]), torch.cat([v, u]), torch.cat([w, w]), n, dtype, dev)


def symmetric_set(u, v, w, n, dtype, device=None) -> CSR:
    """Symmetric CSR from undirected pairs with set semantics: each unordered pair kept once (its
    first occurrence's weight), self-loops dropped."""
    dev = _dev(device)
    u, v = _t(u, dev, torch.int64), _t(v, dev, torch.int64)
    w = _t(w, dev, torch.float64)
    keep = u != v
    u, v, w = u[keep], v[keep], w[keep]
    a, b = torch.minimum(u, v), torch.maximum(u, v)
    key = a * n + b
    uk, inv = torch.unique(key, sorted=True, return_inverse=True)
    first = torch.full((uk.numel(),), key.numel(), dtype=torch.int64, device=dev)
    first.scatter_reduce_(0, inv, torch.arange(key.numel(), device=dev), reduce="amin")
    a, b, w = uk // n, uk % n, w[first]
    return coalesce(torch.cat([a, b]), torch.cat([b, a]), torch.cat([w, w]), n, dtype, dev)


def expand_counts(counts, nseg):
    """Segment id of each element given per-segment counts (dynlp/graphs.py:51-57)."""
    return torch.repeat_interleave(torch.arange(nseg, dtype=torch.int32, device=counts.device), counts.long())


def csr_rows(A) -> torch.Tensor:
    """Row index of every stored entry of a CSR matrix (dynlp/graphs.py:62-64)."""
    return expand_counts(torch.diff(A.indptr), A.shape[0])


def row_positions(indptr, rows):
    """Positions of all stored entries in the given rows, and each one's segment (graphs.py:67-75)."""
    rows = rows.long()
    counts = (indptr[rows + 1] - indptr[rows]).long()
    seg = expand_counts(counts, int(rows.numel()))
    if not seg.numel():
        return torch.zeros(0, dtype=torch.int64, device=indptr.device), seg
    excl = torch.cumsum(counts, 0) - counts
    pos = indptr[rows].long()[seg.long()] + (torch.arange(seg.numel(), device=indptr.device) - excl[seg.long()])
    return pos, seg


# ---------------------------------------------------------------------------------------------
# the reference's generators (NumPy RandomState: identical draws to the reference run on NumPy)
# ---------------------------------------------------------------------------------------------
def _rng(seed):
    return np.random.RandomState(seed), np.random.RandomState(seed + 1).permutation


def sbm(n, K=2, deg=10.0, p_in=0.85, seed=0, dtype="float32", device=None) -> Dataset:
    """Planted partition (dynlp/graphs.py:100-112)."""
    rs, perm = _rng(seed)
    y = rs.randint(0, K, size=n).astype(np.int32)
    members, sizes = np.argsort(y).astype(np.int64), np.bincount(y, minlength=K).astype(np.int64)
    offs, m = np.cumsum(sizes) - sizes, int(n * deg / 2)
    u = rs.randint(0, n, size=m).astype(np.int64)
    intra = rs.random_sample(m) < p_in
    yu = y[u]
    v_in = members[offs[yu] + (rs.random_sample(m) * sizes[yu]).astype(np.int64)]
    v = np.where(intra, v_in, rs.randint(0, n, size=m).astype(np.int64))
    w = np.where(y[u] == y[v], 0.4 + 0.6 * rs.random_sample(m), 0.1 + 0.6 * rs.random_sample(m))
    dev = _dev(device)
    return Dataset(f"sbm-n{n}-K{K}-d{deg:g}", symmetric_from_pairs(u, v, w, n, dtype, dev), _t(y, dev), K,
                   _t(perm(n), dev))


def erdos_renyi(n, K=2, deg=5.0, seed=0, dtype="float32", device=None) -> Dataset:
    """dynlp/graphs.py:115-121."""
    rs, perm = _rng(seed)
    m = int(n * deg / 2)
    u, v = rs.randint(0, n, size=m).astype(np.int64), rs.randint(0, n, size=m).astype(np.int64)
    w = 0.1 + 0.9 * rs.random_sample(m)
    dev = _dev(device)
    A = symmetric_from_pairs(u, v, w, n, dtype, dev)
    return Dataset(f"er-n{n}-d{deg:g}", A, _t(rs.randint(0, K, size=n).astype(np.int32), dev), K, _t(perm(n), dev))


def knn_graph(X, k, dtype, device=None) -> CSR:
    """Symmetric cosine kNN graph of the (L2-normalised) dense rows of X (dynlp/graphs.py:78-93):
    each row's k most similar other rows (similarities of one row block at a time, top-k on the
    device), every unordered pair kept once with the similarity of its first occurrence in row-major
    order, clamped below at 1e-3. Sparse rows (the reference's TF-IDF documents) are not taken."""
    if not torch.is_tensor(X) and not isinstance(X, np.ndarray):
        raise TypeError("knn_graph takes dense rows (a NumPy array or a tensor)")
    dev = _dev(device) if not torch.is_tensor(X) else X.device
    Xt = _t(X, dev, torch.float32)
    n = int(Xt.shape[0])
    block = max(1, min(n, (1 << 26) // max(n, 1)))
    nbr = torch.empty((n, k), dtype=torch.int64, device=dev)
    sim = torch.empty((n, k), dtype=torch.float32, device=dev)
    for s in range(0, n, block):
        e = min(n, s + block)
        S = Xt[s:e] @ Xt.T
        S[torch.arange(e - s, device=dev), torch.arange(s, e, device=dev)] = -float("inf")
        sim[s:e], nbr[s:e] = torch.topk(S, k, dim=1)
    u = torch.arange(n, device=dev).repeat_interleave(k)
    v = nbr.reshape(-1)
    key = torch.minimum(u, v) * n + torch.maximum(u, v)
    order = torch.argsort(key, stable=True)
    ks = key[order]
    head = torch.ones_like(ks, dtype=torch.bool)
    head[1:] = ks[1:] != ks[:-1]
    first = order[head]  # the first occurrence of each pair, in key order
    return symmetric_from_pairs(u[first], v[first], sim.reshape(-1)[first].clamp(min=1e-3), n, dtype, dev)


def synth(n=50_000, K=10, k=5, dim=16, subs=5, seed=0, dtype="float32", device=None) -> Dataset:
    """The reference's mixture for DynLP's step 1 (dynlp/graphs.py:124-143): K classes of `subs`
    Gaussian sub-clusters in `dim` dimensions with spreads over a factor 8, a quarter of the
    tightest sub-clusters each shadowed by one of another class placed next to it, points on the
    unit sphere, cosine kNN with k neighbours. The draws are the reference's, in its order, on a
    NumPy RandomState (float32 arithmetic as there), so the points equal the reference run on NumPy."""
    rs, perm = _rng(seed)
    m = K * subs
    f32 = np.float32
    ctr = rs.standard_normal((m, dim)).astype(f32)
    ctr *= 10 / np.linalg.norm(ctr, axis=1, keepdims=True)
    spread = (0.4 * 8 ** rs.random_sample(m)).astype(f32)
    for a in np.argsort(spread)[: max(2, m // 4)].tolist():
        b = (a + subs * int(rs.randint(1, K))) % m if K > 1 else a
        step = rs.standard_normal(dim).astype(f32)
        spread[b] = spread[a]
        ctr[b] = ctr[a] + step / np.linalg.norm(step) * spread[a] * dim ** 0.5
    sub = rs.randint(0, m, size=n)
    X = ctr[sub] + spread[sub, None] * rs.standard_normal((n, dim)).astype(f32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    dev = _dev(device)
    return Dataset(f"synth{K}", knn_graph(X, k, dtype, dev), _t((sub // subs).astype(np.int32), dev), K, _t(perm(n), dev))


def build_cached(spec, data_dir=DATA_DIR, device=None):
    """data_dir/<spec>.npz, built if missing (dynlp/graphs.py:187-204): `synthN` is synth(K=N) saved
    as an upper-triangle edge list with labels (no order: loading draws the reference's). The IMDB
    review graph (downloads, TF-IDF) is not built here."""
    path = os.path.join(data_dir, f"{spec}.npz")
    if os.path.exists(path):
        return path
    if not re.fullmatch(r"synth\d+", spec):
        raise ValueError(f"unknown dataset {spec!r} (synthN, or an edge-list .npz; IMDB is not built here)")
    os.makedirs(data_dir, exist_ok=True)
    return save_npz(synth(K=int(spec[5:]), device=device), path, with_order=False)


# ---------------------------------------------------------------------------------------------
# benchmark workloads (seeded default_rng, set semantics)
# ---------------------------------------------------------------------------------------------
def _weights(rng, m, weights):
    if weights == "unit":
        return np.ones(m)
    if weights == "lognormal":
        return rng.lognormal(0.0, 0.5, size=m)
    raise ValueError(weights)


def planted_partition(n, blocks, deg_in, deg_cross, weights="unit", seed=0, dtype="float32", device=None):
    """SBM with `blocks` equal contiguous blocks (y = block id): n*deg_in/2 in-block pairs (u
    uniform, v uniform in u's block) and n*deg_cross/2 cross-block pairs (v uniform in another
    block); duplicates kept once, self-loops dropped; unit or lognormal(0, 0.5) weights."""
    rng = np.random.default_rng(seed)
    bs = n // blocks
    y = np.minimum(np.arange(n) // bs, blocks - 1).astype(np.int32)
    m_in, m_x = int(round(n * deg_in / 2)), int(round(n * deg_cross / 2))
    u1 = rng.integers(0, n, m_in)
    lo = y[u1].astype(np.int64) * bs
    hi = np.where(y[u1] == blocks - 1, n, lo + bs)
    v1 = lo + (rng.random(m_in) * (hi - lo)).astype(np.int64)
    u2 = rng.integers(0, n, m_x)
    other = (y[u2] + rng.integers(1, blocks, m_x)) % blocks if blocks > 1 else y[u2]
    lo2 = other.astype(np.int64) * bs
    hi2 = np.where(other == blocks - 1, n, lo2 + bs)
    v2 = lo2 + (rng.random(m_x) * (hi2 - lo2)).astype(np.int64)
    u, v = np.concatenate([u1, u2]), np.concatenate([v1, v2])
    w = _weights(rng, u.shape[0], weights)
    dev = _dev(device)
    A = symmetric_set(u, v, w, n, dtype, dev)
    name = f"sbm-n{n}-b{blocks}-d{deg_in:g}+{deg_cross:g}-{weights}"
    return Dataset(name, A, _t(y, dev), blocks, torch.arange(n, device=dev))


def er_graph(n, mean_deg, K, weights="unit", seed=0, dtype="float32", device=None) -> Dataset:
    """Erdos-Renyi: n*mean_deg/2 uniform pairs (set semantics), labels uniform in [0, K)."""
    rng = np.random.default_rng(seed)
    m = int(round(n * mean_deg / 2))
    u, v = rng.integers(0, n, m), rng.integers(0, n, m)
    w = _weights(rng, m, weights)
    y = rng.integers(0, K, n).astype(np.int32)
    dev = _dev(device)
    return Dataset(f"er-n{n}-d{mean_deg:g}-K{K}", symmetric_set(u, v, w, n, dtype, dev), _t(y, dev), K,
                   torch.arange(n, device=dev))


def label_mask(n, frac, seed=0, device=None) -> torch.Tensor:
    """Uniformly random labelled set of round(frac * n) vertices (bool, device)."""
    rng = np.random.default_rng(seed + 101)
    m = np.zeros(n, dtype=bool)
    m[rng.choice(n, int(round(frac * n)), replace=False)] = True
    return _t(m, _dev(device))


class EdgeUpdates:
    """Edge-update batches on a symmetric graph: `ins_frac` of each batch inserts uniform random
    non-edges (with the workload's weight law), the rest deletes uniform random existing edges.
    Tracks the live edge set on the host; batches are NumPy arrays (u, v, w) / (u, v)."""

    def __init__(self, A: CSR, seed=0, weights="unit"):
        self.n = A.shape[0]
        indptr = A.indptr.cpu().numpy().astype(np.int64)
        cols = A.indices.cpu().numpy().astype(np.int64)
        rows = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(indptr))
        up = rows < cols
        self.keys = np.sort(rows[up] * self.n + cols[up])
        self.rng = np.random.default_rng(seed + 7)
        self.weights = weights

    def next(self, size, ins_frac=0.5):
        n, rng = self.n, self.rng
        ni = int(round(size * ins_frac))
        nd = size - ni
        pick = rng.choice(self.keys.shape[0], nd, replace=False)
        dk = self.keys[pick]
        self.keys = np.delete(self.keys, pick)
        ik = np.zeros(0, dtype=np.int64)
        while ik.shape[0] < ni:
            need = ni - ik.shape[0]
            a, b = rng.integers(0, n, 2 * need + 16), rng.integers(0, n, 2 * need + 16)
            ok = a != b
            k = np.minimum(a, b)[ok] * n + np.maximum(a, b)[ok]
            pos = np.searchsorted(self.keys, k)
            pos = np.minimum(pos, self.keys.shape[0] - 1) if self.keys.shape[0] else pos
            absent = (self.keys.shape[0] == 0) | (self.keys[pos] != k) if self.keys.shape[0] else np.ones_like(k, bool)
            k = k[absent]
            k = k[~np.isin(k, ik)]
            _, first = np.unique(k, return_index=True)
            ik = np.concatenate([ik, k[np.sort(first)][:need]])
        self.keys = np.insert(self.keys, np.searchsorted(self.keys, np.sort(ik)), np.sort(ik))
        iw = _weights(rng, ni, self.weights).astype(np.float32)
        return dict(ins_u=(ik // n).astype(np.int32), ins_v=(ik % n).astype(np.int32), ins_w=iw,
                    del_u=(dk // n).astype(np.int32), del_v=(dk % n).astype(np.int32))


def from_npz(path, dtype="float32", seed=0, name=None, device=None) -> Dataset:
    """An edge list on disk (dynlp/graphs.py:176-184): arrays src, dst, y and optional w (default 1)
    and order (default a RandomState(seed + 1) permutation, the reference's draw); the graph is the
    symmetric coalesced CSR of the pairs (duplicates summed, self-loops dropped), K = max(y) + 1."""
    import os
    z = np.load(path)
    keys = set(z.files)
    y = np.asarray(z["y"]).astype(np.int32)
    n = int(y.shape[0])
    src, dst = np.asarray(z["src"]).astype(np.int64), np.asarray(z["dst"]).astype(np.int64)
    w = np.asarray(z["w"]) if "w" in keys else np.ones(src.shape[0])
    order = np.asarray(z["order"]).astype(np.int64) if "order" in keys else np.random.RandomState(seed + 1).permutation(n)
    dev = _dev(device)
    A = symmetric_from_pairs(src, dst, w, n, dtype, dev)
    return Dataset(name or os.path.basename(path), A, _t(y, dev), int(y.max()) + 1 if n else 0, _t(order, dev))


def save_npz(ds: Dataset, path, with_order=True):
    """The edge-list format of `from_npz` (the reference's graph cache, dynlp/graphs.py:201-203): the
    upper triangle of A as src < dst with weights w, the labels y and (optionally) the order."""
    A = ds.A
    rows = csr_rows(A).long()
    up = rows < A.indices.long()
    arrays = dict(src=rows[up].cpu().numpy(), dst=A.indices.long()[up].cpu().numpy(),
                  w=A.data[up].cpu().numpy(), y=ds.y.cpu().numpy().astype(np.int32))
    if with_order:
        arrays["order"] = ds.order.cpu().numpy().astype(np.int64)
    np.savez(path, **arrays)
    return path


def load(spec: str, *, n=100_000, K=2, deg=10.0, p_in=0.85, seed=0, dtype="float32", data_dir=DATA_DIR,
         device=None) -> Dataset:
    """dynlp/graphs.py:207-214: the synthetic families, edge lists on disk (`*.npz`) and the cached
    synth kNN sets (`synthN`); the IMDB review graph (downloads) is out of scope."""
    if spec == "sbm":
        return sbm(n, K, deg, p_in, seed, dtype, device)
    if spec == "er":
        return erdos_renyi(n, K, deg, seed, dtype, device)
    if spec.endswith(".npz"):
        return from_npz(spec, dtype, seed, device=device)
    return from_npz(build_cached(spec, data_dir, device), dtype, seed, name=spec, device=device)

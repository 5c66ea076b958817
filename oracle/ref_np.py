"""NumPy/SciPy restatement of the reference's hot path (TEST INFRASTRUCTURE ONLY: the checker).

Each function cites the reference (shishir9159/DynLPlus) file:line it restates. Arrays are NumPy,
sparse matrices SciPy CSR. Pinned against the reference's own outputs in tests/golden/*.npz.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as ssp
import scipy.sparse.csgraph as csg


# ---------------------------------------------------------------------------------------------
# graphs (dynlp/graphs.py)
# ---------------------------------------------------------------------------------------------
def coalesce(rows, cols, vals, n, dtype):
    """Canonical CSR: duplicates summed, self-loops dropped (dynlp/graphs.py:36-44)."""
    keep = rows != cols
    coo = ssp.coo_matrix((np.asarray(vals)[keep].astype(dtype),
                          (np.asarray(rows)[keep].astype(np.int32), np.asarray(cols)[keep].astype(np.int32))),
                         shape=(n, n))
    coo.sum_duplicates()
    A = coo.tocsr()
    A.sum_duplicates()
    return A


def symmetric_from_pairs(u, v, w, n, dtype):
    """dynlp/graphs.py:47-48."""
    return coalesce(np.concatenate([u, v]), np.concatenate([v, u]), np.concatenate([w, w]), n, dtype)


def csr_rows(A):
    """Row index of every stored entry (dynlp/graphs.py:62-64)."""
    return np.repeat(np.arange(A.shape[0], dtype=np.int32), np.diff(A.indptr))


# ---------------------------------------------------------------------------------------------
# connected components (dynlp/cc.py:8-23)
# ---------------------------------------------------------------------------------------------
def connected_components(n, rows, cols):
    """Hook (scatter-min of the larger root to the smaller) + full pointer jumping until no edge
    crosses two labels, then the rank relabel by unique (dynlp/cc.py:8-23)."""
    if n == 0:
        return np.zeros(0, dtype=np.int32), 0
    lab = np.arange(n, dtype=np.int32)
    rows, cols = np.asarray(rows, dtype=np.int32), np.asarray(cols, dtype=np.int32)
    while True:
        lr, lc = lab[rows], lab[cols]
        diff = lr != lc
        if not diff.any():
            break
        lr, lc = lr[diff], lc[diff]
        np.minimum.at(lab, np.maximum(lr, lc), np.minimum(lr, lc))
        while True:
            nxt = lab[lab]
            if (nxt == lab).all():
                break
            lab = nxt
    uniq, inv = np.unique(lab, return_inverse=True)
    return inv.astype(np.int32).ravel(), int(uniq.shape[0])


def connected_components_fast(n, rows, cols):
    """Same labels as connected_components for large inputs: SciPy labels components in the order
    of their first vertex when scanning 0..n-1, which is the rank of the minimum vertex id."""
    if n == 0:
        return np.zeros(0, dtype=np.int32), 0
    G = ssp.coo_matrix((np.ones(len(rows), dtype=np.int8), (np.asarray(rows), np.asarray(cols))), shape=(n, n))
    nc, lab = csg.connected_components(G, directed=False)
    return lab.astype(np.int32), int(nc)


def min_vertex_roots(labels):
    """parent[v] = smallest vertex of v's component, from rank labels."""
    n = labels.shape[0]
    first = np.full(labels.max() + 1 if n else 0, n, dtype=np.int64)
    np.minimum.at(first, labels, np.arange(n))
    return first[labels].astype(np.int32)


# ---------------------------------------------------------------------------------------------
# kernels (dynlp/kernels.py) -- the kernels' definitions, as the reference's fallbacks state them
# ---------------------------------------------------------------------------------------------
def spmm_axpy(W, X, a=None, b=1.0):
    """Y = a*X + b*(W@X) (dynlp/kernels.py:140-166, :240-266)."""
    Y = b * (W @ X)
    if a is not None:
        Y = a[:, None] * X + Y
    return Y.astype(X.dtype)


def frontier_jacobi(W, frontier, X, rhs, diag, delta):
    """(rhs[f] + W[f] @ X) / diag[f] and the changed flag (dynlp/kernels.py:473-474)."""
    Y = (rhs[frontier] + W[frontier] @ X) / diag[frontier][:, None]
    return Y, (np.abs(Y - X[frontier]) > delta).any(axis=1)


def push_scatter(W, frontier, D, R, mark):
    """R += W[:, frontier] @ D for symmetric W; mark touched (dynlp/kernels.py:483-486)."""
    sub = W[frontier]
    seg = np.searchsorted(sub.indptr[1:], np.arange(sub.nnz), side="right")
    np.add.at(R, sub.indices, sub.data[:, None] * D[seg])
    mark[sub.indices] = 1


def mark_neighbors(W, rows, mark):
    """dynlp/kernels.py:492."""
    mark[W[rows].indices] = 1


# ---------------------------------------------------------------------------------------------
# solvers (dynlp/solvers.py)
# ---------------------------------------------------------------------------------------------
def apply_A(W, diag, X):
    """diag*X - W@X (dynlp/solvers.py:46-49)."""
    return diag[:, None] * X - W @ X


def rho_cols(diag, R):
    """max_u |R_uc| / diag_u (dynlp/solvers.py:52-54)."""
    return (np.abs(R) / diag[:, None]).max(axis=0) if R.shape[0] else np.zeros(R.shape[1])


def violation(diag, R, eps_d):
    """max |R_uc| / (eps_c diag_u) (dynlp/solvers.py:57-59)."""
    return float((np.abs(R) / (eps_d[None, :] * diag[:, None])).max()) if R.shape[0] else 0.0


def pcg(W, diag, Z, rhs, eps, M=None, max_iter=100_000, patience=400):
    """Block PCG, one CG per column, until |r_c| <= eps_c diag (dynlp/solvers.py:66-97).
    Returns (Z, iterations)."""
    M = M or (lambda R: R / diag[:, None])
    eps_d = np.asarray(eps, dtype=Z.dtype)
    R = rhs - apply_A(W, diag, Z)
    best = violation(diag, R, eps_d)
    it = 0
    if best <= 1:
        return Z, it
    P = Y = M(R)
    rz, stall = (R * Y).sum(axis=0), 0
    for _ in range(max_iter):
        AP = apply_A(W, diag, P)
        pAp = (P * AP).sum(axis=0)
        alpha = np.where(pAp > 0, rz / np.where(pAp > 0, pAp, 1), 0)
        Z += alpha[None, :] * P
        R -= alpha[None, :] * AP
        it += 1
        v = violation(diag, R, eps_d)
        if v <= 1:
            R = rhs - apply_A(W, diag, Z)
            if (v := violation(diag, R, eps_d)) <= 1:
                break
        best, stall = (v, 0) if v < 0.9 * best else (best, stall + 1)
        if stall >= patience:
            break
        Y = M(R)
        rz_new = (R * Y).sum(axis=0)
        P = Y + np.where(rz > 0, rz_new / np.where(rz > 0, rz, 1), 0)[None, :] * P
        rz = rz_new
    return Z, it


def push(W, diag, Z, R, eps, budget_edges=None, max_iter=10**7, record=False):
    """Synchronous residual push = Jacobi on the violating set (dynlp/solvers.py:100-125).

    Returns (Z, R, converged, iterations, rounds) where rounds lists, per round, the sorted
    candidate set that pushed and the sorted touched set (when record=True)."""
    eps_d = np.asarray(eps, dtype=Z.dtype)
    n = W.shape[0]

    def violating(idx):
        return (np.abs(R[idx]) > eps_d[None, :] * diag[idx][:, None]).any(axis=1)

    all_idx = np.arange(n, dtype=np.int32)
    cand, edges, it, best, stall = all_idx[violating(all_idx)], 0, 0, float("inf"), 0
    rounds = []
    indptr = W.indptr
    while cand.shape[0] and it < max_iter:
        D = R[cand] / diag[cand][:, None]
        Z[cand] += D
        R[cand] = 0
        mark = np.zeros(n, dtype=np.uint8)
        mark[cand] = 1
        edges += int((indptr[cand + 1] - indptr[cand]).sum())
        push_scatter(W, cand, D, R, mark)
        touched = np.flatnonzero(mark).astype(np.int32)
        if record:
            rounds.append((cand.copy(), touched.copy()))
        cand, it = touched[violating(touched)], it + 1
        if it % 32 == 0:
            if budget_edges is not None and edges > budget_edges:
                break
            v = violation(diag, R, eps_d)
            best, stall = (v, 0) if v < 0.99 * best else (best, stall + 1)
            if stall >= 8:
                break
    return Z, R, cand.shape[0] == 0, it, rounds


def dynlp_frontier(W, diag, rhs, X, seed_rows, delta, max_iter=10**7, record=False):
    """DynLP's frontier Jacobi loop (dynlp/solvers.py:227-238): returns (X, iterations, frontiers)."""
    frontier = np.asarray(seed_rows, dtype=np.int32)
    it, fronts = 0, []
    n = W.shape[0]
    while frontier.shape[0] and it < max_iter:
        if record:
            fronts.append(frontier.copy())
        Y, ch = frontier_jacobi(W, frontier, X, rhs, diag, delta)
        it += 1
        upd = frontier[ch]
        if not upd.shape[0]:
            break
        X[upd] = Y[ch]
        mark = np.zeros(n, dtype=np.uint8)
        mark[upd] = 1
        mark_neighbors(W, upd, mark)
        frontier = np.flatnonzero(mark).astype(np.int32)
    return X, it, fronts


def predict(F, K):
    """dynlp/solvers.py:166-167."""
    return (F[:, 0] > 0.5).astype(np.int32) if K == 2 else F.argmax(axis=1).astype(np.int32)


# ---------------------------------------------------------------------------------------------
# system assembly (dynlp/stream.py:142-177)
# ---------------------------------------------------------------------------------------------
def build_system(A, y, K, active, labeled, eta=0.0, dtype=np.float64):
    """The grounded harmonic system of one batch (dynlp/stream.py:142-167, without the new-vertex
    components): U = active unlabelled vertices whose component (within active unlabelled) holds
    label weight; W = A[U,U] in CSR order; B = A @ onehot(y_L); s = sum(B)+eta; diag = s+rowsum(W);
    rhs = B (class 1 only when K == 2)."""
    n = A.shape[0]
    rows, cols = csr_rows(A), A.indices
    prior = np.full(1 if K == 2 else K, 0.5 if K == 2 else 1.0 / K)
    onehot = np.zeros((n, K), dtype=dtype)
    li = np.flatnonzero(active & labeled)
    onehot[li, y[li]] = 1
    Bfull = A.astype(dtype) @ onehot
    Um = active & ~labeled
    U0 = np.flatnonzero(Um)
    loc = np.full(n, -1, dtype=np.int32)
    loc[U0] = np.arange(U0.shape[0], dtype=np.int32)
    keep = Um[rows] & Um[cols]
    lab, ncomp = connected_components_fast(int(U0.shape[0]), loc[rows[keep]], loc[cols[keep]])
    gw = np.zeros(ncomp, dtype=dtype)
    np.add.at(gw, lab, Bfull[U0].sum(axis=1))
    grounded = gw[lab] > 0
    Um = Um.copy()
    Um[U0[~grounded]] = False
    U = np.flatnonzero(Um)
    n_u = U.shape[0]
    loc = np.full(n, -1, dtype=np.int32)
    loc[U] = np.arange(n_u, dtype=np.int32)
    keep = Um[rows] & Um[cols]
    indptr = np.zeros(n_u + 1, dtype=np.int32)
    indptr[1:] = np.cumsum(np.bincount(loc[rows[keep]], minlength=n_u))
    W = ssp.csr_matrix((A.data[keep].astype(dtype), loc[cols[keep]], indptr), shape=(n_u, n_u))
    Bm = Bfull[U]
    s = Bm.sum(axis=1) + eta
    diag = s + np.asarray(W.sum(axis=1)).ravel()
    rhs = (Bm[:, 1:2] if K == 2 else Bm) + eta * prior[None, :]
    # cc_labels: the reference's component labels of the active unlabelled vertices U0 (stream.py:153)
    return dict(U=U, W=W, s=s, diag=diag, B=Bm, rhs=rhs, prior=prior, n_ungrounded=int((~grounded).sum()),
                U0=U0, cc_labels=lab, n_comp=ncomp)


# ---------------------------------------------------------------------------------------------
# edge batches (new functionality; set semantics on the symmetric graph)
# ---------------------------------------------------------------------------------------------
def apply_edges(A, ins_u, ins_v, ins_w, del_u, del_v):
    """A' = A with the undirected edges (del_u, del_v) removed, then (ins_u, ins_v, ins_w) set.
    Deletions of absent edges and self-loops are ignored; an insertion of a present edge sets its
    weight; within a batch deletions apply before insertions, and a repeated insertion keeps the
    last weight given."""
    n = A.shape[0]
    A = A.tocoo()
    key = A.row.astype(np.int64) * n + A.col
    val = A.data.copy()
    du, dv = np.asarray(del_u, dtype=np.int64), np.asarray(del_v, dtype=np.int64)
    dkeys = np.concatenate([du * n + dv, dv * n + du])
    live = ~np.isin(key, dkeys)
    key, val = key[live], val[live]
    iu, iv = np.asarray(ins_u, dtype=np.int64), np.asarray(ins_v, dtype=np.int64)
    iw = np.asarray(ins_w, dtype=A.dtype)
    ok = iu != iv
    iu, iv, iw = iu[ok], iv[ok], iw[ok]
    ikeys = np.concatenate([iu * n + iv, iv * n + iu])
    iw2 = np.concatenate([iw, iw])
    # last occurrence wins for repeated keys
    order = np.arange(ikeys.shape[0])
    uk, first_rev = np.unique(ikeys[::-1], return_index=True)
    last = order[::-1][first_rev]
    keep = ~np.isin(key, uk)
    key = np.concatenate([key[keep], uk])
    val = np.concatenate([val[keep], iw2[last]])
    o = np.argsort(key, kind="stable")
    key, val = key[o], val[o]
    return ssp.csr_matrix((val, (key // n, key % n)), shape=(n, n))


def relres(W, diag, Z, rhs):
    """max_c ||rhs_c - A Z_c||_2 / ||rhs_c||_2 in float64."""
    W64 = W.astype(np.float64)
    R = rhs.astype(np.float64) - apply_A(W64, diag.astype(np.float64), Z.astype(np.float64))
    num = np.sqrt((R * R).sum(axis=0))
    den = np.sqrt((rhs.astype(np.float64) ** 2).sum(axis=0))
    return float((num / np.where(den > 0, den, 1)).max())


# ---------------------------------------------------------------------------------------------
# aggregation AMG (dynlp/amg.py)
# ---------------------------------------------------------------------------------------------
def handshake(n, rows, cols, w, rounds):
    """Heavy-edge handshake matching; unmatched vertices join a matched neighbour (amg.py:32-64)."""
    agg = np.full(n, -1, dtype=np.int64)
    matched = np.zeros(n, dtype=bool)
    ar = np.arange(n, dtype=np.int64)

    def best_choice(er, ec, ew):
        best = np.full(n, -np.inf, dtype=ew.dtype)
        np.maximum.at(best, er, ew)
        tie = ew >= best[er]
        choice = np.full(n, n, dtype=np.int64)
        np.minimum.at(choice, er[tie], ec[tie].astype(np.int64))
        return choice

    for _ in range(rounds):
        ok = ~matched[rows] & ~matched[cols]
        if not ok.any():
            break
        choice = best_choice(rows[ok], cols[ok], w[ok])
        has = choice < n
        partner = np.where(has, choice, 0)
        mutual = has & (choice[partner] == ar)
        matched |= mutual
        agg = np.where(mutual, np.minimum(ar, partner), agg)
    ok = ~matched[rows] & matched[cols]
    if ok.any():
        choice = best_choice(rows[ok], cols[ok], w[ok])
        has = choice < n
        agg[has] = agg[choice[has]]
    left = agg < 0
    agg[left] = ar[left]
    uniq, inv = np.unique(agg, return_inverse=True)
    return inv.ravel().astype(np.int64), int(uniq.shape[0])


def coarsen(W, s, agg, nc):
    """W_c sums the inter-aggregate weights, s_c the grounding (amg.py:67-74)."""
    rows = csr_rows(W)
    rc, cc = agg[rows], agg[W.indices]
    off = rc != cc
    Wc = coalesce(rc[off], cc[off], W.data[off], nc, W.data.dtype)
    sc = np.zeros(nc, dtype=s.dtype)
    np.add.at(sc, agg, s)
    return Wc, sc


class AMGOracle:
    """V-cycle preconditioner (amg.py:77-134), same defaults."""

    def __init__(self, W, s, *, max_coarse=1500, passes=2, rounds=3, omega=0.7, nu=1, max_levels=25, min_ratio=0.85,
                 coarse_sweeps=20):
        self.omega, self.nu, self.coarse_sweeps = omega, nu, coarse_sweeps
        self.levels = []
        dt = W.data.dtype
        n = W.shape[0]
        cur = dict(W=W, s=s, diag=s + W @ np.ones(n, dtype=dt))
        while n > max_coarse and len(self.levels) < max_levels:
            agg = np.arange(n, dtype=np.int64)
            nc, Wp = n, cur["W"]
            for _ in range(passes):
                a2, nc2 = handshake(Wp.shape[0], csr_rows(Wp), Wp.indices, Wp.data, rounds)
                agg = a2[agg]
                Wp, _ = coarsen(Wp, np.zeros(Wp.shape[0], dtype=dt), a2, nc2)
                nc = nc2
            if nc > min_ratio * n:
                break
            Wc, sc = coarsen(cur["W"], cur["s"], agg, nc)
            cur["agg"] = agg
            self.levels.append(cur)
            cur = dict(W=Wc, s=sc, diag=sc + Wc @ np.ones(nc, dtype=dt))
            n = nc
        self.coarse = cur
        self.inv = None
        if n <= 4 * max_coarse:
            Ad = -cur["W"].toarray().astype(np.float64)
            Ad[np.arange(n), np.arange(n)] += cur["diag"].astype(np.float64)
            self.inv = np.linalg.inv(Ad)
        self.sizes = [L["W"].shape[0] for L in self.levels] + [n]

    def _apply(self, L, X):
        return L["diag"][:, None] * X - L["W"] @ X

    def _smooth(self, L, X, R, sweeps):
        for _ in range(sweeps):
            X = X + self.omega * (R - self._apply(L, X)) / L["diag"][:, None]
        return X

    def _cycle(self, lvl, R):
        if lvl == len(self.levels):
            L = self.coarse
            if self.inv is not None:
                return self.inv @ R
            X = self.omega * R / L["diag"][:, None]
            return self._smooth(L, X, R, self.coarse_sweeps - 1)
        L = self.levels[lvl]
        X = self.omega * R / L["diag"][:, None]
        X = self._smooth(L, X, R, self.nu - 1)
        nc = (self.levels[lvl + 1]["W"] if lvl + 1 < len(self.levels) else self.coarse["W"]).shape[0]
        Rr = R - self._apply(L, X)
        Rc = np.zeros((nc, R.shape[1]))
        np.add.at(Rc, L["agg"], Rr)
        X = X + self._cycle(lvl + 1, Rc)[L["agg"]]
        return self._smooth(L, X, R, self.nu)

    def __call__(self, R):
        return self._cycle(0, R)


# ---------------------------------------------------------------------------------------------
# vertex-arrival streams and new-vertex warm starts (dynlp/stream.py:61-177, dynlp/cc.py:26-83,
# dynlp/solvers.py:128-163)
# ---------------------------------------------------------------------------------------------
def stream_schedule(y, K, order, label_frac=0.01, init_frac=0.1, n_batches=10, del_frac=0.1, seed=0):
    """The reference Stream's up-front draws (dynlp/stream.py:89-128) on a NumPy RandomState:
    the labelled set, the arrival order (one labelled vertex of every class moved into the initial
    snapshot), the initial size n0 and the (inserted, deleted) vertex lists of every batch."""
    y = np.asarray(y)
    n = y.shape[0]
    rs = np.random.RandomState(seed + 7)
    cand = np.flatnonzero(y >= 0)
    labeled = np.zeros(n, dtype=bool)
    labeled[cand[rs.permutation(cand.shape[0])[: max(K, int(label_frac * n))]]] = True
    order = np.array(order, dtype=np.int64, copy=True)
    n0 = max(int(init_frac * n), 2 * K)
    pos = np.empty(n, dtype=np.int64)
    pos[order] = np.arange(n)
    for c in range(K):
        lc = np.flatnonzero(labeled & (y == c))
        if lc.shape[0] == 0:
            lc = np.flatnonzero(y == c)[:1]
            labeled[lc] = True
        if lc.shape[0] and int(pos[lc].min()) >= n0:
            free = np.flatnonzero(~labeled[order[:n0]])
            v, j = int(lc[0]), int(free[int(rs.randint(0, free.shape[0]))])
            a, pv = int(order[j]), int(pos[v])
            order[j], order[pv], pos[v], pos[a] = v, a, j, pv
    chunks = np.array_split(order[n0:], n_batches) if n_batches > 0 else []
    active = np.zeros(n, dtype=bool)
    sched = []
    for t in range(1 + len(chunks)):
        ins = order[:n0] if t == 0 else chunks[t - 1]
        dele = np.zeros(0, dtype=np.int64)
        if t:
            pool = np.flatnonzero(active & ~labeled)
            nd = min(int(del_frac * ins.shape[0]), max(pool.shape[0] - 1, 0))
            if nd > 0:
                dele = pool[rs.permutation(pool.shape[0])[:nd]]
        active[ins] = True
        active[dele] = False
        sched.append((np.asarray(ins, np.int64), np.asarray(dele, np.int64)))
    return labeled, order, n0, sched


def _lightest_edge(nc, cu, cv, de):
    """Per component with an outgoing edge: the lightest one (ties: smallest other side)
    (dynlp/cc.py:26-34)."""
    best = np.full(nc, np.inf, dtype=np.float32)
    np.minimum.at(best, cu, de)
    nb = np.full(nc, nc, dtype=np.int32)
    sel = de <= best[cu]
    np.minimum.at(nb, cu[sel], cv[sel])
    c = np.flatnonzero(nb < nc).astype(np.int32)
    return c, nb[c], best[c]


def fh_components(m, rows, cols, d, k, ground=None):
    """Felzenszwalb-Huttenlocher merging in Boruvka rounds (dynlp/cc.py:37-73): every component
    takes its lightest outgoing edge and merges across it when d <= min over both sides of
    Int(C) + k / |C|; then, with `ground`, components without ground join their lightest
    neighbour until none is left."""
    lab = np.arange(m, dtype=np.int32)
    Int = np.zeros(m, dtype=np.float32)
    size = np.ones(m, dtype=np.float32)
    rows, cols, d = np.asarray(rows, np.int32), np.asarray(cols, np.int32), np.asarray(d, np.float32)
    nc, fh = m, True
    while rows.shape[0]:
        cu, cv = lab[rows], lab[cols]
        ext = cu != cv
        if not fh:
            g = np.zeros(nc, dtype=np.float32)
            np.add.at(g, lab, ground)
            ext &= g[cu] == 0
        if not ext.any():
            break
        c, t, dc = _lightest_edge(nc, cu[ext], cv[ext], d[ext])
        if fh:
            ok = dc <= np.minimum(Int[c] + k / size[c], Int[t] + k / size[t])
            if not ok.any():
                if ground is None:
                    break
                fh = False
                continue
            c, t, dc = c[ok], t[ok], dc[ok]
        root, nc = connected_components(nc, c, t)
        Int2 = np.zeros(nc, dtype=np.float32)
        size2 = np.zeros(nc, dtype=np.float32)
        np.maximum.at(Int2, root, Int)
        np.maximum.at(Int2, root[c], dc)
        np.add.at(size2, root, size)
        lab, Int, size = root[lab], Int2, size2
    return lab, nc


def new_components(m, lr, lc, w, tau, wmax, ground):
    """DynLP step 1 for the m new vertices (dynlp/stream.py:67-81): components over edges
    heavier than tau among new vertices, and the adaptive (FH) ones on dissimilarities 1 - w/wmax
    scaled by each endpoint's mean dissimilarity (dynlp/cc.py:76-83)."""
    w = np.asarray(w)
    on = w > 0
    s = np.zeros(m, dtype=np.float32)
    cnt = np.zeros(m, dtype=np.float32)
    np.add.at(s, lr, np.where(on, 1 - w / wmax, 0).astype(np.float32))
    np.add.at(cnt, lr, on.astype(np.float32))
    s = s / np.maximum(cnt, 1) + 1e-6
    e = on & (lc >= 0)
    r, c, we = lr[e], lc[e], w[e]
    heavy = we > tau
    out = {"tau": connected_components(m, r[heavy], c[heavy])}
    if m == 0:
        out["fh"] = (np.zeros(0, dtype=np.int32), 0)
    else:
        d = (1 - we / wmax) / np.sqrt(s[r] * s[c])
        out["fh"] = fh_components(m, r, c, d, float(d.mean()) if d.shape[0] else 0.0,
                                  np.asarray(ground).astype(np.float32))
    return out


def stream_system(A, y, K, active, labeled, prevU, ins, dele, tau, wmax, eta=0.0, dtype=np.float64):
    """Stream._build (dynlp/stream.py:142-177): the grounded system plus the new rows (not in U at
    the previous batch), DynLP's seed (new rows and neighbours of inserted/deleted vertices) and
    the new vertices' components."""
    S = build_system(A, y, K, active, labeled, eta=eta, dtype=dtype)
    U, W, Bm = S["U"], S["W"], S["B"]
    n, n_u = A.shape[0], U.shape[0]
    is_new = ~prevU[U]
    touch = np.zeros(n, dtype=dtype)
    touch[ins], touch[dele] = 1, 1
    seed = is_new | ((A.astype(dtype) @ touch)[U] > 0)
    new = np.flatnonzero(is_new)
    nl = np.full(n_u, -1, dtype=np.int32)
    nl[new] = np.arange(new.shape[0], dtype=np.int32)
    rW = csr_rows(W)
    on = is_new[rW]
    S.update(is_new=is_new, seed=seed,
             comps=new_components(int(is_new.sum()), nl[rW[on]], nl[W.indices[on]], W.data[on], tau, wmax,
                                  Bm[is_new].sum(axis=1)))
    return S


def _comp_avg(lab, nc, S_rows, T_rows, fallback):
    """Per component of the new vertices: sum S / sum T (T = 0: fallback) (dynlp/solvers.py:128-135)."""
    S = np.zeros((nc,) + S_rows.shape[1:], dtype=S_rows.dtype)
    T = np.zeros(nc, dtype=S_rows.dtype)
    np.add.at(S, lab, S_rows)
    np.add.at(T, lab, T_rows)
    ok = T > 0
    Tn = np.where(ok, T, 1)
    if S.ndim == 2:
        return np.where(ok[:, None], S / Tn[:, None], fallback)
    return np.where(ok, S / Tn, fallback)


def supernode_init(W, B, K, prior, is_new, comps, X, known=None, comp="tau"):
    """New rows start at their component's average (dynlp/solvers.py:138-153): the share of the
    component's weight to each labelled class (known=None, DynLP's rule), or with `known` the
    weighted average over labelled and known neighbours."""
    new = np.flatnonzero(is_new)
    if new.shape[0] == 0:
        return X
    Bc = B[:, 1:2] if K == 2 else B
    s_, t = Bc[new], B[new].sum(axis=1)
    if known is not None:
        kf = known.astype(X.dtype)
        Wn = W[new]
        s_ = s_ + Wn @ (X * kf[:, None])
        t = t + Wn @ kf
    lab, nc = comps[comp]
    X = X.copy()
    X[new] = _comp_avg(lab, nc, s_, t, prior[None, :])[lab]
    return X


def init_h(W, B, is_new, comps, H, known, fallback, comp="fh"):
    """New rows: h = 1 + the component's weighted average h of known neighbours (labelled ones
    count with h = 0) (dynlp/solvers.py:156-163)."""
    new = np.flatnonzero(is_new)
    H = H.copy()
    if new.shape[0]:
        kf = known.astype(H.dtype)
        Wn = W[new]
        lab, nc = comps[comp]
        hc = _comp_avg(lab, nc, Wn @ (H[:, 0] * kf), B[new].sum(axis=1) + Wn @ kf, fallback - 1) + 1
        H[new, 0] = hc[lab]
    return H

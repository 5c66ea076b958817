"""Connected components: bit-exact labels against the reference's outputs and the oracle (GPU)."""
import numpy as np
import pytest
import torch

from conftest import golden_csr, load_golden
from dynlplus_b200 import cc
from dynlplus_b200.backend import CSR
from oracle import ref_np as O

pytestmark = pytest.mark.gpu


def T(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def test_matches_reference_golden():
    g = load_golden("cc.npz")
    for i in range(int(g["ncases"])):
        n = int(g[f"c{i}_n"])
        lab, nc = cc.connected_components(n, T(g[f"c{i}_rows"]), T(g[f"c{i}_cols"]))
        np.testing.assert_array_equal(lab.cpu().numpy(), g[f"c{i}_labels"])
        assert nc == int(g[f"c{i}_ncomp"])


@pytest.mark.parametrize("n,m", [(1, 0), (10, 5), (100_000, 50_000), (1_000_000, 5_000_000), (2_000_000, 800_000)])
def test_random_graphs_match_oracle(n, m):
    rs = np.random.RandomState(n % 97)
    r, c = rs.randint(0, n, m), rs.randint(0, n, m)
    lab, nc = cc.connected_components(n, T(r.astype(np.int32)), T(c.astype(np.int32)))
    want, wnc = O.connected_components_fast(n, r, c)
    np.testing.assert_array_equal(lab.cpu().numpy(), want)
    assert nc == wnc
    roots = cc.min_vertex_roots(n, T(r.astype(np.int32)), T(c.astype(np.int32)))
    np.testing.assert_array_equal(roots.cpu().numpy(), O.min_vertex_roots(want))


def test_endpoint_out_of_range_is_an_error():
    with pytest.raises(ValueError):
        cc.connected_components(4, T(np.array([0, 7], np.int32)), T(np.array([1, 2], np.int32)))


def test_graph_components_with_sink_match_grounding():
    """The grounding check of Stream._build (dynlp/stream.py:150-159) on the reference's system
    fixture: vertices whose component reaches a labelled vertex are exactly U."""
    g = load_golden("system.npz")
    for b in (0, 2):
        p = f"b{b}"
        A = golden_csr(g, f"{p}_A")
        act, lab = g[f"{p}_active"], g[f"{p}_labeled"]
        G = CSR.from_scipy(A)
        vmask = T((act & ~lab).astype(np.uint8))
        sink = T((act & lab).astype(np.uint8))
        parent, err = cc.graph_components(G, vmask, sink)
        assert int(err.item()) == 0
        par = parent.cpu().numpy()
        n = A.shape[0]
        U = np.flatnonzero((act & ~lab) & (par[:n] == par[n]))
        np.testing.assert_array_equal(U, g[f"{p}_U"])
        assert par[n] == par[par[n]]  # compressed


@pytest.mark.parametrize("n,deg,seed", [(5, 2.0, 0), (50, 1.0, 1), (200_000, 6.0, 2), (300_000, 1.2, 3)])
def test_graph_components_sampled_order_matches_oracle(n, deg, seed):
    """The sampling-then-skip order (with a workspace) and the hook-every-entry order (without)
    give the oracle's min-vertex-id roots, sink included, on masked random graphs: a dense one
    (one dominant component) and a sparse one (many small components)."""
    import scipy.sparse as ssp
    from dynlplus_b200 import _lib
    from dynlplus_b200.backend import ptr, stream
    rs = np.random.RandomState(seed)
    m = int(n * deg / 2)
    u, v = rs.randint(0, n, m), rs.randint(0, n, m)
    keep = u != v
    A = ssp.coo_matrix((np.ones(2 * keep.sum()), (np.r_[u[keep], v[keep]], np.r_[v[keep], u[keep]])),
                       shape=(n, n)).tocsr()
    A.sum_duplicates()
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    key = np.minimum(rows, A.indices).astype(np.int64) * n + np.maximum(rows, A.indices)
    A.data = np.where(key * 2654435761 % 1000 < 50, 0.0, 1.0)  # inert pairs (weight 0), symmetric
    labeled = rs.rand(n) < 0.01
    vmask = (rs.rand(n) < 0.97) & ~labeled
    G = CSR.from_scipy(A, dtype="float32")
    live = np.asarray(A.data) != 0
    r, c = rows[live], A.indices[live]
    inm = vmask[r] & vmask[c]
    tos = vmask[r] & labeled[c]
    want = O.min_vertex_roots(O.connected_components_fast(n + 1, np.r_[r[inm], r[tos]],
                                                          np.r_[c[inm], np.full(tos.sum(), n)])[0])
    vm, sk = T(vmask.astype(np.uint8)), T(labeled.astype(np.uint8))  # held until the launches are done
    got = []
    for use_ws in (True, False):
        parent = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        ws = torch.empty(_lib.lib().dlp_cc_graph_workspace_bytes(), dtype=torch.uint8, device="cuda")
        indptr = G.indptr
        _lib.call("dlp_cc_graph", n, ptr(indptr[:-1]), ptr(indptr[1:]), ptr(G.indices), ptr(G.data), 0,
                  ptr(vm), ptr(sk), ptr(parent), ptr(err),
                  ptr(ws) if use_ws else None, ws.numel() if use_ws else 0, stream())
        assert int(err.item()) == 0
        got.append(parent.cpu().numpy())
    np.testing.assert_array_equal(got[0], want)
    np.testing.assert_array_equal(got[1], want)


def _grounded_oracle(A, vmask, labeled):
    n = A.shape[0]
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    live = np.asarray(A.data) != 0
    r, c = rows[live], A.indices[live]
    inm = vmask[r] & vmask[c]
    tos = vmask[r] & ~vmask[c] & labeled[c]
    par = O.min_vertex_roots(O.connected_components_fast(n + 1, np.r_[r[inm], r[tos]],
                                                         np.r_[c[inm], np.full(tos.sum(), n)])[0])
    return vmask & (par[:n] == par[n])


@pytest.mark.parametrize("case", ["dense", "sparse", "path"])
def test_ground_reach_matches_components(case):
    """Reachability grounding (in place over a previous grounded set) equals the component test of
    the reference's Stream._build (dynlp/stream.py:150-159): a dense random graph settles in a few
    sweeps; a long path (label at its far end) exceeds the sweep budget and finishes with the
    union-find; a near-critical sparse graph takes either route."""
    import scipy.sparse as ssp
    rs = np.random.RandomState({"dense": 5, "sparse": 6, "path": 7}[case])
    if case == "path":
        n = 5000
        u = np.arange(n - 1)
        A = ssp.coo_matrix((np.ones(2 * (n - 1)), (np.r_[u, u + 1], np.r_[u + 1, u])), shape=(n, n)).tocsr()
        labeled = np.zeros(n, bool)
        labeled[n - 1] = True
        vmask = ~labeled
        vmask[n // 3] = False  # cuts the path: the first third stays ungrounded
    else:
        n, deg = (200_000, 6.0) if case == "dense" else (300_000, 1.2)
        m = int(n * deg / 2)
        u, v = rs.randint(0, n, m), rs.randint(0, n, m)
        keep = u != v
        A = ssp.coo_matrix((np.ones(2 * keep.sum()), (np.r_[u[keep], v[keep]], np.r_[v[keep], u[keep]])),
                           shape=(n, n)).tocsr()
        A.sum_duplicates()
        rows = np.repeat(np.arange(n), np.diff(A.indptr))
        key = np.minimum(rows, A.indices).astype(np.int64) * n + np.maximum(rows, A.indices)
        A.data = np.where(key * 2654435761 % 1000 < 50, 0.0, 1.0)
        labeled = rs.rand(n) < 0.01
        vmask = (rs.rand(n) < 0.97) & ~labeled
    want = _grounded_oracle(A, vmask, labeled)
    G = CSR.from_scipy(A, dtype="float32")
    old = rs.rand(n) < 0.5
    umask = T(old.astype(np.uint8))
    in_t = torch.zeros(n, dtype=torch.uint8, device="cuda")
    vm, sk = T(vmask.astype(np.uint8)), T(labeled.astype(np.uint8))
    changes, sweeps = cc.ground_reach(G, vm, sk, umask, in_t, w=G.data)
    got = umask.cpu().numpy().astype(bool)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(in_t.cpu().numpy().astype(bool), got != old)
    assert changes == int((got != old).sum())
    if case == "path":
        assert sweeps < 0  # the fallback ran
    elif case == "dense":
        assert 0 < sweeps <= 32  # settled by the sweeps (a near-critical sparse graph may need the fallback)


def _warm_case(kind, rng):
    """(n, symmetric scipy CSR with some zero-weight entries, vmask) for the warm labelling."""
    import scipy.sparse as ssp
    if kind == "er":
        n = 30_000
        m = 5 * n
        u, v = rng.integers(0, n, m), rng.integers(0, n, m)
    elif kind == "path":  # one long chain: far deeper than the search's levels and sweeps
        n = 20_000
        u, v = np.arange(n - 1), np.arange(1, n)
    else:  # many small components
        n = 20_000
        u = rng.integers(0, n, n // 2)
        v = np.minimum(n - 1, u + rng.integers(1, 4, n // 2))
    ok = u != v
    u, v = u[ok], v[ok]
    w = np.where(rng.random(u.size) < 0.1, 0.0, 1.0).astype(np.float32)  # inert entries
    A = ssp.coo_matrix((np.concatenate([w, w]), (np.concatenate([u, v]), np.concatenate([v, u]))), shape=(n, n))
    A = A.tocsr()
    A.sum_duplicates()
    A.data = np.where(A.data > 0, 1.0, 0.0).astype(np.float32)
    return n, A, (rng.random(n) < 0.95).astype(np.uint8)


@pytest.mark.parametrize("kind", ["er", "path", "pieces"])
def test_warm_labelling_matches_union_find_over_calls(kind):
    """dlp_cc_graph_warm equals dlp_cc_graph (no sink) call after call while the graph changes and
    the seed the workspace carries goes stale: edges deleted around it, its vertex cut off, new
    edges merging components."""
    from dynlplus_b200 import _lib
    from dynlplus_b200.backend import code, ptr, stream
    rng = np.random.default_rng({"er": 1, "path": 2, "pieces": 3}[kind])
    n, A, vm = _warm_case(kind, rng)
    ws = torch.zeros(int(_lib.lib().dlp_cc_graph_warm_workspace_bytes(n)), dtype=torch.uint8, device="cuda")
    wsg = torch.zeros(int(_lib.lib().dlp_cc_graph_workspace_bytes()), dtype=torch.uint8, device="cuda")
    vmask = T(vm)
    for call in range(6):
        G = CSR.from_scipy(A)
        got = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        want = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        err = torch.zeros(2, dtype=torch.int32, device="cuda")
        _lib.call("dlp_cc_graph_warm", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.data), code(G.data),
                  ptr(vmask), ptr(got), ptr(err[0:1]), ptr(ws), ws.numel(), stream())
        _lib.call("dlp_cc_graph", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.data), code(G.data),
                  ptr(vmask), None, ptr(want), ptr(err[1:2]), ptr(wsg), wsg.numel(), stream())
        assert int(err.sum()) == 0
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy(), err_msg=f"{kind} call {call}")
        # the next graph: cut the seed the workspace now holds off from everything, then flip
        # the weights of random entries (deletions and revivals, kept symmetric)
        seed = int(ws[:4].view(torch.int32).item())
        A = A.tolil()
        if 0 <= seed < n:
            A[seed, :] = 0
            A[:, seed] = 0
        A = A.tocsr()
        A.eliminate_zeros()
        k = rng.integers(0, A.nnz, max(A.nnz // 20, 1))
        r = np.repeat(np.arange(n), np.diff(A.indptr))[k]
        c = A.indices[k]
        A = A.tolil()
        for a, b in zip(r, c):
            A[a, b] = A[b, a] = 0.0 if rng.random() < 0.7 else 1.0
        u = rng.integers(0, n, 200)
        v = rng.integers(0, n, 200)
        for a, b in zip(u, v):
            if a != b:
                A[a, b] = A[b, a] = 1.0
        A = A.tocsr()

"""Workload generators, the edge-update stream and the CPU baseline solver (host logic, no GPU).

The bench's inputs come from these generators: a symmetric, loop-free CSR with set semantics (each
undirected pair stored once per direction, unit weights stay 1.0), labels equal to the block id for
the planted partition, and update batches whose inserts are current non-edges and whose deletes are
current edges. The CPU baseline (`oracle.edge_cpu`) must keep every batch's scores at the relative
residual target on the rebuilt system.
"""
import numpy as np
import pytest
import torch

from dynlplus_b200 import graphs
from oracle import ref_np as O
from oracle.edge_cpu import EdgeSolverCPU, static_solve


def canonical(A):
    """Checks the CSR invariants every kernel relies on and returns the matrix as SciPy fp64."""
    n = A.shape[0]
    ip = A.indptr.numpy().astype(np.int64)
    ix = A.indices.numpy().astype(np.int64)
    assert ip[0] == 0 and ip[-1] == ix.shape[0] and (np.diff(ip) >= 0).all()
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ip))
    assert (rows != ix).all(), "self-loop stored"
    assert (np.diff(rows * n + ix) > 0).all(), "columns unsorted or duplicated within a row"
    S = A.to_scipy().astype(np.float64)
    assert abs(S - S.T).max() == 0 if S.nnz else True, "not symmetric"
    return S


@pytest.mark.parametrize("weights", ["unit", "lognormal"])
def test_planted_partition_shape_and_labels(weights):
    n, blocks, d_in, d_x = 6000, 4, 9.0, 3.0
    ds = graphs.planted_partition(n, blocks, d_in, d_x, weights=weights, seed=3, device="cpu")
    S = canonical(ds.A)
    y = ds.y.numpy()
    np.testing.assert_array_equal(y, np.arange(n) // (n // blocks))
    assert ds.K == blocks
    coo = S.tocoo()
    same = y[coo.row] == y[coo.col]
    # expected degree d_in + d_x; set semantics loses only the rare repeated pair at this size
    assert 0.99 * (d_in + d_x) <= S.nnz / n <= d_in + d_x
    assert abs(same.mean() - d_in / (d_in + d_x)) < 0.01
    if weights == "unit":
        assert (coo.data == 1.0).all()  # duplicates are kept once, never summed
    else:
        assert (coo.data > 0).all()
        lw = np.log(coo.data)
        assert abs(lw.mean()) < 0.02 and abs(lw.std() - 0.5) < 0.02
    again = graphs.planted_partition(n, blocks, d_in, d_x, weights=weights, seed=3, device="cpu")
    assert abs(again.A.to_scipy() - ds.A.to_scipy()).max() == 0
    other = graphs.planted_partition(n, blocks, d_in, d_x, weights=weights, seed=4, device="cpu")
    assert abs(other.A.to_scipy().astype(np.float64) - S).max() > 0


def test_er_graph_degree_and_labels():
    n, deg, K = 5000, 10.0, 8
    ds = graphs.er_graph(n, deg, K, seed=1, device="cpu")
    S = canonical(ds.A)
    assert 0.99 * deg <= S.nnz / n <= deg
    y = ds.y.numpy()
    assert y.min() >= 0 and y.max() < K and np.bincount(y, minlength=K).min() > 0.8 * n / K
    assert (S.data == 1.0).all()
    np.testing.assert_array_equal(ds.order.numpy(), np.arange(n))


def test_label_mask_count_and_seed():
    m = graphs.label_mask(10_000, 0.005, seed=2, device="cpu").numpy()
    assert m.dtype == bool and m.sum() == 50
    np.testing.assert_array_equal(m, graphs.label_mask(10_000, 0.005, seed=2, device="cpu").numpy())
    assert (m != graphs.label_mask(10_000, 0.005, seed=3, device="cpu").numpy()).any()


def test_set_semantics_versus_coalesce():
    # pairs (0,1,w=2) and (1,0,w=5) name the same undirected edge; (2,2) is a self-loop
    u, v, w = np.array([0, 1, 2, 1]), np.array([1, 0, 2, 2]), np.array([2.0, 5.0, 1.0, 3.0])
    Sset = graphs.symmetric_set(u, v, w, 3, "float64", device="cpu").to_scipy().toarray()
    np.testing.assert_array_equal(Sset, [[0, 2, 0], [2, 0, 3], [0, 3, 0]])  # the first weight given
    Ssum = graphs.symmetric_from_pairs(u, v, w, 3, "float64", device="cpu").to_scipy().toarray()
    np.testing.assert_array_equal(Ssum, [[0, 7, 0], [7, 0, 3], [0, 3, 0]])  # duplicates summed
    np.testing.assert_array_equal(Ssum, O.symmetric_from_pairs(u, v, w, 3, np.float64).toarray())


def test_symmetric_from_pairs_matches_the_oracle_on_random_pairs():
    rs = np.random.RandomState(5)
    n, m = 400, 3000
    u, v, w = rs.randint(0, n, m), rs.randint(0, n, m), rs.rand(m)
    G = graphs.symmetric_from_pairs(u, v, w, n, "float64", device="cpu").to_scipy()
    R = O.symmetric_from_pairs(u, v, w, n, np.float64)
    np.testing.assert_array_equal(G.indptr, R.indptr)
    np.testing.assert_array_equal(G.indices, R.indices)
    np.testing.assert_allclose(G.data, R.data, rtol=1e-15)


def test_row_positions_and_csr_rows():
    ds = graphs.er_graph(300, 4.0, 3, seed=9, device="cpu")
    A = ds.A
    ip = A.indptr.numpy().astype(np.int64)
    np.testing.assert_array_equal(graphs.csr_rows(A).numpy(), O.csr_rows(A.to_scipy()))
    rows = np.array([5, 0, 5, 299, 17, 17, 42])  # repeats kept, in the order given
    pos, seg = graphs.row_positions(A.indptr, torch.as_tensor(rows))
    want_pos = np.concatenate([np.arange(ip[r], ip[r + 1]) for r in rows])
    want_seg = np.concatenate([np.full(ip[r + 1] - ip[r], i) for i, r in enumerate(rows)])
    np.testing.assert_array_equal(pos.numpy(), want_pos)
    np.testing.assert_array_equal(seg.numpy(), want_seg)
    pos, seg = graphs.row_positions(A.indptr, torch.zeros(0, dtype=torch.int64))
    assert pos.numel() == 0 and seg.numel() == 0


@pytest.mark.parametrize("ins_frac,weights", [(0.5, "unit"), (0.3, "lognormal"), (1.0, "unit"), (0.0, "unit")])
def test_edge_updates_insert_non_edges_and_delete_edges(ins_frac, weights):
    ds = graphs.er_graph(3000, 6.0, 4, seed=11, device="cpu")
    n = ds.n
    S = ds.A.to_scipy().tocoo()
    live = set((S.row[S.row < S.col].astype(np.int64) * n + S.col[S.row < S.col]).tolist())
    up = graphs.EdgeUpdates(ds.A, seed=11, weights=weights)
    A = ds.A.to_scipy().astype(np.float64)
    for size in (400, 1, 999, 0):
        b = up.next(size, ins_frac=ins_frac)
        ni, nd = int(round(size * ins_frac)), size - int(round(size * ins_frac))
        assert b["ins_u"].shape[0] == ni and b["del_u"].shape[0] == nd
        assert (b["ins_u"] < b["ins_v"]).all() and (b["del_u"] < b["del_v"]).all()
        ik = b["ins_u"].astype(np.int64) * n + b["ins_v"]
        dk = b["del_u"].astype(np.int64) * n + b["del_v"]
        assert np.unique(ik).shape[0] == ni and np.unique(dk).shape[0] == nd
        assert not (set(ik.tolist()) & live), "an insert names a present edge"
        assert set(dk.tolist()) <= live, "a delete names an absent edge"
        if weights == "unit":
            assert (b["ins_w"] == 1.0).all()
        else:
            assert (b["ins_w"] > 0).all()
        live = (live - set(dk.tolist())) | set(ik.tolist())
        np.testing.assert_array_equal(up.keys, np.array(sorted(live), dtype=np.int64))
        A = O.apply_edges(A, b["ins_u"], b["ins_v"], b["ins_w"].astype(np.float64), b["del_u"], b["del_v"])
        C = A.tocoo()
        up_keys = np.sort(C.row[C.row < C.col].astype(np.int64) * n + C.col[C.row < C.col])
        np.testing.assert_array_equal(up_keys, up.keys)  # the stream's edge set is the patched graph's


def test_cpu_baseline_holds_the_target_across_batches():
    n, K, target = 2000, 4, 1e-6
    ds = graphs.planted_partition(n, K, 4.0, 1.5, seed=6, device="cpu")  # sparse: splits and regrounding
    A = ds.A.to_scipy().astype(np.float64)
    y = ds.y.numpy()
    lab = graphs.label_mask(n, 0.03, seed=6, device="cpu").numpy()
    Z0 = static_solve(A, y, lab, K, target)
    solver = EdgeSolverCPU(A, y, lab, K, Z0, target)
    up = graphs.EdgeUpdates(ds.A, seed=6)
    for _ in range(4):
        S = solver.step(up.next(300))
        U, C = S["U"], solver.C
        rhs = np.concatenate([S["rhs"], S["diag"][:, None]], axis=1)
        R = rhs - O.apply_A(S["W"], S["diag"], solver.Z[U])
        rel = np.sqrt((R * R).sum(axis=0)) / np.sqrt((rhs * rhs).sum(axis=0))
        assert rel[:C].max() <= target and rel[C] <= 1e3 * target  # the h column is solved loosely
        out = np.ones(n, dtype=bool)
        out[U] = False
        assert (solver.Z[out, :C] == 0).all() and (solver.Z[out, C] == 1).all()  # inert rows

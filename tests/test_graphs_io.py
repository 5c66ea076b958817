"""Edge-list npz format (dynlp/graphs.py:176-204) and the reference-identical generators (CPU)."""
import os

import numpy as np
import pytest

from dynlplus_b200 import graphs
from oracle import ref_np as O


def test_from_npz_matches_coalesced_pairs_and_round_trips(tmp_path):
    rs = np.random.RandomState(0)
    n = 60
    src, dst, w, y = rs.randint(0, n, 300), rs.randint(0, n, 300), rs.rand(300), rs.randint(0, 4, n)
    p = str(tmp_path / "g.npz")
    np.savez(p, src=src, dst=dst, w=w, y=y)
    ds = graphs.from_npz(p, dtype="float64", device="cpu")
    A = O.symmetric_from_pairs(src, dst, w, n, np.float64)
    G = ds.A.to_scipy()
    assert ds.K == 4 and ds.name == "g.npz"
    np.testing.assert_array_equal(G.indptr, A.indptr)
    np.testing.assert_array_equal(G.indices, A.indices)
    np.testing.assert_allclose(G.data, A.data, rtol=1e-15)
    np.testing.assert_array_equal(ds.order.numpy(), np.random.RandomState(1).permutation(n))  # the default draw
    q = str(tmp_path / "h.npz")
    graphs.save_npz(ds, q)
    ds2 = graphs.from_npz(q, dtype="float64", device="cpu")
    assert abs(ds2.A.to_scipy() - G).max() <= 1e-15
    np.testing.assert_array_equal(ds2.order.numpy(), ds.order.numpy())
    np.testing.assert_array_equal(ds2.y.numpy(), y)
    assert graphs.load(q, dtype="float64", device="cpu").n == n


def test_unweighted_npz_gets_unit_weights(tmp_path):
    p = str(tmp_path / "u.npz")
    np.savez(p, src=np.array([0, 1, 2]), dst=np.array([1, 2, 0]), y=np.array([0, 1, 1]))
    ds = graphs.from_npz(p, device="cpu")
    assert ds.A.nnz == 6 and float(ds.A.data.min()) == 1.0 and ds.K == 2


SYNTH_CASES = [dict(n=1200, K=2, k=6, subs=2, seed=7, dtype="float64"),
               dict(n=3000, K=3, k=5, dim=16, subs=5, seed=1, dtype="float32")]


def _golden_csr(g, prefix):
    return g[f"{prefix}_indptr"], g[f"{prefix}_indices"], g[f"{prefix}_data"]


def _same_graph(A, ref, rtol):
    G = A.to_scipy()
    ip, ix, d = ref
    np.testing.assert_array_equal(G.indptr, ip)
    np.testing.assert_array_equal(G.indices, ix)
    np.testing.assert_allclose(G.data, d, rtol=rtol)


def test_synth_matches_reference(golden):
    """dynlp/graphs.py:124-143 run by the reference (tests/golden/graphs.npz): same neighbour sets,
    labels and arrival order; similarities to fp32 rounding (a different GEMM)."""
    g = golden("graphs.npz")
    for i, kw in enumerate(SYNTH_CASES):
        ds = graphs.synth(**kw, device="cpu")
        _same_graph(ds.A, _golden_csr(g, f"s{i}_A"), 1e-5)
        np.testing.assert_array_equal(ds.y.numpy(), g[f"s{i}_y"])
        np.testing.assert_array_equal(ds.order.numpy(), g[f"s{i}_order"])
        assert ds.K == int(g[f"s{i}_K"]) and ds.name == str(g[f"s{i}_name"])


def test_knn_graph_matches_reference(golden):
    """dynlp/graphs.py:78-93: pairs found from both sides kept once (the first occurrence's
    similarity), clamped at 1e-3."""
    g = golden("graphs.npz")
    A = graphs.knn_graph(g["knn_X"], 4, "float32", device="cpu")
    _same_graph(A, _golden_csr(g, "knn_A"), 1e-5)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0 and (S.data >= 1e-3).all() and (S.diagonal() == 0).all()


def test_synth_cache_and_load(tmp_path, monkeypatch):
    """build_cached / load("synthN") (dynlp/graphs.py:187-214): an existing cache file is read as is
    (no order stored, so loading draws the reference's permutation), a missing one is built from
    synth(K=N), and names other than synthN are refused."""
    small = graphs.synth(n=800, K=3, k=5, seed=2, device="cpu")
    graphs.save_npz(small, str(tmp_path / "synth3.npz"), with_order=False)
    ds = graphs.load("synth3", data_dir=str(tmp_path), dtype="float32", device="cpu")
    assert ds.name == "synth3" and ds.K == 3 and ds.n == 800
    assert abs(ds.A.to_scipy() - small.A.to_scipy()).max() < 1e-6
    np.testing.assert_array_equal(ds.order.numpy(), np.random.RandomState(1).permutation(800))
    made = []
    monkeypatch.setattr(graphs, "synth", lambda K, device=None: made.append(K) or small)
    path = graphs.build_cached("synth4", data_dir=str(tmp_path / "new"))
    assert made == [4] and os.path.exists(path)
    with pytest.raises(ValueError):
        graphs.build_cached("imdb", data_dir=str(tmp_path))

"""Edge-list npz format (dynlp/graphs.py:176-204) and the reference-identical generators (CPU)."""
import numpy as np

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

"""The oracle against the reference's own property tests (tests/test_dynlp.py), on the host: its block
PCG matches a direct solve, the absorption bound holds for any iterate, joint class columns give the
binary column, an fp64 correction certifies the path graph where the fp32 solve alone cannot, its
AMG V-cycle is a symmetric positive definite operator, its FH components cut a bridge and merge a
weak chain, and the synth kNN graph keeps its k neighbours. These pin the checker itself; the GPU
tests compare the device path with it."""
import numpy as np
import pytest
import scipy.sparse as ssp

from conftest import direct_solve
from dynlplus_b200 import graphs
from oracle import ref_np as O


def batch_systems(n, K, deg, seed, label_frac, init_frac, n_batches):
    """The oracle's systems of a vertex-arrival stream over an SBM graph (dynlp/stream.py:84-177)."""
    ds = graphs.sbm(n, K=K, deg=deg, seed=seed, dtype="float64", device="cpu")
    A, y = ds.A.to_scipy().astype(np.float64), ds.y.numpy()
    lab, _, _, sched = O.stream_schedule(y, K, ds.order.numpy(), label_frac=label_frac, init_frac=init_frac,
                                         n_batches=n_batches)
    active = np.zeros(n, dtype=bool)
    for ins, dele in sched:
        active[ins], active[dele] = True, False
        yield O.build_system(A, y, K, active.copy(), lab)


def dense(S):
    return (ssp.diags(S["diag"]) - S["W"]).tocsr()


def cols(X, n):
    return np.asarray(X).reshape(n, -1)


@pytest.mark.parametrize("K", [2, 4])
def test_pcg_matches_direct_solve(K):
    """tests/test_dynlp.py:97-106 (the fp64 Reference solve) on the oracle's PCG."""
    for S in batch_systems(2000, K, 6, 2, 0.02, 0.3, 2):
        A, rhs = dense(S), S["rhs"]
        Z, it = O.pcg(S["W"], S["diag"], np.zeros_like(rhs), rhs, [1e-12] * rhs.shape[1])
        assert it > 0
        assert np.abs(Z - cols(direct_solve(A, rhs), A.shape[0])).max() < 1e-7


def test_certificate_bound_is_valid_for_any_iterate():
    """tests/test_dynlp.py:136-145: |F - F*| <= rho h elementwise, rho = max |rhs - A F| / diag."""
    S = next(batch_systems(1500, 2, 6, 5, 0.03, 0.5, 0))
    A, rhs, d = dense(S), S["rhs"], S["diag"]
    Fd, h = cols(direct_solve(A, rhs), A.shape[0]), cols(direct_solve(A, d), A.shape[0])
    rs = np.random.RandomState(0)
    for scale in (1e-1, 1e-3):
        F = Fd + scale * rs.standard_normal(Fd.shape)
        rho = float((np.abs(rhs - A @ F) / d[:, None]).max())
        assert (np.abs(F - Fd) <= rho * h + 1e-12).all()


def test_multiclass_columns_consistent_with_binary():
    """tests/test_dynlp.py:148-156: both class columns (rhs = B) solved jointly give the binary
    column (rhs = class 1), and the two sum to one."""
    S = next(batch_systems(2000, 2, 6, 6, 0.03, 0.4, 0))
    W, d = S["W"], S["diag"]
    B = S["B"]
    Z2, _ = O.pcg(W, d, np.zeros_like(B), B.copy(), [1e-12, 1e-12])
    Z1, _ = O.pcg(W, d, np.zeros_like(S["rhs"]), S["rhs"].copy(), [1e-12])
    np.testing.assert_allclose(Z2[:, 1], Z1[:, 0], atol=1e-8)
    np.testing.assert_allclose(Z2.sum(axis=1), 1.0, atol=1e-8)


def test_path_graph_needs_the_fp64_correction():
    """tests/test_dynlp.py:225-243: a path labelled only at its ends has h ~ 9e4, so the fp32 solve
    alone cannot certify 1e-3 (rho h stays above it) while one fp64 correction of its residual
    (dynlp/solvers.py:322-337) does, with the error inside the certificate."""
    n = 600
    u = np.arange(n - 1)
    A0 = O.symmetric_from_pairs(u, u + 1, np.ones(n - 1), n, np.float64)
    y = (np.arange(n) >= n // 2).astype(np.int32)
    lab = np.zeros(n, dtype=bool)
    lab[[0, n - 1]] = True
    S = O.build_system(A0, y, 2, np.ones(n, dtype=bool), lab)
    A, rhs, d = dense(S), S["rhs"], S["diag"]
    Fd, h = cols(direct_solve(A, rhs), A.shape[0]), cols(direct_solve(A, d), A.shape[0])
    assert h.max() > 1e4
    W32, d32 = S["W"].astype(np.float32), d.astype(np.float32)
    Z32, _ = O.pcg(W32, d32, np.zeros(rhs.shape, np.float32), rhs.astype(np.float32), [1e-7])
    Z = Z32.astype(np.float64)

    def cert(Z):
        return float((np.abs(rhs - A @ Z) / d[:, None]).max()) * float(h.max())

    assert cert(Z) > 1e-3
    R = rhs - A @ Z
    D, _ = O.pcg(S["W"], d, np.zeros_like(R), R, [1e-3 / (1.25 * h.max())])
    Z = Z + D
    assert cert(Z) <= 1e-3
    assert np.abs(Z - Fd).max() <= cert(Z) * 1.05 + 1e-9


def test_amg_vcycle_is_symmetric_positive_definite():
    """tests/test_dynlp.py:159-166 on a second graph family, an SBM system large enough for two
    levels at the default coarsest size: the V-cycle applied to the identity is a symmetric matrix
    with positive eigenvalues."""
    S = next(batch_systems(4000, 3, 8, 7, 0.02, 0.9, 0))
    n = S["W"].shape[0]
    amg = O.AMGOracle(S["W"], S["s"])
    assert len(amg.sizes) >= 2 and amg.sizes[0] > amg.sizes[-1]
    M = amg(np.eye(n))
    assert np.abs(M - M.T).max() <= 1e-10 * np.abs(M).max()
    assert np.linalg.eigvalsh((M + M.T) / 2).min() > 0


def test_amg_vcycle_spd_on_the_reference_graph():
    """tests/test_dynlp.py:158-165 exactly: the synth kNN graph (n=1200, K=2, k=6, 2 sub-clusters,
    seed 7), the whole graph active with 2% labels, AMG with max_coarse=50 (two levels or more)."""
    ds = graphs.synth(1200, K=2, k=6, subs=2, seed=7, dtype="float64", device="cpu")
    A, y = ds.A.to_scipy().astype(np.float64), ds.y.numpy()
    lab, _, _, sched = O.stream_schedule(y, 2, ds.order.numpy(), label_frac=0.02, init_frac=1.0, n_batches=0)
    active = np.zeros(A.shape[0], dtype=bool)
    active[sched[0][0]] = True
    S = O.build_system(A, y, 2, active, lab)
    amg = O.AMGOracle(S["W"], S["s"], max_coarse=50)
    assert len(amg.levels) >= 2
    n = S["W"].shape[0]
    M = amg(np.eye(n))
    np.testing.assert_allclose(M, M.T, atol=1e-10)
    assert np.linalg.eigvalsh((M + M.T) / 2).min() > 0


def _same_partition(a, b):
    a, b = [int(x) for x in a], [int(x) for x in b]
    return len(set(zip(a, b))) == len(set(a)) == len(set(b))


def _components(edges, m, tau, ground=None):
    """new_components on an explicit undirected edge list, every vertex new (as the reference's
    helper in tests/test_dynlp.py:49-53)."""
    a, b, w = (np.asarray(x) for x in zip(*edges))
    g = np.ones(m) if ground is None else np.asarray(ground, dtype=np.float64)
    return O.new_components(m, np.concatenate([a, b]), np.concatenate([b, a]),
                            np.concatenate([w, w]).astype(np.float32), tau, 1.0, g)


def test_adaptive_components_cut_a_bridge_that_tau_chains():
    """tests/test_dynlp.py:56-62: two tight cliques joined by an edge above the global mean but weak
    relative to both are one tau component and two FH components."""
    edges = [(a + o, b + o, 0.95 + 0.01 * ((a + b) % 3)) for o in (0, 6) for a in range(6) for b in range(a + 1, 6)]
    edges.append((5, 6, 0.8))
    comps = _components(edges, 12, tau=0.5)
    assert comps["tau"][1] == 1
    assert comps["fh"][1] == 2 and _same_partition(comps["fh"][0], [0] * 6 + [1] * 6)


def test_adaptive_components_merge_a_sparse_cluster():
    """tests/test_dynlp.py:65-71: a weak chain (every edge below tau) stays singletons under tau but
    is one FH component, a component without labelled contact joining its strongest neighbour."""
    edges = [(i, i + 1, 0.3 + 0.02 * (i % 3)) for i in range(7)]
    comps = _components(edges, 8, tau=0.5, ground=[1, 0, 0, 0, 0, 0, 0, 0])
    assert comps["tau"][1] == 8
    assert comps["fh"][1] == 1


def test_synth_graph():
    """tests/test_dynlp.py:173-177 on graphs.synth: symmetric, similarities in (0, 1], and every
    vertex keeps its k = 5 neighbours."""
    ds = graphs.synth(3000, K=10, seed=1, device="cpu")
    S = ds.A.to_scipy()
    assert ds.n == 3000 and ds.K == 10 and abs(S - S.T).max() == 0
    assert S.data.min() > 0 and S.data.max() <= 1
    assert np.diff(S.indptr).min() >= 5

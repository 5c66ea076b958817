"""Aggregation AMG on the device against the reference's outputs (GPU)."""
import numpy as np
import pytest
import torch

from conftest import direct_solve, golden_csr, load_golden
from dynlplus_b200 import amg, graphs, solvers, stream
from dynlplus_b200.backend import CSR
from oracle import ref_np as O

pytestmark = pytest.mark.gpu


def test_handshake_and_coarsen_match_reference():
    g = load_golden("amg.npz")
    W = CSR.from_scipy(golden_csr(g, "W"), dtype=torch.float32)
    agg, nc = amg.handshake(W, 3)
    np.testing.assert_array_equal(agg.cpu().numpy(), g["match_agg"])
    assert nc == int(g["match_nc"])
    Wc, sc = amg.coarsen(W, torch.as_tensor(g["s"]).cuda(), agg, nc)
    Wg = golden_csr(g, "match_Wc")
    got = Wc.to_scipy()
    np.testing.assert_array_equal(got.indptr, Wg.indptr)
    np.testing.assert_array_equal(got.indices, Wg.indices)
    np.testing.assert_allclose(got.data, Wg.data, rtol=1e-6)
    np.testing.assert_allclose(sc.cpu().numpy(), g["match_sc"], rtol=1e-6)  # reference: fp32 sums


def test_hierarchy_and_vcycle_match_reference():
    g = load_golden("amg.npz")
    W = CSR.from_scipy(golden_csr(g, "W"), dtype=torch.float32)
    M = amg.AMG(W, torch.as_tensor(g["s"]).cuda(), max_coarse=50)
    assert M.sizes == list(g["sizes"])
    for i, L in enumerate(M.levels):
        np.testing.assert_array_equal(L.agg.cpu().numpy(), g[f"L{i}_agg"])
    R = torch.as_tensor(g["R"]).cuda()
    Y = M(R).double().cpu().numpy()
    np.testing.assert_allclose(Y, g["MR"], rtol=1e-4, atol=1e-5 * abs(g["MR"]).max())


def test_amg_is_symmetric_positive_definite():
    """tests/test_dynlp.py:159-166: the V-cycle operator is symmetric with positive eigenvalues."""
    ds = graphs.sbm(1200, K=2, deg=6, seed=7, dtype="float64")
    lab = graphs.label_mask(1200, 0.02, seed=7)
    S = stream.build_system(ds, torch.ones(1200, dtype=torch.bool, device="cuda"), lab, dtype="float64")
    M = amg.AMG(S.W, S.s, max_coarse=50)
    assert len(M.levels) >= 2
    Mi = M(torch.eye(S.n_u, dtype=torch.float64, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(Mi, Mi.T, atol=1e-6)  # fp32 weights on the levels: 1e-6 instead of 1e-10
    assert np.linalg.eigvalsh((Mi + Mi.T) / 2).min() > 0


@pytest.mark.parametrize("K", [2, 3])
def test_dynlp_plus_amg_certificate(K):
    ds = graphs.sbm(3000, K=K, deg=8, seed=3, dtype="float32")
    lab = graphs.label_mask(3000, 0.02, seed=3)
    S = stream.build_system(ds, torch.ones(3000, dtype=torch.bool, device="cuda"), lab, dtype="float32")
    solver = solvers.DynLPPlus(3000, K, "float32", method="amg", tol=1e-3)
    st = solver.solve(S)
    S64 = S.astype(torch.float64)
    import scipy.sparse as ssp
    import scipy.sparse.linalg as sla
    A = ssp.diags(S64.diag.cpu().numpy()) - S64.W.to_scipy().astype(np.float64)
    Fd = direct_solve(A, S64.rhs.cpu().numpy())
    Fd = Fd.reshape(-1, 1) if Fd.ndim == 1 else Fd
    err = np.abs(solver.scores(S).cpu().numpy() - Fd).max()
    assert st.cert <= 1e-3 * 1.0001 and err <= st.cert * 1.05 + 1e-6, (err, st.cert, st.iters)
    assert st.iters < 60


@pytest.mark.parametrize("method", ["pcg", "amg"])
def test_bf16_sweeps_with_fp64_refinement_reach_1e8(method):
    """Config 3's precision scheme: SpMM on bf16 weights/scores (fp32 accumulation) inside fp32 PCG,
    fp64 residual refinement to rel-res 1e-8; the result is checked against a direct fp64 solve."""
    ds = graphs.planted_partition(20_000, 8, 18.0, 6.0, weights="lognormal", seed=5)
    lab = graphs.label_mask(20_000, 0.01, seed=5)
    S = stream.build_system(ds, torch.ones(20_000, dtype=torch.bool, device="cuda"), lab, dtype="float32")
    solver = solvers.DynLPPlus(20_000, 8, "float32", method=method, tol=1e-3, target_relres=1e-8, lowp=True)
    st = solver.solve(S)
    S64 = S.astype(torch.float64)
    A = S64.W.to_scipy().astype(np.float64)
    F = solver.scores(S).cpu().numpy()
    rel = O.relres(A, S64.diag.cpu().numpy(), F, S64.rhs.cpu().numpy())
    assert rel <= 1e-8 and st.relres <= 1e-8, (rel, st.relres)
    import scipy.sparse as ssp
    import scipy.sparse.linalg as sla
    Fd = direct_solve(ssp.diags(S64.diag.cpu().numpy()) - A, S64.rhs.cpu().numpy())
    assert np.abs(F - Fd).max() <= max(st.cert, 1e-6)


def _unit_sbm_system(n, seed, dtype="float64"):
    """An SBM with unit weights: fp32 level weights and their coarse sums are exact, so the
    device hierarchy equals the oracle's fp64 one entry for entry."""
    ds = graphs.planted_partition(n, 4, 9.0, 3.0, seed=seed)
    lab = graphs.label_mask(n, 0.01, seed=seed)
    return stream.build_system(ds, torch.ones(n, dtype=torch.bool, device="cuda"), lab, dtype=dtype)


def test_device_amg_pcg_matches_oracle():
    """dlp_pcg_amg (the loop on the device) against the oracle's pcg with its AMG (dynlp/solvers.py:66-97
    with M = amg.AMG) in fp64: the same iteration count and the same iterate."""
    S = _unit_sbm_system(30_000, 8)
    M = amg.AMG(S.W, S.s, max_coarse=200)
    C = S.rhs.shape[1]
    eps = [1e-7] * C
    Z = torch.zeros((S.n_u, C), dtype=torch.float64, device="cuda")
    st = solvers.Stats()
    solvers.pcg(S, Z, S.rhs, eps, M, 10_000, st)
    W = S.W.to_scipy().astype(np.float64)
    Mo = O.AMGOracle(W, S.s.cpu().numpy(), max_coarse=200)
    assert Mo.sizes == M.sizes
    Zo, it = O.pcg(W, S.diag.cpu().numpy(), np.zeros((S.n_u, C)), S.rhs.cpu().numpy(), eps, M=Mo)
    assert st.iters == it, (st.iters, it)
    np.testing.assert_allclose(Z.cpu().numpy(), Zo, rtol=1e-9, atol=1e-12 * np.abs(Zo).max())


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_device_amg_pcg_graph_equals_host_loop_and_caps(dt):
    """The device-side loop (CUDA graph WHILE node) and the host-driven launches give bit-identical
    iterates; a cap of 3 iterations stops at 3 with DLP_ERR_CAP handled as the reference's cap."""
    S = _unit_sbm_system(20_000, 9, "float32" if dt == torch.float32 else "float64")
    M = amg.AMG(S.W, S.s, max_coarse=200)
    C = S.rhs.shape[1]
    eps = [1e-5] * C
    out = []
    for graph in (True, False):
        Z = torch.zeros((S.n_u, C), dtype=dt, device="cuda")
        st = solvers.Stats()
        solvers.pcg(S, Z, S.rhs, eps, M, 10_000, st, use_graph=graph, target_relres=1e-6)
        out.append((Z, st.iters, st.relres))
    assert out[0][1] == out[1][1] and torch.equal(out[0][0], out[1][0])
    # fp32 sweeps (the V-cycle included) stop at their own floor, 3e-6 to 7e-5 on this system; the
    # solvers reach the target through the fp64 refinement around them
    assert out[0][2] <= (1e-4 if dt == torch.float32 else 1e-6)
    Z = torch.zeros((S.n_u, C), dtype=dt, device="cuda")
    st = solvers.Stats()
    solvers.pcg(S, Z, S.rhs, eps, M, 3, st)
    assert st.iters == 3


def test_vcycle_one_call_matches_oracle_cycle():
    """dlp_amg_vcycle (every level in one library call) against the oracle's V-cycle, fp64."""
    S = _unit_sbm_system(30_000, 10)
    M = amg.AMG(S.W, S.s, max_coarse=200)
    W = S.W.to_scipy().astype(np.float64)
    Mo = O.AMGOracle(W, S.s.cpu().numpy(), max_coarse=200)
    R = torch.as_tensor(np.random.RandomState(0).randn(S.n_u, 5)).cuda()
    np.testing.assert_allclose(M(R).cpu().numpy(), Mo(R.cpu().numpy()), rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("n", [1, 7, 300, 1500])
def test_dense_spd_inverse_matches_numpy(n):
    """The coarse operator's inverse (dlp_dense_spd_inverse) against NumPy's, on a grounded-Laplacian
    shaped SPD matrix."""
    from dynlplus_b200 import _lib
    from dynlplus_b200.backend import ptr, stream, workspace
    rs = np.random.RandomState(n)
    W = rs.rand(n, n) * (rs.rand(n, n) < 0.05)
    W = np.triu(W, 1)
    W = W + W.T
    A = np.diag(W.sum(1) + rs.rand(n) + 0.1) - W
    At = torch.as_tensor(A).cuda().contiguous()
    ws = workspace("inv_test").get(_lib.lib().dlp_dense_spd_inverse_workspace_bytes(n))
    _lib.call("dlp_dense_spd_inverse", n, ptr(At), ptr(ws), ws.numel(), stream())
    want = np.linalg.inv(A)
    np.testing.assert_allclose(At.cpu().numpy(), want, rtol=0, atol=1e-10 * np.abs(want).max())


@pytest.mark.parametrize("m,nc", [(1, 3), (2047, 40), (300_001, 1000), (2_000_003, 250_000)])
def test_radix_sort_of_pairs_is_stable(m, nc):
    """dlp_sort_pairs against torch's stable sort: equal keys keep their order (the values are the
    positions), and the no-entry marker (INT64_MAX) sorts last."""
    from dynlplus_b200 import _lib
    from dynlplus_b200.backend import ptr, stream, workspace
    g = torch.Generator(device="cuda").manual_seed(m)
    key = torch.randint(0, nc * nc, (m,), generator=g, device="cuda", dtype=torch.int64)
    key = key // 7  # many equal keys
    key[torch.rand(m, generator=g, device="cuda") < 0.2] = 2**63 - 1
    val = torch.arange(m, dtype=torch.float64, device="cuda")
    want_k, order = torch.sort(key, stable=True)
    k2, v2 = key.clone(), val.clone()
    kt, vt = torch.empty_like(k2), torch.empty_like(v2)  # spare arrays, alive until the sort has run
    ws = workspace("sort_test").get(_lib.lib().dlp_sort_pairs_workspace_bytes(m))
    _lib.call("dlp_sort_pairs", m, nc * nc, ptr(k2), ptr(v2), ptr(kt), ptr(vt), ptr(ws), ws.numel(), stream())
    torch.cuda.synchronize()
    assert torch.equal(k2, want_k)
    assert torch.equal(v2, val[order])

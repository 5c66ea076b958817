"""Solvers, system assembly and the edge stream against the reference's outputs (golden fixtures)
and the oracle (GPU)."""
import numpy as np
import pytest
import scipy.sparse as ssp
import scipy.sparse.linalg as sla
import torch

from conftest import direct_solve, golden_csr, load_golden
from dynlplus_b200 import graphs, kernels, solvers, stream
from dynlplus_b200.backend import CSR
from oracle import ref_np as O

pytestmark = pytest.mark.gpu


def T(x, dt=None):
    t = torch.as_tensor(np.ascontiguousarray(x))
    return (t.to(dt) if dt is not None else t).cuda()


def golden_system(dt=torch.float64):
    g = load_golden("solvers.npz")
    A = golden_csr(g, "W")
    n = A.shape[0]
    S = stream.System(t=0, U=torch.arange(n, device="cuda"), W=CSR.from_scipy(A, dtype=dt), s=T(g["diag"], dt),
                      diag=T(g["diag"], dt), B=T(g["rhs"], dt), rhs=T(g["rhs"], dt), prior=T(np.full(3, 1 / 3), dt),
                      is_new=torch.zeros(n, dtype=torch.bool, device="cuda"),
                      seed=torch.zeros(n, dtype=torch.bool, device="cuda"), comps={}, K=3, C=3, eta=0.0,
                      n_inserted=0, n_deleted=0, n_active=n)
    return g, A, S


@pytest.mark.parametrize("b", [0, 2])
def test_build_system_matches_reference(b):
    g = load_golden("system.npz")
    p = f"b{b}"
    A = golden_csr(g, f"{p}_A")
    ds = graphs.Dataset("fixture", CSR.from_scipy(A), T(g[f"{p}_y"]), int(g[f"{p}_K"]),
                        torch.arange(A.shape[0], device="cuda"))
    S = stream.build_system(ds, T(g[f"{p}_active"]), T(g[f"{p}_labeled"]), dtype="float64")
    np.testing.assert_array_equal(S.U.cpu().numpy(), g[f"{p}_U"])
    Wg = golden_csr(g, f"{p}_W")
    np.testing.assert_array_equal(S.W.indptr.cpu().numpy(), Wg.indptr)
    np.testing.assert_array_equal(S.W.indices.cpu().numpy(), Wg.indices)
    np.testing.assert_array_equal(S.W.data.cpu().numpy(), Wg.data)
    for k in ("s", "diag", "B", "rhs"):
        np.testing.assert_allclose(getattr(S, k).cpu().numpy(), g[f"{p}_{k}"], rtol=1e-12, err_msg=k)
    assert S.n_ungrounded == int(g[f"{p}_n_ungrounded"])


@pytest.mark.parametrize("graph", [True, False])
def test_fused_pcg_matches_reference(graph):
    """Same iteration counts as the reference's pcg (dynlp/solvers.py:66-97) and the same iterate."""
    g, A, S = golden_system()
    for tag in ("pcg_loose", "pcg_tight"):
        Z = torch.zeros((A.shape[0], 3), dtype=torch.float64, device="cuda")
        st = solvers.Stats()
        solvers.pcg(S, Z, S.rhs, g[f"{tag}_eps"].tolist(), solvers.jacobi_M(S), 10_000, st, use_graph=graph)
        assert st.iters == int(g[f"{tag}_iters"]), (tag, st.iters, int(g[f"{tag}_iters"]))
        np.testing.assert_allclose(Z.cpu().numpy(), g[f"{tag}_Z"], rtol=1e-8, atol=1e-11)


def test_fused_pcg_fp32_and_relres_target():
    g, A, S = golden_system()
    S32 = S.astype(torch.float32)
    Z = solvers.padded_empty(A.shape[0], 3, torch.float32, "cuda")
    Z.zero_()
    st = solvers.Stats()
    solvers.pcg(S32, Z, S32.rhs, None, solvers.jacobi_M(S32), 10_000, st, target_relres=1e-5)
    rel = O.relres(A, g["diag"], Z.double().cpu().numpy(), g["rhs"])
    assert rel <= 1e-5 * 1.01 and st.iters < 200, (rel, st.iters)


def _whole_row_system(C, n=3000, seed=None):
    rs = np.random.RandomState(C if seed is None else seed)
    A = O.symmetric_from_pairs(rs.randint(0, n, 24000), rs.randint(0, n, 24000), rs.rand(24000) + 0.1, n,
                               np.float64)
    diag = np.asarray(A.sum(axis=1)).ravel() + 0.5
    rhs = rs.rand(n, C)
    S = stream.System(t=0, U=torch.arange(n, device="cuda"), W=CSR.from_scipy(A, dtype=torch.float32),
                      s=T(diag, torch.float32), diag=T(diag, torch.float32), B=T(rhs, torch.float32),
                      rhs=T(rhs, torch.float32), prior=T(np.full(C, 1 / C), torch.float32),
                      is_new=torch.zeros(n, dtype=torch.bool, device="cuda"),
                      seed=torch.zeros(n, dtype=torch.bool, device="cuda"), comps={}, K=C, C=C, eta=0.0,
                      n_inserted=0, n_deleted=0, n_active=n)
    return S, A, diag, rhs


@pytest.mark.parametrize("C", [8, 9, 12])
@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("eps", [None, 1e-6])
def test_two_kernel_iteration_follows_three_kernel_one(C, graph, eps):
    """fp32 solves whose rows take the whole-row gather (8 floats in one load, 9-12 in two) run two
    kernels per iteration (the SpMM also
    sums q = sum AP^2/diag and predicts beta; one sweep updates R, Z and the next direction, P and AP
    trading places). Against the three-kernel iteration on the same system: iteration counts within
    one, scores equal to fp32 rounding, and both meet the target on the fp64 residual."""
    S, A, diag, rhs = _whole_row_system(C)
    out = []
    try:
        for two in (True, False):
            solvers.TWO_KERNEL = two
            Z = solvers.padded_empty(A.shape[0], C, torch.float32, "cuda")
            st = solvers.Stats()
            solvers.pcg(S, Z, S.rhs, None if eps is None else [eps] * C, solvers.jacobi_M(S), 10_000, st,
                        target_relres=1e-5, use_graph=graph, zero_start=True)
            out.append((Z.double().cpu().numpy(), st.iters))
    finally:
        solvers.TWO_KERNEL = True
    (Z2, it2), (Z3, it3) = out
    assert abs(it2 - it3) <= 1, (it2, it3)
    Ad = ssp.diags(diag) - A
    for Zx in (Z2, Z3):
        rel = np.linalg.norm(rhs - Ad @ Zx, axis=0) / np.linalg.norm(rhs, axis=0)
        assert rel.max() <= 1e-5 * 1.01, rel.max()
    np.testing.assert_allclose(Z2, Z3, rtol=0, atol=2e-5 * np.abs(Z3).max())


def test_two_kernel_iteration_cap_and_odd_counts():
    """The two-kernel loop stopped at 1, 2, 3 and 5 iterations (P and AP trade places every
    iteration): the iterate equals the three-kernel one at the same count, in the device-side loop
    and in host-driven chunks of 3."""
    C = 9
    S, A, diag, rhs = _whole_row_system(C, seed=3)
    try:
        for cap in (1, 2, 3, 5):
            res = []
            for two in (True, False):
                solvers.TWO_KERNEL = two
                for graph in (True, False):
                    Z = solvers.padded_empty(A.shape[0], C, torch.float32, "cuda")
                    st = solvers.Stats()
                    solvers.pcg(S, Z, S.rhs, None, solvers.jacobi_M(S), cap, st, target_relres=1e-9,
                                use_graph=graph, zero_start=True, check_every=3)
                    assert st.iters == cap
                    res.append(Z.double().cpu().numpy())
            for Zx in res[1:]:
                np.testing.assert_allclose(Zx, res[0], rtol=0, atol=1e-5 * np.abs(res[0]).max())
    finally:
        solvers.TWO_KERNEL = True


@pytest.mark.parametrize("C", [9, 10, 11, 12])
@pytest.mark.parametrize("graph", [True, False])
def test_fused_pcg_fp32_whole_rows(C, graph):
    """fp32 blocks of 9-12 columns take the apply's whole-row path (each gathered and own row of P in
    one 256-bit and one 128-bit load, AP stored whole into its padded rows): the relative-residual
    target holds in fp64 and the solve matches the direct one."""
    rs = np.random.RandomState(C)
    n = 3000
    A = O.symmetric_from_pairs(rs.randint(0, n, 24000), rs.randint(0, n, 24000), rs.rand(24000) + 0.1, n,
                               np.float64)
    diag = np.asarray(A.sum(axis=1)).ravel() + 0.5
    rhs = rs.rand(n, C)
    S = stream.System(t=0, U=torch.arange(n, device="cuda"), W=CSR.from_scipy(A, dtype=torch.float32),
                      s=T(diag, torch.float32), diag=T(diag, torch.float32), B=T(rhs, torch.float32),
                      rhs=T(rhs, torch.float32), prior=T(np.full(C, 1 / C), torch.float32),
                      is_new=torch.zeros(n, dtype=torch.bool, device="cuda"),
                      seed=torch.zeros(n, dtype=torch.bool, device="cuda"), comps={}, K=C, C=C, eta=0.0,
                      n_inserted=0, n_deleted=0, n_active=n)
    Z = solvers.padded_empty(n, C, torch.float32, "cuda")
    st = solvers.Stats()
    solvers.pcg(S, Z, S.rhs, None, solvers.jacobi_M(S), 10_000, st, target_relres=1e-5, use_graph=graph,
                zero_start=True)
    Zn = Z.double().cpu().numpy()
    Ad = ssp.diags(diag) - A
    rel = np.linalg.norm(rhs - Ad @ Zn, axis=0) / np.linalg.norm(rhs, axis=0)
    assert rel.max() <= 1e-5 * 1.01 and st.iters < 300, (rel.max(), st.iters)
    np.testing.assert_allclose(Zn, direct_solve(Ad, rhs), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("graph", [True, False])
def test_fused_pcg_zero_start_is_the_same_solve(graph):
    """Mode bit 2 (Z == 0 on entry: R = rhs, no SpMM) gives the reference's iteration counts and
    iterate, exactly as the plain start from Z = 0 does."""
    g, A, S = golden_system()
    for tag in ("pcg_loose", "pcg_tight"):
        out = []
        for zs in (False, True):
            Z = torch.zeros((A.shape[0], 3), dtype=torch.float64, device="cuda")
            st = solvers.Stats()
            solvers.pcg(S, Z, S.rhs, g[f"{tag}_eps"].tolist(), solvers.jacobi_M(S), 10_000, st, use_graph=graph,
                        zero_start=zs)
            assert st.iters == int(g[f"{tag}_iters"]), (tag, zs, st.iters)
            out.append(Z.cpu().numpy())
        np.testing.assert_allclose(out[1], out[0], rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(out[1], g[f"{tag}_Z"], rtol=1e-8, atol=1e-11)


@pytest.mark.parametrize("graph", [True, False])
def test_fused_pcg_zero_start_ignores_incoming_z(graph):
    """A zero start sets Z = 0 itself: a Z full of NaN gives the reference's iteration counts and the
    same iterate as a zeroed Z."""
    g, A, S = golden_system()
    for tag in ("pcg_loose", "pcg_tight"):
        out = []
        for fill in (0.0, float("nan")):
            Z = torch.full((A.shape[0], 3), fill, dtype=torch.float64, device="cuda")
            st = solvers.Stats()
            solvers.pcg(S, Z, S.rhs, g[f"{tag}_eps"].tolist(), solvers.jacobi_M(S), 10_000, st, use_graph=graph,
                        zero_start=True)
            assert st.iters == int(g[f"{tag}_iters"]), (tag, fill, st.iters)
            out.append(Z.cpu().numpy())
        np.testing.assert_array_equal(out[1], out[0])


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
@pytest.mark.parametrize("n,C", [(1, 1), (1000, 3), (300_000, 9), (50_000, 33)])
def test_residual_stats_match_torch(dt, n, C):
    """dlp_residual_stats: rho_cols, column sums of squares of R and rhs, max |h| in one pass."""
    gen = torch.Generator(device="cuda").manual_seed(n + C)
    ldr = C + (1 if dt == torch.float64 and C % 2 else 0)
    R = torch.randn((n, ldr), generator=gen, device="cuda", dtype=torch.float64).to(dt)[:, :C]
    rhs = torch.randn((n, C), generator=gen, device="cuda", dtype=torch.float64).to(dt)
    diag = (torch.rand(n, generator=gen, device="cuda", dtype=torch.float64) + 0.5).to(dt)
    Z = torch.randn((n, C + 2), generator=gen, device="cuda", dtype=torch.float64).to(dt)
    S = stream.System(t=0, U=torch.arange(n, device="cuda"), W=None, s=diag, diag=diag, B=rhs, rhs=rhs, prior=None,
                      is_new=None, seed=None, comps={}, K=C, C=C, eta=0.0, n_inserted=0, n_deleted=0, n_active=n)
    rc, ss, bb, hm = solvers.residual_stats(S, R, rhs=rhs, H=Z[:, C:C + 1])
    R64, d64 = R.double(), diag.double()
    np.testing.assert_allclose(rc, (R64.abs() / d64[:, None]).max(0).values.cpu().numpy(), rtol=1e-15)
    np.testing.assert_allclose(ss, (R64 ** 2).sum(0).cpu().numpy(), rtol=1e-12)
    np.testing.assert_allclose(bb, (rhs.double() ** 2).sum(0).cpu().numpy(), rtol=1e-12)
    assert hm == float(Z[:, C].double().abs().max())
    rc2, ss2, bb2, hm2 = solvers.residual_stats(S, R)
    assert rc2 == rc and ss2 == ss and bb2 is None and hm2 is None


def test_push_rounds_match_reference():
    g, A, S = golden_system()
    Z, R = T(g["push_Z0"]), T(g["push_R0"])
    ops = kernels.FrontierOps(S.W, 3)
    rec = []
    Z, R, ok = solvers.push(S, Z, R, g["push_eps"].tolist(), ops, solvers.Stats(), record=rec)
    assert ok == bool(g["push_ok"]) and len(rec) == int(g["push_rounds"])
    off, cand = g["push_cand_off"], g["push_cand"]
    for k, (c, _t) in enumerate(rec):
        np.testing.assert_array_equal(c.cpu().numpy(), cand[off[k]:off[k + 1]])
    np.testing.assert_allclose(Z.cpu().numpy(), g["push_Z"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(R.cpu().numpy(), g["push_R"], rtol=1e-6, atol=1e-13)
    # touched sets equal the oracle's too
    Zo, Ro, oko, ito, rounds = O.push(A, g["diag"], g["push_Z0"].copy(), g["push_R0"].copy(), g["push_eps"], record=True)
    for (c, t), (co, to) in zip(rec, rounds):
        np.testing.assert_array_equal(t.cpu().numpy(), to)


def test_dynlp_frontier_matches_oracle():
    g, A, S = golden_system()
    rs = np.random.RandomState(3)
    seed = np.zeros(A.shape[0], dtype=bool)
    seed[rs.choice(A.shape[0], 50, replace=False)] = True
    S.seed = T(seed)
    solver = solvers.DynLP(A.shape[0], 3, "float64", delta=1e-6)
    rec = []
    solver.solve(S, record=rec)
    X0 = np.full((A.shape[0], 3), 1 / 3)
    Xo, it, fronts = O.dynlp_frontier(A, g["diag"], g["rhs"], X0, np.flatnonzero(seed), 1e-6, record=True)
    assert len(rec) == len(fronts)
    for a, b in zip(rec, fronts):
        np.testing.assert_array_equal(a.cpu().numpy(), b)
    np.testing.assert_allclose(solver.F.cpu().numpy(), Xo, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("method", ["pcg", "auto"])
@pytest.mark.parametrize("K", [2, 3])
def test_dynlp_plus_certificate_holds(method, K):
    """tests/test_dynlp.py:109-120 on our stack: cert <= tol and err <= 1.05 cert."""
    ds = graphs.sbm(3000, K=K, deg=8, seed=3, dtype="float32")
    rs = np.random.RandomState(0)
    lab = np.zeros(3000, bool)
    lab[rs.choice(3000, 60, replace=False)] = True
    S = stream.build_system(ds, torch.ones(3000, dtype=torch.bool, device="cuda"), T(lab), dtype="float32")
    solver = solvers.DynLPPlus(3000, K, "float32", method=method, tol=1e-3)
    st = solver.solve(S)
    S64 = S.astype(torch.float64)
    Wd = S64.W.to_scipy().astype(np.float64)
    Ad = ssp.diags(S64.diag.cpu().numpy()) - Wd
    Fd = direct_solve(Ad, S64.rhs.cpu().numpy())
    Fd = Fd.reshape(-1, 1) if Fd.ndim == 1 else Fd
    err = np.abs(solver.scores(S).cpu().numpy() - Fd).max()
    assert st.cert <= 1e-3 * 1.0001
    assert err <= st.cert * 1.05 + 1e-6, (err, st.cert)


def test_dynlp_plus_relres_target_fp32():
    ds = graphs.er_graph(20_000, 10, 8, seed=1)
    lab = graphs.label_mask(20_000, 0.005, seed=1)
    S = stream.build_system(ds, torch.ones(20_000, dtype=torch.bool, device="cuda"), lab, dtype="float32")
    solver = solvers.DynLPPlus(20_000, 8, "float32", method="pcg", tol=1e-3, target_relres=1e-8)
    st = solver.solve(S)
    S64 = S.astype(torch.float64)
    A = S64.W.to_scipy().astype(np.float64)
    rel = O.relres(A, S64.diag.cpu().numpy(), solver.scores(S).cpu().numpy(), S64.rhs.cpu().numpy())
    assert rel <= 1e-8 and st.relres <= 1e-8, (rel, st.relres)


def _oracle_edge_system(A_sc, y, K, lab):
    n = A_sc.shape[0]
    return O.build_system(A_sc, y, K, np.ones(n, bool), lab)


@pytest.mark.parametrize("weights", ["unit", "lognormal"])
def test_edge_stream_matches_rebuilt_system(weights):
    """After every edge batch the resident system equals the system rebuilt from scratch on the
    updated graph (the oracle's apply_edges + build_system), on its solved rows; inert rows carry
    no live entries, diag 1 and rhs 0 (tests/test_incremental.py:18-41 for edge batches)."""
    n, K = 4000, 3
    ds = graphs.planted_partition(n, K, 3.0, 1.0, weights=weights, seed=2)  # sparse: splits and regrounding
    lab = graphs.label_mask(n, 0.01, seed=2)
    es = stream.EdgeStream(ds, lab, slack_frac=0.0, slack_min=0)  # no slack: forces repacking
    up = graphs.EdgeUpdates(ds.A, seed=3, weights=weights)
    A_sc = ds.A.to_scipy().astype(np.float64)
    y, labn = ds.y.cpu().numpy(), lab.cpu().numpy()
    for t in range(6):
        b = up.next(300 if t % 2 else 1200, ins_frac=0.3 if t < 3 else 0.7)
        S = es.apply_edges(**b)
        A_sc = O.apply_edges(A_sc, b["ins_u"], b["ins_v"], b["ins_w"].astype(np.float64), b["del_u"], b["del_v"])
        # graph equality
        G = es.G.to_csr("aw").to_scipy().astype(np.float64)
        assert abs(G - A_sc.astype(np.float32).astype(np.float64)).max() == 0
        ref = _oracle_edge_system(A_sc.astype(np.float32).astype(np.float64), y, K, labn)
        U = S.solved.cpu().numpy()
        np.testing.assert_array_equal(np.flatnonzero(U), ref["U"])
        S64 = S.astype(torch.float64)
        Wd = es.G.to_csr("w").to_scipy().astype(np.float64)
        Uidx = ref["U"]
        assert abs(Wd[Uidx][:, Uidx] - ref["W"]).max() < 1e-12
        out = ~U
        assert abs(Wd[out]).sum() == 0 and abs(Wd[:, out]).sum() == 0
        np.testing.assert_allclose(S64.diag.cpu().numpy()[Uidx], ref["diag"], rtol=1e-10)
        np.testing.assert_allclose(S64.rhs.cpu().numpy()[Uidx], ref["rhs"], rtol=1e-10, atol=1e-12)
        assert (S64.diag.cpu().numpy()[out] == 1).all() and (S64.rhs.cpu().numpy()[out] == 0).all()
    assert es.counters["rebuilds"] >= 1 and es.counters["ground_changes"] >= 1


def test_incremental_solver_relres_on_edge_batches():
    n, K = 20_000, 4
    ds = graphs.er_graph(n, 10, K, seed=5)
    lab = graphs.label_mask(n, 0.01, seed=5)
    es = stream.EdgeStream(ds, lab)
    up = graphs.EdgeUpdates(ds.A, seed=5)
    solver = solvers.IncrementalLP(n, K, "float32", tol=1e-3, method="pcg", target_relres=1e-6, full_every=4)
    st = solver.solve(es.system)
    assert st.relres <= 1e-6
    for t in range(5):
        S = es.apply_edges(**up.next(400))
        st = solver.solve(S)
        S64 = S.astype(torch.float64)
        A = es.G.to_csr("w").to_scipy().astype(np.float64)
        F = solver.Z.cpu().numpy()[:, :K]
        rel = O.relres(A, S64.diag.cpu().numpy(), F, S64.rhs.cpu().numpy())
        assert rel <= 1e-6 and st.relres <= 1e-6, (t, rel, st.relres, st.path)
        # kept residual equals a fresh one (drift)
        R_true = S64.rhs_h.cpu().numpy() - (S64.diag.cpu().numpy()[:, None] * solver.Z.cpu().numpy() - A @ solver.Z.cpu().numpy())
        drift = np.abs(R_true - solver.R.cpu().numpy()).max() / S64.diag.cpu().numpy().min()
        assert drift < 1e-9, drift


@pytest.mark.parametrize("K", [4, 8, 17])
def test_incremental_solver_class_sum(K):
    """class_sum: the refinement's corrections solve K - 1 class columns and h and set the last class
    to one minus the others (the scores of a grounded row sum to one). On an edge stream: every
    column meets the relative-residual target on the fp64 residual, the kept residual stays the true
    one, the scores sum to one on the solved rows and match the full solve's to 1e-5."""
    n = 20_000
    ds = graphs.er_graph(n, 10, K, seed=6)
    lab = graphs.label_mask(n, 0.01, seed=6)
    up = graphs.EdgeUpdates(ds.A, seed=6)
    batches = [up.next(400) for _ in range(5)]
    out = []
    for cs in (True, False):
        es = stream.EdgeStream(ds, lab)
        solver = solvers.IncrementalLP(n, K, "float32", tol=1e-3, method="pcg", target_relres=1e-6, full_every=4,
                                       class_sum=cs)
        solver.solve(es.system)
        for t, b in enumerate(batches):
            S = es.apply_edges(**b)
            st = solver.solve(S)
            S64 = S.astype(torch.float64)
            A = es.G.to_csr("w").to_scipy().astype(np.float64)
            Z = solver.Z.cpu().numpy()
            rel = O.relres(A, S64.diag.cpu().numpy(), Z[:, :K], S64.rhs.cpu().numpy())
            assert rel <= 1e-6 and st.relres <= 1e-6, (cs, t, rel, st.relres)
            R_true = S64.rhs_h.cpu().numpy() - (S64.diag.cpu().numpy()[:, None] * Z - A @ Z)
            assert np.abs(R_true - solver.R.cpu().numpy()).max() / S64.diag.cpu().numpy().min() < 1e-9
        solved = S.solved.cpu().numpy()
        if cs:
            np.testing.assert_allclose(Z[solved, :K].sum(axis=1), 1.0, rtol=0, atol=1e-12)
        out.append(Z[:, :K])
    np.testing.assert_allclose(out[0], out[1], rtol=0, atol=1e-5)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("C", [2, 4, 9])
def test_fused_push_reaches_tolerance(dtype, C):
    """tests/test_incremental.py:66-81: the asynchronous push converges, its kept residual is the
    true one (up to rounding) and meets eps everywhere."""
    ds = graphs.sbm(4000, K=2, deg=8.0, seed=9, dtype="float32")
    lab = graphs.label_mask(4000, 0.03, seed=9)
    es = stream.EdgeStream(ds, lab)
    s = es.system.astype(dtype)
    rs = np.random.RandomState(0)
    solved = s.solved.cpu().numpy()
    rhs = T(rs.random_sample((4000, C)) * solved[:, None], dtype)
    Z = torch.zeros((4000, C), dtype=dtype, device="cuda")
    R = solvers.residual(s, Z, rhs)
    eps = [1e-5 if dtype == torch.float64 else 1e-4] * C
    cand = kernels.flatnonzero((R.abs() > 0).any(dim=1).to(torch.uint8))
    fp = kernels.FusedPush(s.W, C)
    rounds, ok, edges = fp.run(Z, R, s.diag, eps, cand, 100_000)
    assert ok and rounds > 0 and edges > 0
    R_true = solvers.residual(s, Z, rhs)
    np.testing.assert_allclose(R.cpu().numpy(), R_true.cpu().numpy(), atol=1e-4 if dtype == torch.float32 else 1e-10)
    viol = (R_true.abs() / s.diag.to(dtype)[:, None]).max().item() / eps[0]
    assert viol <= 1.0 + (0.05 if dtype == torch.float32 else 1e-6), viol


def test_incremental_push_path_on_small_batches():
    """IncrementalLP's small-batch branch (dynlp/solvers.py:414-422) certifies with the fused push."""
    n, K = 6000, 3
    ds = graphs.planted_partition(n, K, 6.0, 2.0, seed=4)
    lab = graphs.label_mask(n, 0.02, seed=4)
    es = stream.EdgeStream(ds, lab)
    up = graphs.EdgeUpdates(ds.A, seed=4)
    solver = solvers.IncrementalLP(n, K, "float32", tol=1e-3, push_frac=0.2)
    solver.solve(es.system)
    paths = []
    for _ in range(4):
        S = es.apply_edges(**up.next(40))
        st = solver.solve(S)
        paths.append(st.path)
        S64 = S.astype(torch.float64)
        A = es.G.to_csr("w").to_scipy().astype(np.float64)
        U = S.solved.cpu().numpy()
        Ad = ssp.diags(S64.diag.cpu().numpy()) - A
        Fd = direct_solve(Ad, S64.rhs.cpu().numpy())
        err = np.abs(solver.Z.cpu().numpy()[U, :K] - Fd[U]).max()
        assert st.cert <= 1e-3 * 1.0001 and err <= st.cert * 1.05 + 1e-9, (st.path, err, st.cert)
    assert "inc-push" in paths, paths


def _empty_i32():
    return np.zeros(0, np.int32)


@pytest.mark.parametrize("order", ["appends_first", "reinserts_first"])
def test_reinsert_of_squeezed_edges_next_to_appends(order):
    """Edges deleted in one batch and inserted again in the next, in the same batch as insertions
    of new edges into the same rows. Each deleted edge is its row's last stored entry, so after the
    squeeze its column id is still in the freed slot, which the new edges of that row are appended
    into: a lookup that ran while appends were in flight could take that slot for the deleted edge.
    The resident graph must equal the oracle's graph after each batch, symmetric and with every
    weight in place."""
    n, K = 20_000, 3
    ds = graphs.er_graph(n, 8, K, seed=21)
    lab = graphs.label_mask(n, 0.02, seed=21)
    es = stream.EdgeStream(ds, lab)
    A_sc = ds.A.to_scipy().astype(np.float64)
    rbeg, rend = es.G.rbeg.cpu().numpy(), es.G.rend.cpu().numpy()
    col = es.G.indices.cpu().numpy()
    rng = np.random.default_rng(0)
    rows = rng.choice(n, 6000, replace=False)
    last = {}
    for a in rows:
        if rend[a] > rbeg[a]:
            c = int(col[rend[a] - 1])
            last[(min(a, c), max(a, c))] = a
    du = np.array([k[0] for k in last], np.int32)
    dv = np.array([k[1] for k in last], np.int32)
    es.apply_edges(del_u=du, del_v=dv)
    A_sc = O.apply_edges(A_sc, _empty_i32(), _empty_i32(), np.zeros(0), du, dv)
    G = es.G.to_csr("aw").to_scipy().astype(np.float64)
    assert abs(G - A_sc).max() == 0
    # the next batch: the deleted edges again (weight 2) and a new edge (weight 3) on each of their rows
    Acoo = A_sc.tolil()
    nu, nv = [], []
    for (a, c), r in last.items():
        while True:
            b = int(rng.integers(0, n))
            if b != r and Acoo[r, b] == 0 and (min(r, b), max(r, b)) not in last:
                break
        nu.append(r)
        nv.append(b)
    nu, nv = np.array(nu, np.int32), np.array(nv, np.int32)
    if order == "appends_first":
        iu, iv = np.concatenate([nu, du]), np.concatenate([nv, dv])
        iw = np.concatenate([np.full(nu.size, 3.0), np.full(du.size, 2.0)]).astype(np.float32)
    else:
        iu, iv = np.concatenate([du, nu]), np.concatenate([dv, nv])
        iw = np.concatenate([np.full(du.size, 2.0), np.full(nu.size, 3.0)]).astype(np.float32)
    S = es.apply_edges(ins_u=iu, ins_v=iv, ins_w=iw)
    A_sc = O.apply_edges(A_sc, iu, iv, iw.astype(np.float64), _empty_i32(), _empty_i32())
    G = es.G.to_csr("aw").to_scipy().astype(np.float64)
    assert abs(G - G.T).max() == 0
    assert abs(G - A_sc).max() == 0
    # the grounded system follows the graph
    ref = _oracle_edge_system(A_sc, ds.y.cpu().numpy(), K, lab.cpu().numpy())
    np.testing.assert_array_equal(np.flatnonzero(S.solved.cpu().numpy()), ref["U"])
    np.testing.assert_allclose(S.astype(torch.float64).diag.cpu().numpy()[ref["U"]], ref["diag"], rtol=1e-12)


def test_coalesced_batches_then_one_solve():
    """Several edge batches patched before one solve (the serving loop's coalescing,
    apply_edges(keep_pending=True)): the solve refreshes every row any batch changed, so the scores
    meet the relative residual on the oracle's system rebuilt from the final graph."""
    n, K = 20_000, 4
    ds = graphs.er_graph(n, 10, K, seed=12)
    lab = graphs.label_mask(n, 0.01, seed=12)
    es = stream.EdgeStream(ds, lab)
    up = graphs.EdgeUpdates(ds.A, seed=12)
    solver = solvers.IncrementalLP(n, K, "float32", tol=1e-3, method="pcg", target_relres=1e-6, full_every=64)
    solver.solve(es.system)
    A_sc = ds.A.to_scipy().astype(np.float64)
    for rnd in range(2):
        for i in range(3):
            b = up.next(500)
            S = es.apply_edges(**b, keep_pending=i > 0)
            A_sc = O.apply_edges(A_sc, b["ins_u"], b["ins_v"], b["ins_w"].astype(np.float64), b["del_u"], b["del_v"])
        st = solver.solve(S)
        ref = _oracle_edge_system(A_sc, ds.y.cpu().numpy(), K, lab.cpu().numpy())
        U = ref["U"]
        F = solver.Z[:, :K].cpu().numpy()[U]
        rel = O.relres(ref["W"], ref["diag"], F, ref["rhs"])
        assert rel <= 1e-6 and st.relres <= 1e-6, (rnd, rel, st.relres)


@pytest.mark.parametrize("C", [5, 6, 8])
def test_row_sweep_keeps_padding_and_follows_column_sweep(C):
    """The two-kernel iteration's sweep takes one row per thread where R, Z, P and AP all have
    32-byte rows of at most 8 floats (k_pcg_fused_rows8), else one (row, column) element per thread.
    Through the C ABI with every buffer on an 8-float pitch (padding columns of R and Z holding a
    sentinel) against the same solve with Z on a 12-float pitch (the element sweep): the sentinels
    stay, the scores agree to fp32 rounding, the iteration counts within one, and both meet the
    relative-residual target on the fp64 residual."""
    from dynlplus_b200 import _lib
    from dynlplus_b200.backend import code, ld, ptr, stream, workspace
    import ctypes as ct
    S, A, diag, rhs = _whole_row_system(C, seed=11)
    n = A.shape[0]
    W = S.W
    d32 = S.diag.to(torch.float32).contiguous()
    b32 = S.rhs.to(torch.float32).contiguous()
    rn = (ct.c_double * C)(*[float(x) for x in np.linalg.norm(rhs, axis=0)])
    out = []
    for ldz in (8, 12):
        Rb = torch.full((n, 8), -7.0, dtype=torch.float32, device="cuda")
        Zb = torch.full((n, ldz), -7.0, dtype=torch.float32, device="cuda")
        Zb[:, :C] = 0.0
        P = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
        AP = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
        R, Z = Rb[:, :C], Zb[:, :C]
        ws = workspace("pcg_test").get(_lib.lib().dlp_pcg_workspace_bytes(C))
        it, viol, rel, status = ct.c_int32(0), ct.c_double(0), ct.c_double(0), ct.c_int32(0)
        _lib.call("dlp_pcg", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(W.data), code(W.data), n, C, ptr(d32),
                  ptr(b32), ld(b32), ptr(Z), ld(Z), ptr(R), ld(R), ptr(P), ld(P), ptr(AP), ld(AP), code(Z), None, rn,
                  1e-5, 2 | 4, 10_000, 400, 8, 1, W.nnz / n, ptr(ws), ws.numel(), ct.byref(it), ct.byref(viol),
                  ct.byref(rel), ct.byref(status), stream(), None, None, 0)
        torch.cuda.synchronize()
        assert status.value == 5, status.value
        assert (Zb[:, C:] == -7.0).all() and (Rb[:, C:] == -7.0).all()
        out.append((Z.double().cpu().numpy(), it.value))
    (Zr, itr), (Ze, ite) = out
    assert abs(itr - ite) <= 1, (itr, ite)
    Ad = ssp.diags(diag) - A
    for Zx in (Zr, Ze):
        relv = np.linalg.norm(rhs - Ad @ Zx, axis=0) / np.linalg.norm(rhs, axis=0)
        assert relv.max() <= 1e-5 * 1.01, relv.max()
    np.testing.assert_allclose(Zr, Ze, rtol=0, atol=2e-5 * np.abs(Ze).max())

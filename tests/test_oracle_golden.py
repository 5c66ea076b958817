"""The oracle restates the reference faithfully: it reproduces the reference's own outputs
(tests/golden/*.npz, made by running the reference itself on the CPU) (CPU-only)."""
import numpy as np
import pytest

from conftest import golden_csr, load_golden
from oracle import ref_np as O


def test_cc_matches_reference():
    g = load_golden("cc.npz")
    for i in range(int(g["ncases"])):
        n = int(g[f"c{i}_n"])
        lab, nc = O.connected_components(n, g[f"c{i}_rows"], g[f"c{i}_cols"])
        np.testing.assert_array_equal(lab, g[f"c{i}_labels"])
        assert nc == int(g[f"c{i}_ncomp"])
        lab2, nc2 = O.connected_components_fast(n, g[f"c{i}_rows"], g[f"c{i}_cols"])
        np.testing.assert_array_equal(lab2, g[f"c{i}_labels"])
        assert nc2 == nc


@pytest.mark.parametrize("C", [1, 3, 9, 17])
def test_kernel_definitions_match_reference(C):
    g = load_golden("kernels.npz")
    W = golden_csr(g, "W")
    f, diag = g["frontier"], g["diag"]
    X, rhs, a, D = g[f"C{C}_X"], g[f"C{C}_rhs"], g[f"C{C}_a"], g[f"C{C}_D"]
    Y, ch = O.frontier_jacobi(W, f, X, rhs, diag, 1e-2)
    np.testing.assert_allclose(Y, g[f"C{C}_jacY"], rtol=1e-13)
    np.testing.assert_array_equal(ch.astype(np.uint8), g[f"C{C}_jacch"])
    R = np.zeros_like(X)
    mark = np.zeros(W.shape[0], dtype=np.uint8)
    O.push_scatter(W, f, D, R, mark)
    np.testing.assert_allclose(R, g[f"C{C}_pushR"], rtol=1e-13, atol=1e-15)
    np.testing.assert_array_equal(mark, g[f"C{C}_pushmark"])
    mk = np.zeros(W.shape[0], dtype=np.uint8)
    O.mark_neighbors(W, f, mk)
    np.testing.assert_array_equal(mk, g[f"C{C}_marknb"])
    assert int(np.diff(W.indptr)[f].sum()) == int(g[f"C{C}_edges"]) // 3  # jacobi + push + mark each count
    if C > 1:
        np.testing.assert_allclose(O.spmm_axpy(W, X), g[f"C{C}_spmm"], rtol=1e-13)
    np.testing.assert_allclose(O.spmm_axpy(W, X, a=a, b=-1.0), g[f"C{C}_applyA"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("b", [0, 2])
def test_system_matches_reference(b):
    g = load_golden("system.npz")
    p = f"b{b}"
    A = golden_csr(g, f"{p}_A")
    S = O.build_system(A, g[f"{p}_y"], int(g[f"{p}_K"]), g[f"{p}_active"], g[f"{p}_labeled"])
    np.testing.assert_array_equal(S["U"], g[f"{p}_U"])
    Wg = golden_csr(g, f"{p}_W")
    np.testing.assert_array_equal(S["W"].indptr, Wg.indptr)
    np.testing.assert_array_equal(S["W"].indices, Wg.indices)
    np.testing.assert_allclose(S["W"].data, Wg.data, rtol=0)
    for k in ("s", "diag", "B", "rhs"):
        np.testing.assert_allclose(S[k], g[f"{p}_{k}"], rtol=1e-13, err_msg=k)
    assert S["n_ungrounded"] == int(g[f"{p}_n_ungrounded"])


def test_pcg_matches_reference():
    g = load_golden("solvers.npz")
    W, diag, rhs = golden_csr(g, "W"), g["diag"], g["rhs"]
    for tag in ("pcg_loose", "pcg_tight"):
        Z, it = O.pcg(W, diag, np.zeros_like(rhs), rhs.copy(), g[f"{tag}_eps"])
        assert it == int(g[f"{tag}_iters"]), tag
        np.testing.assert_allclose(Z, g[f"{tag}_Z"], rtol=1e-9, atol=1e-12)


def test_push_rounds_match_reference():
    g = load_golden("solvers.npz")
    W, diag = golden_csr(g, "W"), g["diag"]
    Z, R, ok, it, rounds = O.push(W, diag, g["push_Z0"].copy(), g["push_R0"].copy(), g["push_eps"], record=True)
    assert ok == bool(g["push_ok"]) and it == int(g["push_rounds"])
    off, cand = g["push_cand_off"], g["push_cand"]
    for k, (c, _touched) in enumerate(rounds):
        np.testing.assert_array_equal(c, cand[off[k]:off[k + 1]])
    np.testing.assert_allclose(Z, g["push_Z"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(R, g["push_R"], rtol=1e-9, atol=1e-16)


def test_apply_edges_set_semantics():
    """Edge batches: delete-then-insert, symmetric, self-loops and absent deletions ignored."""
    A = O.symmetric_from_pairs(np.array([0, 1, 2]), np.array([1, 2, 3]), np.ones(3), 5, np.float64)
    B = O.apply_edges(A, [0, 4, 2, 2], [4, 4, 3, 1], [2.0, 9.0, 5.0, 7.0], [1, 3, 0], [2, 4, 4])
    D = B.toarray()
    assert D[0, 4] == D[4, 0] == 2.0            # inserted
    assert D[4, 4] == 0                          # self-loop ignored
    assert D[2, 3] == D[3, 2] == 5.0             # insertion of a present edge sets its weight
    assert D[1, 2] == D[2, 1] == 7.0             # deleted then re-inserted in the same batch
    assert D[0, 1] == 1.0                        # untouched
    assert (D == D.T).all()


def test_amg_matches_reference():
    g = load_golden("amg.npz")
    W = golden_csr(g, "W")
    a2, nc = O.handshake(W.shape[0], O.csr_rows(W), W.indices, W.data, 3)
    np.testing.assert_array_equal(a2, g["match_agg"])
    assert nc == int(g["match_nc"])
    Wc, sc = O.coarsen(W, g["s"], a2, nc)
    Wg = golden_csr(g, "match_Wc")
    assert abs(Wc - Wg).max() <= 1e-6 * abs(Wg).max()
    np.testing.assert_allclose(sc, g["match_sc"], rtol=1e-6)  # the reference sums fp32 groundings in fp32
    amg = O.AMGOracle(W, g["s"].astype(np.float32), max_coarse=50)
    assert amg.sizes == list(g["sizes"])
    for i, L in enumerate(amg.levels):
        np.testing.assert_array_equal(L["agg"], g[f"L{i}_agg"])
    np.testing.assert_allclose(amg(g["R"].astype(np.float64)), g["MR"], rtol=1e-4, atol=1e-5 * abs(g["MR"]).max())


def _stream_fixture():
    g = load_golden("stream.npz")
    A = golden_csr(g, "A")
    return g, A, g["y"], int(g["K"])


def test_stream_schedule_matches_reference():
    g, A, y, K = _stream_fixture()
    lab, order, n0, sched = O.stream_schedule(y, K, g["order_in"], label_frac=0.02, init_frac=0.2, n_batches=4,
                                              del_frac=0.1, seed=1)
    np.testing.assert_array_equal(lab, g["labeled"])
    np.testing.assert_array_equal(order, g["order"])
    assert n0 == int(g["n0"]) and len(sched) == int(g["nbatches"])
    for t, (ins, dele) in enumerate(sched):
        np.testing.assert_array_equal(ins, g[f"t{t}_ins"])
        np.testing.assert_array_equal(dele, g[f"t{t}_del"])
    assert float(A.data.mean()) == float(g["tau"]) and float(A.data.max()) == float(g["wmax"])


def test_stream_systems_and_warm_starts_match_reference():
    """Every batch of Stream._build: U, the new rows, DynLP's seed, the tau and FH components of
    the new vertices (exact), and the warm starts supernode_init / init_h (dynlp/solvers.py:128-163)."""
    g, A, y, K = _stream_fixture()
    n = A.shape[0]
    labeled = g["labeled"]
    active, prevU = np.zeros(n, bool), np.zeros(n, bool)
    for t in range(int(g["nbatches"])):
        ins, dele = g[f"t{t}_ins"], g[f"t{t}_del"]
        active[ins], active[dele] = True, False
        S = O.stream_system(A, y, K, active, labeled, prevU, ins, dele, float(g["tau"]), float(g["wmax"]))
        p = f"s{t}"
        np.testing.assert_array_equal(S["U"], g[f"{p}_U"])
        np.testing.assert_array_equal(S["is_new"], g[f"{p}_is_new"])
        np.testing.assert_array_equal(S["seed"], g[f"{p}_seed"])
        for name in ("tau", "fh"):
            lab, nc = S["comps"][name]
            np.testing.assert_array_equal(lab, g[f"{p}_{name}"], err_msg=f"{p} {name}")
            assert nc == int(g[f"{p}_{name}_nc"])
        np.testing.assert_allclose(S["diag"], g[f"{p}_diag"], rtol=1e-13)
        np.testing.assert_allclose(S["rhs"], g[f"{p}_rhs"], rtol=1e-13, atol=1e-15)
        prior = np.full(K, 1.0 / K)
        X0 = O.supernode_init(S["W"], S["B"], K, prior, S["is_new"], S["comps"], g[f"{p}_X"], comp="tau")
        np.testing.assert_allclose(X0, g[f"{p}_sn_tau"], rtol=1e-13)
        known = ~S["is_new"]
        X1 = O.supernode_init(S["W"], S["B"], K, prior, S["is_new"], S["comps"], g[f"{p}_X"], known, comp="fh")
        np.testing.assert_allclose(X1, g[f"{p}_sn_fh"], rtol=1e-13)
        H1 = O.init_h(S["W"], S["B"], S["is_new"], S["comps"], g[f"{p}_H"], known, 7.0)
        np.testing.assert_allclose(H1, g[f"{p}_ih"], rtol=1e-13)
        prevU = np.zeros(n, bool)
        prevU[S["U"]] = True

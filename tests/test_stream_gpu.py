"""Vertex-arrival streams (dynlp/stream.py:84-346) and new-vertex warm starts
(dynlp/solvers.py:128-163) on the device, against the reference's own outputs (GPU)."""
import numpy as np
import pytest
import torch

from conftest import golden_csr, load_golden
from dynlplus_b200 import graphs, solvers, stream
from dynlplus_b200.backend import CSR

pytestmark = pytest.mark.gpu

KW = dict(init_frac=0.2, n_batches=4, label_frac=0.02, del_frac=0.1, seed=1)


def T(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def _dataset(g, key):
    A = golden_csr(g, key)
    return graphs.Dataset("fixture", CSR.from_scipy(A), T(g["y"]), int(g["K"]), T(g["order_in"]))


def test_stream_schedule_matches_reference():
    g = load_golden("stream.npz")
    st = stream.Stream(_dataset(g, "A"), dtype="float64", **KW)
    np.testing.assert_array_equal(st.labeled.cpu().numpy(), g["labeled"])
    np.testing.assert_array_equal(st.order.cpu().numpy(), g["order"])
    assert st.n0 == int(g["n0"]) and len(st) == int(g["nbatches"])
    assert st.tau == float(g["tau"]) and st.wmax == float(g["wmax"])
    for t, (ins, dele) in enumerate(st.schedule):
        np.testing.assert_array_equal(ins.cpu().numpy(), g[f"t{t}_ins"])
        np.testing.assert_array_equal(dele.cpu().numpy(), g[f"t{t}_del"])


def test_stream_systems_components_and_warm_starts_match_reference():
    """Every batch: U, new rows, DynLP's seed, the tau and FH components of the new vertices
    (exact), the system (1e-12) and the warm starts supernode_init / init_h (1e-12)."""
    g = load_golden("stream.npz")
    st = stream.Stream(_dataset(g, "A"), dtype="float64", **KW)
    for t, S in enumerate(st.batches()):
        p = f"s{t}"
        np.testing.assert_array_equal(S.U.cpu().numpy(), g[f"{p}_U"])
        np.testing.assert_array_equal(S.is_new.cpu().numpy(), g[f"{p}_is_new"])
        np.testing.assert_array_equal(S.seed.cpu().numpy(), g[f"{p}_seed"])
        for name in ("tau", "fh"):
            lab, nc = S.comps[name]
            np.testing.assert_array_equal(lab.cpu().numpy(), g[f"{p}_{name}"], err_msg=f"{p} {name}")
            assert nc == int(g[f"{p}_{name}_nc"])
        np.testing.assert_allclose(S.diag.cpu().numpy(), g[f"{p}_diag"], rtol=1e-12)
        np.testing.assert_allclose(S.rhs.cpu().numpy(), g[f"{p}_rhs"], rtol=1e-12, atol=1e-14)
        X = solvers.supernode_init(S, T(g[f"{p}_X"]), comp="tau")
        np.testing.assert_allclose(X.cpu().numpy(), g[f"{p}_sn_tau"], rtol=1e-12)
        known = ~S.is_new
        X = solvers.supernode_init(S, T(g[f"{p}_X"]), known, comp="fh")
        np.testing.assert_allclose(X.cpu().numpy(), g[f"{p}_sn_fh"], rtol=1e-12)
        H = solvers.init_h(S, T(g[f"{p}_H"]), known, 7.0)
        np.testing.assert_allclose(H.cpu().numpy(), g[f"{p}_ih"], rtol=1e-12)


def test_incremental_stream_matches_reference():
    """The resident form: solved rows, changed rows (within U), new rows, seed, components of the
    new vertices over the masked weights, and the global-index fp64 system (inert rows diag 1,
    rhs 0) after every batch (dynlp/stream.py:300-346)."""
    g = load_golden("stream.npz")
    ds = _dataset(g, "A32")
    ist = stream.IncrementalStream(ds, ball_hops=3, dtype="float32", **KW)
    assert ist.tau == float(g["tau32"]) and ist.wmax == float(g["wmax32"])
    prev_diag = prev_rhs = None
    for t, S in enumerate(ist.batches()):
        p = f"i{t}"
        solved = S.solved.cpu().numpy()
        np.testing.assert_array_equal(solved, g[f"{p}_solved"])
        # changed rows: every solved row whose equation changed is listed, and nothing outside the
        # reference's list (which also names rows touched by a vertex that left U and re-entered
        # it in the same batch, whose equations are unchanged)
        ch = np.zeros(solved.shape[0], bool)
        ch[S.changed.cpu().numpy()] = True
        ours = np.flatnonzero(ch & solved)
        assert set(ours) <= set(g[f"{p}_changed"].tolist())
        if prev_diag is not None:
            moved = (g[f"{p}_diag"] != prev_diag) | (g[f"{p}_rhs"] != prev_rhs).any(axis=1)
            assert set(np.flatnonzero(moved & solved)) <= set(ours)
        prev_diag, prev_rhs = g[f"{p}_diag"], g[f"{p}_rhs"]
        np.testing.assert_array_equal(S.is_new.cpu().numpy(), g[f"{p}_is_new"])
        np.testing.assert_array_equal(S.seed.cpu().numpy(), g[f"{p}_seed"])
        for name in ("tau", "fh"):
            lab, nc = S.comps[name]
            np.testing.assert_array_equal(lab.cpu().numpy(), g[f"{p}_{name}"], err_msg=f"{p} {name}")
            assert nc == int(g[f"{p}_{name}_nc"])
        S64 = S.astype(torch.float64)
        np.testing.assert_allclose(S64.diag.cpu().numpy(), g[f"{p}_diag"], rtol=1e-12)
        np.testing.assert_allclose(S64.rhs.cpu().numpy(), g[f"{p}_rhs"], rtol=1e-12, atol=1e-14)
        assert S.n_ungrounded == int(g[f"{p}_n_ungrounded"])


@pytest.mark.parametrize("name", ["dynlp", "dynlp-fh", "dynlp+pcg", "dynlp+inc"])
def test_solvers_on_vertex_stream_are_close_to_direct(name):
    """The solvers with their warm starts on every batch of the vertex stream: DynLP to its delta
    contract, DynLP+ / the resident solver within their certified bound of a direct solve."""
    import scipy.sparse as ssp
    from conftest import direct_solve
    g = load_golden("stream.npz")
    ds = _dataset(g, "A32")
    n, K = ds.n, ds.K
    inc = name == "dynlp+inc"
    st = (stream.IncrementalStream if inc else stream.Stream)(ds, dtype="float32", **KW)
    if name.startswith("dynlp-") or name == "dynlp":
        solver = solvers.DynLP(n, K, "float32", delta=1e-7, comp="fh" if name == "dynlp-fh" else "tau")
    elif inc:
        solver = solvers.IncrementalLP(n, K, "float32", tol=1e-4)
    else:
        solver = solvers.DynLPPlus(n, K, "float32", method="pcg", tol=1e-4)
    for S in st.batches():
        stt = solver.solve(S)
        S64 = S.astype(torch.float64)
        Wd = S64.W.to_scipy().astype(np.float64)
        U = torch.nonzero(S.solved, as_tuple=False).flatten().cpu().numpy() if inc else np.arange(S.n_u)
        A = (ssp.diags(S64.diag.cpu().numpy()) - Wd).tocsr()[U][:, U]
        Fd = direct_solve(A, S64.rhs.cpu().numpy()[U])
        F = (solver.F if inc else solver.scores(S)).double().cpu().numpy()[U] if not inc else \
            solver.F.cpu().numpy()[U]
        err = abs(F - Fd).max()
        if name.startswith("dynlp") and "+" not in name:
            assert err < 1e-3, err
        else:
            assert err <= max(1.05 * stt.cert, 1e-9), (err, stt.cert)


@pytest.mark.parametrize("incremental", [False, True])
def test_streaming_benchmark_rows(tmp_path, incremental):
    """The reference's streaming benchmark (dynlp/bench.py) on a small SBM stream: one CSV row per
    batch and solver with the reference's columns; certified solvers within their bound of F*."""
    import csv
    from dynlplus_b200 import bench as sb
    out = str(tmp_path / "run.csv")
    names = "itlp,dynlp,dynlp-fh,dynlp+pcg,dynlp+auto" + (",dynlp+inc" if incremental else "")
    argv = ["--dataset", "sbm", "--n", "6000", "--classes", "3", "--deg", "8", "--batches", "3", "--init-frac", "0.4",
            "--label-frac", "0.02", "--solvers", names, "--out", out, "--no-warmup"] + (["--incremental"] if incremental
                                                                                        else [])
    rows = sb.main(argv)
    assert len(rows) == 4 * len(names.split(","))
    with open(out) as fh:
        r = list(csv.DictReader(fh))
    assert list(r[0].keys()) == sb.FIELDS and len(r) == len(rows)
    for row in rows:
        if row["solver"].startswith("dynlp+"):
            assert row["err_max"] <= max(1.05 * row["cert_self"], 1e-9), row
        assert 0.0 <= row["acc_true"] <= 1.0
    # the run's CSV through the results matrix: one line per solver, iterations summed over batches
    from dynlplus_b200 import matrix
    agg = matrix.main(str(tmp_path))
    assert [g["solver"] for g in agg] == names.split(",")
    for g in agg:
        assert g["iters"] == sum(r["iters"] for r in rows if r["solver"] == g["solver"])
    assert (tmp_path / "matrix.md").read_text(encoding="utf-8").startswith("# Method matrix:")

"""Parity at the sizes of the benchmark workloads (GPU): the edge stream of ER n=1,000,000 (mean
degree 10, k=8, 0.5% labelled, batches of 10,000 updates) and the SBM n=100,000 static solve plus a
1,000-update batch (k=4, 1% labelled), each batch against the oracle on the same seeded inputs:

  - the grounded set U and the component labels of the active unlabelled subgraph, bit-exact
    (Stream._build, dynlp/stream.py:142-177; connected_components, dynlp/cc.py:8-23);
  - the scores within 1e-5 of an fp64 solve of the oracle's rebuilt system (CG to a relative
    residual of 1e-11; the solution of the system does not depend on the start, so the CG starts
    from the GPU's scores to save iterations), relative to the largest score, and the relative
    residual <= 1e-6 on the oracle's system;
  - the argmax labels (predict, dynlp/solvers.py:166-167) equal to those of the fp64 solution except
    on near-ties: rows whose two best fp64 scores differ by at most twice the score error.
"""
import numpy as np
import pytest

from dynlplus_b200 import graphs, solvers, stream
from oracle import edge_cpu as E
from oracle import ref_np as O

pytestmark = pytest.mark.gpu

SCORE_RTOL = 1e-5   # score error relative to the largest score
RELRES = 1e-6       # relative residual of every label column


def _fp64_solution(ref, warm):
    """fp64 block Jacobi-PCG on the oracle's system to a relative residual of 1e-11 per column."""
    W, diag, rhs = ref["W"], ref["diag"], ref["rhs"]
    rn = np.sqrt((rhs * rhs).sum(axis=0))
    Z, _ = E.pcg_relres(W, diag, rhs, np.array(warm, dtype=np.float64), 1e-11, rn, max_iter=5000)
    return Z


def _check_batch(es, solver, S, A_sc, y, labn, K):
    """All the checks of one batch; returns their figures."""
    n = A_sc.shape[0]
    ref = O.build_system(A_sc, y, K, np.ones(n, bool), labn)
    U = ref["U"]
    # grounded set and component labels, bit-exact
    np.testing.assert_array_equal(np.flatnonzero(S.solved.cpu().numpy()), U)
    lab, ncomp = es.components()
    assert ncomp == ref["n_comp"]
    np.testing.assert_array_equal(lab.cpu().numpy(), ref["cc_labels"])
    # scores against the fp64 solution of the rebuilt system
    C = 1 if K == 2 else K
    F = solver.Z[:, :C].cpu().numpy()[U]
    Fs = _fp64_solution(ref, F)
    err = float(np.abs(F - Fs).max())
    scale = float(np.abs(Fs).max())
    assert err <= SCORE_RTOL * scale, (err, scale)
    rel = O.relres(ref["W"], ref["diag"], F, ref["rhs"])
    assert rel <= RELRES, rel
    # labels: equal to the fp64 solution's except on near-ties
    labels, _, _, _ = solver.relabel(S)
    got = labels.cpu().numpy()
    assert (got[np.setdiff1d(np.arange(n), U)] == -1).all()
    got = got[U]
    want = O.predict(Fs, K)
    if K == 2:
        tie = np.abs(Fs[:, 0] - 0.5) <= err
    else:
        top = np.sort(Fs, axis=1)
        tie = (top[:, -1] - top[:, -2]) <= 2 * err
    bad = got != want
    assert not (bad & ~tie).any(), (int(bad.sum()), int((bad & ~tie).sum()))
    return dict(err=err / scale, relres=rel, agree=float((~bad).mean()), near_ties=int(tie.sum()))


def _run(ds, lab, K, batches):
    n = ds.n
    es = stream.EdgeStream(ds, lab, components=True)
    solver = solvers.IncrementalLP(n, K, "float32", tol=1e-3, method="pcg", target_relres=RELRES, full_every=16)
    S = es.system
    solver.solve(S)
    A_sc = ds.A.to_scipy().astype(np.float64)
    y, labn = ds.y.cpu().numpy(), lab.cpu().numpy()
    _check_batch(es, solver, S, A_sc, y, labn, K)
    out = []
    for b in batches:
        S = es.apply_edges(**b)
        st = solver.solve(S)
        assert st.relres <= RELRES, st.relres
        A_sc = O.apply_edges(A_sc, b["ins_u"], b["ins_v"], b["ins_w"].astype(np.float64), b["del_u"], b["del_v"])
        out.append(_check_batch(es, solver, S, A_sc, y, labn, K))
    return out


def test_edge_stream_er1M_matches_oracle():
    """ER n=1,000,000, mean degree 10, k=8, 0.5% labelled: three batches of 10,000 updates."""
    n, K = 1_000_000, 8
    ds = graphs.er_graph(n, 10.0, K, seed=0)
    lab = graphs.label_mask(n, 0.005, seed=0)
    up = graphs.EdgeUpdates(ds.A, seed=0)
    info = _run(ds, lab, K, [up.next(10_000) for _ in range(3)])
    assert all(i["agree"] > 0.999 for i in info), info


def test_sbm100k_static_and_batch_match_oracle():
    """SBM n=100,000, 4 blocks (degree 12 in + 4 cross), unit weights, 1% labelled, k=4: the static
    solve, then one batch of 1,000 updates (500 insertions of non-edges, 500 deletions)."""
    n, K = 100_000, 4
    ds = graphs.planted_partition(n, 4, 12.0, 4.0, seed=0)
    lab = graphs.label_mask(n, 0.01, seed=0)
    up = graphs.EdgeUpdates(ds.A, seed=0)
    _run(ds, lab, K, [up.next(1000)])


def test_binary_column_edge_stream_matches_oracle():
    """K = 2 (the reference's one-column binary path, dynlp/stream.py:167): SBM n=50,000 with sparse
    cross edges and deletions that cut vertices off, so the grounded set and components move."""
    n, K = 50_000, 2
    ds = graphs.planted_partition(n, 2, 4.0, 1.0, seed=3)
    lab = graphs.label_mask(n, 0.01, seed=3)
    up = graphs.EdgeUpdates(ds.A, seed=3)
    _run(ds, lab, K, [up.next(4000, ins_frac=0.2), up.next(4000, ins_frac=0.8)])

"""Residual push with device-resident frontiers (dlp_fused_push) against the oracle's synchronous
push (dynlp/solvers.py:100-125), its round cap and cancellation, and its graph cache under two
threads (GPU)."""
import ctypes as ct
import threading

import numpy as np
import pytest
import torch

from dynlplus_b200 import _lib, backend, graphs, kernels, solvers, stream
from dynlplus_b200.backend import code, ld, ptr
from oracle import ref_np as O

pytestmark = pytest.mark.gpu


def _problem(C, dtype=torch.float64, n=5000, seed=4):
    """A resident graph with inert entries (labelled and ungrounded rows, deleted edges, slack) and
    a random right-hand side on its solved rows; R = rhs for Z = 0."""
    ds = graphs.er_graph(n, 8, 3, weights="lognormal", seed=seed)
    lab = graphs.label_mask(n, 0.03, seed=seed)
    es = stream.EdgeStream(ds, lab)
    es.apply_edges(**graphs.EdgeUpdates(ds.A, seed=seed, weights="lognormal").next(600))
    s = es.system.astype(dtype)
    rs = np.random.RandomState(seed)
    solved = s.solved.cpu().numpy()
    rhs = torch.as_tensor(rs.random_sample((n, C)) * solved[:, None], dtype=dtype).cuda()
    return es, s, rhs


def _oracle_graph(es):
    """The slot graph as SciPy CSR with its inert entries kept (stored entries = edge visits)."""
    return es.G.to_csr("w", drop_zero=False).to_scipy().astype(np.float64)


def _cand(R, diag, eps):
    eps_d = torch.as_tensor(eps, dtype=torch.float64, device=R.device)
    return kernels.flatnonzero(kernels.violating(R, diag, eps_d))


def _residual_of(es, s, Z, rhs):
    Wf = es.G.to_csr("w").to_scipy().astype(np.float64)
    d = s.diag.double().cpu().numpy()
    Zn = Z.double().cpu().numpy()
    return rhs.double().cpu().numpy() - (d[:, None] * Zn - Wf @ Zn)


@pytest.mark.parametrize("C", [1, 3, 9, 17, 33])
def test_fused_push_rounds_match_synchronous_push(C):
    """fp64: the same number of rounds, the same frontier sizes round by round (their totals), the
    same edge visits, and Z, R equal up to the order of the atomic sums."""
    es, s, rhs = _problem(C)
    diag = s.diag
    Z = torch.zeros_like(rhs)
    R = rhs.clone()
    eps = [3e-4] * C
    cand = _cand(R, diag, eps)
    fp = kernels.FusedPush(es.G, C)
    rounds, ok, edges = fp.run(Z, R, diag, eps, cand, 100_000)
    nr, frontier_rows, touched_rows, edges2 = fp.counts()
    Wo = _oracle_graph(es)
    Zo, Ro, conv, it, rec = O.push(Wo, diag.cpu().numpy(), np.zeros((es.n, C)), rhs.cpu().numpy(), eps, record=True)
    assert conv and ok
    assert rounds == it == nr, (rounds, it)
    assert frontier_rows == sum(len(c) for c, _ in rec)
    assert edges == edges2 == sum(int((Wo.indptr[c + 1] - Wo.indptr[c]).sum()) for c, _ in rec)
    assert touched_rows >= max(len(t) for _, t in rec) - max(len(c) for c, _ in rec)
    np.testing.assert_allclose(Z.cpu().numpy(), Zo, rtol=0, atol=1e-12 * max(1.0, np.abs(Zo).max()))
    np.testing.assert_allclose(R.cpu().numpy(), Ro, rtol=0, atol=1e-13 * max(1.0, np.abs(rhs.cpu().numpy()).max()))


@pytest.mark.parametrize("C", [4, 9])
def test_fused_push_fp32_vector_rows(C):
    """fp32 rows padded to 16 bytes take the vector-atomic path; the kept residual is the true one
    up to fp32 rounding, every row meets eps at the end, and padding columns are never written."""
    es, s, rhs = _problem(C, torch.float32)
    G = es.G
    n = es.n
    ldp = (C + 3) // 4 * 4
    Zb = torch.zeros((n, ldp), dtype=torch.float32, device="cuda")
    Rb = torch.zeros((n, ldp), dtype=torch.float32, device="cuda")
    Z, R = Zb[:, :C], Rb[:, :C]
    R.copy_(rhs)
    Rb[:, C:] = 7.0
    eps = [1e-4] * C
    cand = _cand(R, s.diag, eps)
    rounds, ok, edges = kernels.FusedPush(G, C).run(Z, R, s.diag, eps, cand, 100_000)
    assert ok and rounds > 0
    assert bool((Rb[:, C:] == 7.0).all())
    Rt = _residual_of(es, s, Z, rhs)
    # the true residual diag Z - W Z of fp32 scores is known to a few ulps of |Z| * 2 max(diag)
    d = s.diag.double().cpu().numpy()
    floor = 8 * 2.0 ** -24 * float(Z.abs().max()) * 2 * float(d.max())
    np.testing.assert_allclose(R.double().cpu().numpy(), Rt, rtol=0, atol=floor)
    assert (np.abs(Rt) / d[:, None]).max() <= 1e-4 + floor / float(d.min())


def test_fused_push_round_cap_returns_cap():
    """max_rounds = 2 with rows still violating: DLP_ERR_CAP, two rounds, and R is still the residual
    of Z (no residual was taken without being pushed)."""
    C = 3
    es, s, rhs = _problem(C)
    Z, R = torch.zeros_like(rhs), rhs.clone()
    eps = [1e-7] * C
    cand = _cand(R, s.diag, eps)
    G = es.G
    ws = backend.workspace("push_cap").get(_lib.lib().dlp_fused_push_workspace_bytes(es.n, C))
    rounds, conv, edges = ct.c_int32(0), ct.c_int32(0), ct.c_ulonglong(0)
    eps_h = (ct.c_double * C)(*eps)
    st = _lib.lib().dlp_fused_push(ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(G.data), code(G.data), es.n, C,
                                   ptr(s.diag), ptr(Z), ld(Z), ptr(R), ld(R), code(Z), eps_h, ptr(cand),
                                   int(cand.numel()), 2, 8, 1, ptr(ws), ws.numel(), ct.byref(rounds), ct.byref(conv),
                                   ct.byref(edges), backend.stream())
    assert st == _lib.DLP_ERR_CAP, _lib.STATUS.get(st)
    assert rounds.value == 2 and conv.value == 0 and edges.value > 0
    np.testing.assert_allclose(R.cpu().numpy(), _residual_of(es, s, Z, rhs), atol=1e-13)
    # the Python wrapper reports the capped run as not converged, like the reference's FusedPush.run
    Z2, R2 = torch.zeros_like(rhs), rhs.clone()
    r2, ok2, _ = kernels.FusedPush(G, C).run(Z2, R2, s.diag, eps, cand, 2, use_graph=False)
    assert r2 == 2 and not ok2


def test_pcg_iteration_cap_returns_cap():
    """dlp_pcg with max_iter = 2: DLP_ERR_CAP with status 3 and the iterate of two iterations, in
    the device-side loop and in the host-driven one."""
    n, K = 20_000, 4
    ds = graphs.er_graph(n, 10, K, seed=5)
    lab = graphs.label_mask(n, 0.01, seed=5)
    S = stream.EdgeStream(ds, lab).system
    C = S.rhs.shape[1]
    Z = solvers.padded_empty(n, C, torch.float32, "cuda", fill=0.0)
    R = torch.empty((n, C), dtype=torch.float32, device="cuda")
    P = solvers.padded_empty(n, C, torch.float32, "cuda")
    AP = solvers.padded_empty(n, C, torch.float32, "cuda")
    rhs = S.rhs.contiguous()
    ws = backend.workspace("pcg_cap").get(_lib.lib().dlp_pcg_workspace_bytes(C))
    it, viol, rel, status = ct.c_int32(0), ct.c_double(0), ct.c_double(0), ct.c_int32(0)
    eps_h = (ct.c_double * C)(*([1e-9] * C))
    W = S.W
    for graph in (1, 0):
        Z.zero_()
        st = _lib.lib().dlp_pcg(ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(W.data), code(W.data), n, C,
                                ptr(S.diag), ptr(rhs), ld(rhs), ptr(Z), ld(Z), ptr(R), ld(R), ptr(P), ld(P), ptr(AP),
                                ld(AP), code(Z), eps_h, None, 0.0, 1, 2, 400, 8, graph, W.nnz / n, ptr(ws),
                                ws.numel(), ct.byref(it), ct.byref(viol), ct.byref(rel), ct.byref(status),
                                backend.stream(), None, None, 0)
        assert st == _lib.DLP_ERR_CAP and status.value == 3 and it.value == 2, (st, status.value, it.value)
        assert float(Z.abs().sum()) > 0


def test_cancel_word_stops_pcg_and_push():
    """A set cancel word stops the PCG at its first stop decision and the push after its first
    round: both raise Cancelled and leave consistent outputs; with the word cleared they run to
    the end."""
    word = torch.ones(1, dtype=torch.int32, device="cuda")
    n, K = 20_000, 4
    ds = graphs.er_graph(n, 10, K, seed=6)
    lab = graphs.label_mask(n, 0.01, seed=6)
    S = stream.EdgeStream(ds, lab).system
    C = S.rhs.shape[1]
    Z = solvers.padded_empty(n, C, torch.float32, "cuda", fill=0.0)
    backend.set_cancel_word(word)
    try:
        with pytest.raises(_lib.Cancelled):
            solvers.pcg(S, Z, S.rhs, [1e-9] * C, solvers.jacobi_M(S), 10_000, solvers.Stats())
        es, s, rhs = _problem(3)
        Zp, Rp = torch.zeros_like(rhs), rhs.clone()
        eps = [1e-6] * 3
        with pytest.raises(_lib.Cancelled):
            kernels.FusedPush(es.G, 3).run(Zp, Rp, s.diag, eps, _cand(Rp, s.diag, eps), 100_000)
        np.testing.assert_allclose(Rp.cpu().numpy(), _residual_of(es, s, Zp, rhs), atol=1e-13)
        word.zero_()
        st = solvers.Stats()
        solvers.pcg(S, Z, S.rhs, [1e-6] * C, solvers.jacobi_M(S), 10_000, st)
        assert st.iters > 2
        rounds, ok, _ = kernels.FusedPush(es.G, 3).run(Zp, Rp, s.diag, eps, _cand(Rp, s.diag, eps), 100_000)
        assert ok
    finally:
        backend.set_cancel_word(None)


def test_push_graph_cache_two_threads():
    """Two threads push 20 distinct problems each (40 cached loop graphs for a cache of 32, so
    entries are evicted while the other thread replays its graphs): every run converges and keeps
    its residual exact."""
    C = 3
    es, s, rhs = _problem(C)
    eps = [1e-5] * C
    errors = []

    def worker(k):
        try:
            torch.cuda.set_device(0)
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                for i in range(20):
                    Z = torch.zeros_like(rhs)  # fresh buffers: a new problem signature each time
                    R = (rhs * (1.0 + 0.1 * i + k)).contiguous()
                    cand = _cand(R, s.diag, eps)
                    rounds, ok, _ = kernels.FusedPush(es.G, C).run(Z, R, s.diag, eps, cand, 100_000)
                    st.synchronize()
                    if not ok:
                        errors.append((k, i, "not converged"))
                    Rt = _residual_of(es, s, Z, rhs * (1.0 + 0.1 * i + k))
                    if np.abs(Rt - R.cpu().numpy()).max() > 1e-12:
                        errors.append((k, i, "residual drift"))
                    del Z, R
        except Exception as e:  # noqa: BLE001 - reported on the main thread
            errors.append((k, repr(e)))

    th = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errors, errors

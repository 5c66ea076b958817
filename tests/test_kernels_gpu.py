"""Row kernels (SpMM, frontier Jacobi, push scatter, marking, compaction, reductions) against the
reference's outputs (golden fixtures) and the oracle, through the C ABI (GPU)."""
import numpy as np
import pytest
import scipy.sparse as ssp
import torch

from conftest import golden_csr, load_golden
from dynlplus_b200 import _lib, kernels
from dynlplus_b200.backend import CSR
from oracle import ref_np as O

pytestmark = pytest.mark.gpu

TOL = {torch.float32: 1e-5, torch.float64: 1e-12}  # the reference's kernel-test tolerances (test_dynlp.py:209)


def T(x, dt=None, dev="cuda"):
    t = torch.as_tensor(np.ascontiguousarray(x))
    return (t.to(dt) if dt is not None else t).to(dev)


def padded(X, ld, dt):
    """X (n x C) stored in an n x ld buffer (a column view) so the vector-gather path is taken."""
    buf = torch.full((X.shape[0], ld), float("nan"), dtype=dt, device="cuda")
    buf[:, : X.shape[1]] = T(X, dt)
    return buf[:, : X.shape[1]]


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
@pytest.mark.parametrize("C", [1, 3, 9, 17])
@pytest.mark.parametrize("gs", ["auto", 1, 2, 8, 32, 128])
def test_frontier_ops_match_reference(dt, C, gs):
    g = load_golden("kernels.npz")
    A = golden_csr(g, "W")
    W = CSR.from_scipy(A, dtype=dt)
    f, diag = T(g["frontier"]), T(g["diag"], dt)
    X, rhs, D = T(g[f"C{C}_X"], dt), T(g[f"C{C}_rhs"], dt), T(g[f"C{C}_D"], dt)
    ops = kernels.FrontierOps(W, C, gs)
    Y, ch = ops.jacobi(f, X, rhs, diag, 1e-2)
    tol = TOL[dt]
    np.testing.assert_allclose(Y.cpu().numpy(), g[f"C{C}_jacY"], rtol=tol, atol=tol)
    # change flags are exact away from the threshold (float32 rounding can move |Y-X| across it)
    far = np.abs(np.abs(g[f"C{C}_jacY"] - g[f"C{C}_X"][g["frontier"]]) - 1e-2).min(axis=1) > 1e-4
    np.testing.assert_array_equal(ch.cpu().numpy()[far], g[f"C{C}_jacch"].astype(bool)[far])
    R = torch.zeros((A.shape[0], C), dtype=dt, device="cuda")
    mark = torch.zeros(A.shape[0], dtype=torch.uint8, device="cuda")
    ops.push(f, D, R, mark)
    np.testing.assert_allclose(R.cpu().numpy(), g[f"C{C}_pushR"], rtol=tol, atol=1e-5 if dt == torch.float32 else 1e-12)
    np.testing.assert_array_equal(mark.cpu().numpy(), g[f"C{C}_pushmark"])
    mark.zero_()
    ops.mark_neighbors(f, mark)
    np.testing.assert_array_equal(mark.cpu().numpy(), g[f"C{C}_marknb"])
    assert int(ops.edges) == int(g[f"C{C}_edges"])


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
@pytest.mark.parametrize("C", [2, 3, 9, 17])
@pytest.mark.parametrize("ld_pad", [0, 4])
def test_spmm_matches_reference(dt, C, ld_pad):
    g = load_golden("kernels.npz")
    Cg = {2: 3}.get(C, C)
    A = golden_csr(g, "W")
    W = CSR.from_scipy(A, dtype=dt)
    Xn = g[f"C{Cg}_X"][:, :C]
    a = g[f"C{Cg}_a"]
    X = padded(Xn, ((C + 3) // 4) * 4 + ld_pad, dt) if ld_pad else T(Xn, dt)
    tol = TOL[dt]
    np.testing.assert_allclose(kernels.spmm_axpy(W, X).cpu().numpy(), A @ Xn, rtol=tol, atol=tol)
    Y = kernels.spmm_axpy(W, X, a=T(a, dt), b=-1.0)
    np.testing.assert_allclose(Y.cpu().numpy(), a[:, None] * Xn - A @ Xn, rtol=tol, atol=tol)
    if C == Cg:
        np.testing.assert_allclose(Y.cpu().numpy(), g[f"C{C}_applyA"], rtol=tol, atol=tol)


@pytest.mark.parametrize("C", [1, 5, 9, 33, 40, 100])
def test_spmm_widths_and_fp64_residual(C):
    """Every lane layout (row map, class-parallel map, 8 vectors per lane) and the fp64 residual
    over fp32-stored weights: R = rhs - diag*X + W X."""
    rs = np.random.RandomState(C)
    A = O.symmetric_from_pairs(rs.randint(0, 4000, 40000), rs.randint(0, 4000, 40000), rs.rand(40000), 4000,
                               np.float32)
    W = CSR.from_scipy(A)
    X, rhs, d = rs.rand(4000, C), rs.rand(4000, C), rs.rand(4000) + 1
    want = rhs - d[:, None] * X + A.astype(np.float64) @ X
    got = kernels.spmm_axpy(W, T(X), a=T(d), alpha=-1.0, b=1.0, rhs=T(rhs))
    assert got.dtype == torch.float64
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-12, atol=1e-12)
    got32 = kernels.spmm_axpy(W, T(X, torch.float32))
    np.testing.assert_allclose(got32.cpu().numpy(), A @ X.astype(np.float32), rtol=2e-5, atol=2e-5)


@pytest.mark.parametrize("C", [9, 10])
@pytest.mark.parametrize("ld_x,ld_r,ld_y", [(10, 10, 10), (16, 0, 12), (10, 11, 0), (12, 10, 14)])
def test_spmm_fp64_whole_rows(C, ld_x, ld_r, ld_y):
    """fp64 rows of 9-10 values (one lane per row, three loads; the own row and the rhs row read whole
    and the output written in vector stores where their rows are padded and 16-byte aligned; ld 0 =
    unpadded, odd ld = unaligned rows) against numpy: full rows, a row subset in place, compact rows.
    Columns of the output beyond C keep their values."""
    rs = np.random.RandomState(C * 100 + ld_x + ld_r + ld_y)
    n = 3001
    A = O.symmetric_from_pairs(rs.randint(0, n, 30000), rs.randint(0, n, 30000), rs.rand(30000), n, np.float32)
    W = CSR.from_scipy(A)
    X, rhs, d = rs.rand(n, C), rs.rand(n, C), rs.rand(n) + 1
    Xd = padded(X, ld_x, torch.float64)  # NaN in the padding: never read into a result
    rhs_d = padded(rhs, ld_r, torch.float64) if ld_r else T(rhs)
    want = rhs - d[:, None] * X + A.astype(np.float64) @ X

    def out_buf():
        if not ld_y:
            return T(np.zeros((n, C)))
        buf = torch.full((n, ld_y), -7.0, dtype=torch.float64, device="cuda")
        buf[:, :C] = 0.0
        return buf[:, :C]

    Y = out_buf()
    kernels.spmm_axpy(W, Xd, a=T(d), alpha=-1.0, b=1.0, rhs=rhs_d, out=Y)
    np.testing.assert_allclose(Y.cpu().numpy(), want, rtol=1e-12, atol=1e-12)
    if ld_y:
        assert (Y.as_strided((n, ld_y), (ld_y, 1))[:, C:] == -7.0).all()
    Q = np.sort(rs.choice(n, 400, replace=False)).astype(np.int32)
    Y = out_buf()
    kernels.spmm_axpy(W, Xd, a=T(d), alpha=-1.0, b=1.0, rhs=rhs_d, out=Y, rows=T(Q))
    Yn = Y.cpu().numpy()
    np.testing.assert_allclose(Yn[Q], want[Q], rtol=1e-12, atol=1e-12)
    assert (Yn[np.setdiff1d(np.arange(n), Q)] == 0).all()
    Yc = kernels.spmm_axpy(W, Xd, rows=T(Q), compact=True)
    np.testing.assert_allclose(Yc.cpu().numpy(), (A.astype(np.float64) @ X)[Q], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n,C", [(1, 1), (1000, 9), (300_001, 9), (50, 300)])
def test_cols_scale_all_ops(n, C):
    """dlp_cols_scale, op 0 Y = X / s, 1 Y += X s, 2 Y = X s, 3 Y = X + Y s, for every precision pair,
    on padded rows; columns beyond C untouched."""
    rs = np.random.RandomState(n + C)
    X, Y0, sc = rs.rand(n, C) - 0.5, rs.rand(n, C) - 0.5, rs.rand(C) + 0.5
    ops = {0: lambda x, y: x / sc, 1: lambda x, y: y + x * sc, 2: lambda x, y: x * sc, 3: lambda x, y: x + y * sc}
    pairs = [(torch.float64, torch.float32), (torch.float32, torch.float64), (torch.float64, torch.float64),
             (torch.float32, torch.float32)]
    s_d = T(sc)
    for tx, ty in pairs:
        Xd = padded(X, C + 3, tx)
        xw = Xd.double().cpu().numpy()
        for op, f in ops.items():
            buf = torch.full((n, C + 5), 9.0, dtype=ty, device="cuda")
            buf[:, :C] = T(Y0, ty)
            Yd = buf[:, :C]
            yw = Yd.double().cpu().numpy()
            _lib.call("dlp_cols_scale", n, C, Xd.data_ptr(), Xd.stride(0), _lib_code(tx), s_d.data_ptr(), op,
                      Yd.data_ptr(), Yd.stride(0), _lib_code(ty), torch.cuda.current_stream().cuda_stream)
            tol = 1e-6 if torch.float32 in (tx, ty) else 1e-14
            np.testing.assert_allclose(Yd.double().cpu().numpy(), f(xw, yw), rtol=tol, atol=tol)
            assert (buf[:, C:] == 9.0).all()
    Xd = padded(X, C + 3, torch.float32)
    Yb = torch.zeros((n, C), dtype=torch.bfloat16, device="cuda")
    _lib.call("dlp_cols_scale", n, C, Xd.data_ptr(), Xd.stride(0), _lib_code(torch.float32), s_d.data_ptr(), 2,
              Yb.data_ptr(), Yb.stride(0), _lib_code(torch.bfloat16), torch.cuda.current_stream().cuda_stream)
    np.testing.assert_allclose(Yb.double().cpu().numpy(), Xd.double().cpu().numpy() * sc, rtol=1e-2, atol=1e-2)


def _lib_code(dt):
    from dynlplus_b200.backend import DTYPES
    return DTYPES[dt]


def test_spmm_bf16_fp32_accumulation():
    rs = np.random.RandomState(3)
    A = O.symmetric_from_pairs(rs.randint(0, 3000, 30000), rs.randint(0, 3000, 30000), rs.rand(30000), 3000,
                               np.float32)
    W = CSR.from_scipy(A, dtype=torch.bfloat16)
    for C in (4, 9, 16, 17):
        X = T(rs.rand(3000, C), torch.bfloat16)
        Wb = W.data.float().cpu().numpy()
        Ab = ssp.csr_matrix((Wb.astype(np.float64), A.indices, A.indptr), shape=A.shape)
        want = Ab @ X.float().cpu().numpy().astype(np.float64)
        got = kernels.spmm_axpy(W, X)
        assert got.dtype == torch.float32
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-5, atol=1e-5)
        gotb = kernels.spmm_axpy(W, X, out_dtype=torch.bfloat16)
        np.testing.assert_allclose(gotb.float().cpu().numpy(), want, rtol=1e-2, atol=1e-2)


def test_spmm_row_subset_in_place_and_compact():
    rs = np.random.RandomState(4)
    A = O.symmetric_from_pairs(rs.randint(0, 2000, 20000), rs.randint(0, 2000, 20000), rs.rand(20000), 2000,
                               np.float64)
    W = CSR.from_scipy(A)
    X, rhs, d = rs.rand(2000, 5), rs.rand(2000, 5), rs.rand(2000) + 1
    Q = np.sort(rs.choice(2000, 300, replace=False)).astype(np.int32)
    R = T(np.zeros((2000, 5)))
    kernels.spmm_axpy(W, T(X), a=T(d), alpha=-1.0, rhs=T(rhs), rows=T(Q), out=R)
    full = rhs - d[:, None] * X + A @ X
    Rn = R.cpu().numpy()
    np.testing.assert_allclose(Rn[Q], full[Q], rtol=1e-12)
    other = np.setdiff1d(np.arange(2000), Q)
    assert (Rn[other] == 0).all()
    Yc = kernels.spmm_axpy(W, T(X), rows=T(Q), compact=True)
    np.testing.assert_allclose(Yc.cpu().numpy(), (A @ X)[Q], rtol=1e-12)


def test_frontier_jacobi_compaction_list():
    rs = np.random.RandomState(5)
    A = O.symmetric_from_pairs(rs.randint(0, 5000, 50000), rs.randint(0, 5000, 50000), rs.rand(50000), 5000,
                               np.float64)
    W = CSR.from_scipy(A)
    X, rhs = rs.rand(5000, 3), rs.rand(5000, 3)
    diag = A @ np.ones(5000) + 1
    f = np.sort(rs.choice(5000, 2000, replace=False)).astype(np.int32)
    out, cnt = torch.empty(5000, dtype=torch.int32, device="cuda"), torch.zeros(1, dtype=torch.int32, device="cuda")
    ops = kernels.FrontierOps(W, 3)
    Y, ch = ops.jacobi(T(f), T(X), T(rhs), T(diag), 0.05, out_list=out, out_count=cnt)
    Yo, cho = O.frontier_jacobi(A, f, X, rhs, diag, 0.05)
    np.testing.assert_array_equal(ch.cpu().numpy(), cho)
    got = np.sort(out[: int(cnt.item())].cpu().numpy())
    np.testing.assert_array_equal(got, f[cho])


@pytest.mark.parametrize("n", [0, 1, 7, 2047, 2048, 2049, 100_000, 3_000_001])
def test_flatnonzero(n):
    rs = np.random.RandomState(n % 1000)
    flag = (rs.rand(n) < 0.3).astype(np.uint8)
    got = kernels.flatnonzero(T(flag))
    np.testing.assert_array_equal(got.cpu().numpy(), np.flatnonzero(flag))
    if n:
        idx = rs.permutation(n).astype(np.int32)
        got = kernels.flatnonzero(T(flag), idx=T(idx))
        np.testing.assert_array_equal(got.cpu().numpy(), idx[np.flatnonzero(flag)])


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_colreduce(dt):
    rs = np.random.RandomState(6)
    for n, C in ((1, 1), (257, 3), (100_003, 9), (300_000, 33)):
        X, Y, d = rs.randn(n, C), rs.randn(n, C), rs.rand(n) + 0.5
        mask = (rs.rand(n) < 0.5).astype(np.uint8)
        Xt, Yt, dt_ = T(X, dt), T(Y, dt), T(d, dt)
        Xc, Yc, dc = Xt.double().cpu().numpy(), Yt.double().cpu().numpy(), dt_.double().cpu().numpy()
        np.testing.assert_allclose(kernels.colreduce(0, Xt, diag=dt_).cpu().numpy(),
                                   (np.abs(Xc) / dc[:, None]).max(0), rtol=1e-15)
        np.testing.assert_allclose(kernels.colreduce(1, Xt, Y=Yt).cpu().numpy(), (Xc * Yc).sum(0), rtol=1e-10,
                                   atol=1e-10)
        np.testing.assert_allclose(kernels.colreduce(2, Xt).cpu().numpy(), (Xc * Xc).sum(0), rtol=1e-12)
        m = mask.astype(bool)
        want = np.abs(Xc[m]).max(0) if m.any() else np.zeros(C)
        np.testing.assert_allclose(kernels.colreduce(3, Xt, mask=T(mask)).cpu().numpy(), want, rtol=0)
        # deterministic: same bits twice
        a = kernels.colreduce(1, Xt, Y=Yt).cpu().numpy()
        b = kernels.colreduce(1, Xt, Y=Yt).cpu().numpy()
        assert (a == b).all()


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_push_take_and_violating(dt):
    rs = np.random.RandomState(7)
    n, C = 3000, 4
    Z, R, d = rs.rand(n, C), rs.randn(n, C) * 1e-3, rs.rand(n) + 1
    cand = np.sort(rs.choice(n, 500, replace=False)).astype(np.int32)
    Zt, Rt, dt_ = T(Z, dt), T(R, dt), T(d, dt)
    D = torch.empty((500, C), dtype=dt, device="cuda")
    mark = torch.zeros(n, dtype=torch.uint8, device="cuda")
    kernels.push_take(T(cand), Zt, Rt, dt_, D, mark)
    Zc, Rc, dc = Z.astype(np.float64), R.astype(np.float64), d.astype(np.float64)
    if dt == torch.float32:
        Zc, Rc, dc = Z.astype(np.float32), R.astype(np.float32), d.astype(np.float32)
    Dw = Rc[cand] / dc[cand][:, None]
    Zc[cand] += Dw
    Rc[cand] = 0
    np.testing.assert_array_equal(D.cpu().numpy(), Dw)
    np.testing.assert_array_equal(Zt.cpu().numpy(), Zc)
    np.testing.assert_array_equal(Rt.cpu().numpy(), Rc)
    assert mark.cpu().numpy()[cand].all() and mark.sum().item() == 500
    eps = np.array([1e-4, 2e-4, 5e-4, 1e-3])
    fl = kernels.violating(Rt, dt_, T(eps))
    epsd = eps.astype(Rc.dtype)
    want = (np.abs(Rc) > epsd[None, :] * dc[:, None]).any(axis=1)
    np.testing.assert_array_equal(fl.cpu().numpy().astype(bool), want)


def test_invalid_arguments_raise():
    A = O.symmetric_from_pairs(np.array([0]), np.array([1]), np.ones(1), 4, np.float32)
    # 1100 fp32 columns = 275 vectors: beyond 32 vector lanes x 8 vectors per lane
    with pytest.raises(_lib.DLPError):
        kernels.spmm_axpy(CSR.from_scipy(A), T(np.zeros((4, 1100), np.float32)))
    # 300 columns fit (75 vectors) and are exact
    X = np.random.RandomState(0).rand(4, 300).astype(np.float32)
    np.testing.assert_allclose(kernels.spmm_axpy(CSR.from_scipy(A), T(X)).cpu().numpy(), A @ X, rtol=1e-6)


@pytest.mark.parametrize("C", [3, 9, 16])
def test_spmm_lowp_whole_bf16_rows(C):
    """dlp_spmm_lowp, the SpMM of the BF16 sweeps: Y = a*X_own - W X_lo with bf16 weights and gathered
    rows and fp32 accumulation, own row and output. Rows of 16 bf16 values (ld 16, 32 bytes) are
    gathered whole by one 256-bit load; against the same product in fp64 of the bf16 values."""
    from dynlplus_b200.backend import ld, ptr, stream
    from dynlplus_b200.solvers import padded_empty
    rs = np.random.RandomState(C)
    n = 5000
    A = O.symmetric_from_pairs(rs.randint(0, n, 60000), rs.randint(0, n, 60000), rs.rand(60000) + 0.1, n,
                               np.float32)
    W = CSR.from_scipy(A, dtype=torch.float32)
    wb = W.data.to(torch.bfloat16)
    X = T(rs.rand(n, C) - 0.5, torch.float32)
    Xo = padded_empty(n, C, torch.float32, "cuda")
    Xo.copy_(X)
    Xl = torch.zeros((n, 16), dtype=torch.bfloat16, device="cuda")[:, :C]  # 32-byte rows
    Xl.copy_(X)
    a = T(rs.rand(n) + 1.0, torch.float32)
    Ab = ssp.csr_matrix((wb.float().cpu().numpy().astype(np.float64), A.indices, A.indptr), shape=A.shape)
    want = a.double().cpu().numpy()[:, None] * X.double().cpu().numpy() - Ab @ Xl.float().double().cpu().numpy()
    buf = torch.full((n, 16), -7.0, dtype=torch.float32, device="cuda")  # output rows of 16-byte pitch
    for Y in (torch.empty((n, C), dtype=torch.float32, device="cuda"), buf[:, :C]):
        for rep in range(2):
            _lib.call("dlp_spmm_lowp", ptr(W.rbeg), ptr(W.rend), ptr(W.indices), ptr(wb), n, C, ptr(Xl), ld(Xl),
                      ptr(Xo), ld(Xo), ptr(a), 1.0, -1.0, ptr(Y), ld(Y), 0, W.nnz / n, stream())
        np.testing.assert_allclose(Y.double().cpu().numpy(), want, rtol=1e-5, atol=1e-5 * np.abs(want).max())
    assert (buf[:, C:] == -7.0).all()


@pytest.mark.parametrize("C", [9, 10, 11, 12])
@pytest.mark.parametrize("ld_x,ld_y", [(12, 12), (16, 16), (12, 0), (12, 13)])
def test_spmm_fp32_whole_row_epilogue(C, ld_x, ld_y):
    """fp32 rows of 9-12 values gathered whole (two loads per row): the own row of the diagonal term
    read whole and the output written in vector stores of exactly its C values where the rows are
    16-byte aligned (ld 0 = unpadded, odd ld = unaligned rows), against numpy: full rows, a row subset
    in place, compact rows. Columns of the output beyond C keep their values; the results are the
    same values as the per-column epilogue's (same FMAs in the same order)."""
    rs = np.random.RandomState(C * 100 + ld_x + ld_y)
    n = 3001
    A = O.symmetric_from_pairs(rs.randint(0, n, 30000), rs.randint(0, n, 30000), rs.rand(30000), n, np.float32)
    W = CSR.from_scipy(A, dtype=torch.float32)
    X, d = rs.rand(n, C).astype(np.float32), (rs.rand(n) + 1).astype(np.float32)
    Xd = padded(X, ld_x, torch.float32)  # NaN in the padding: never read into a result
    want = d[:, None].astype(np.float64) * X - A.astype(np.float64) @ X.astype(np.float64)

    def out_buf():
        if not ld_y:
            return torch.zeros((n, C), dtype=torch.float32, device="cuda")
        buf = torch.full((n, ld_y), -7.0, dtype=torch.float32, device="cuda")
        buf[:, :C] = 0.0
        return buf[:, :C]

    Y = out_buf()
    kernels.spmm_axpy(W, Xd, a=T(d), b=-1.0, out=Y)
    np.testing.assert_allclose(Y.cpu().numpy(), want, rtol=1e-5, atol=1e-5 * np.abs(want).max())
    if ld_y:
        assert (Y.as_strided((n, ld_y), (ld_y, 1))[:, C:] == -7.0).all()
    Yu = kernels.spmm_axpy(W, T(X), a=T(d), b=-1.0)  # unpadded X and Y: the per-column epilogue
    assert torch.equal(Y, Yu) or np.abs(Y.cpu().numpy() - Yu.cpu().numpy()).max() <= 1e-5 * np.abs(want).max()
    Q = np.sort(rs.choice(n, 400, replace=False)).astype(np.int32)
    Y = out_buf()
    kernels.spmm_axpy(W, Xd, a=T(d), b=-1.0, out=Y, rows=T(Q))
    Yn = Y.cpu().numpy()
    np.testing.assert_allclose(Yn[Q], want[Q], rtol=1e-5, atol=1e-5 * np.abs(want).max())
    assert (Yn[np.setdiff1d(np.arange(n), Q)] == 0).all()
    Yc = kernels.spmm_axpy(W, Xd, rows=T(Q), compact=True)
    np.testing.assert_allclose(Yc.cpu().numpy(), (A.astype(np.float64) @ X.astype(np.float64))[Q], rtol=1e-5,
                               atol=1e-5 * np.abs(want).max())


@pytest.mark.parametrize("C", [5, 7, 8])
@pytest.mark.parametrize("ld_x,ld_y", [(8, 8), (16, 16), (8, 0), (8, 9), (9, 8)])
def test_spmm_fp32_8float_rows(C, ld_x, ld_y):
    """fp32 rows of 5-8 values on a 32-byte pitch gathered whole (one 256-bit load per row): the own
    row of the diagonal term read whole and, for 8 columns on a 32-byte pitch, the output written as a
    whole row; odd pitches take the per-column path. Against numpy: full rows, a row subset in place,
    compact rows. Output columns beyond C keep their values; the results equal the per-column path's."""
    rs = np.random.RandomState(C * 100 + ld_x + ld_y)
    n = 3001
    A = O.symmetric_from_pairs(rs.randint(0, n, 30000), rs.randint(0, n, 30000), rs.rand(30000), n, np.float32)
    W = CSR.from_scipy(A, dtype=torch.float32)
    X, d = rs.rand(n, C).astype(np.float32), (rs.rand(n) + 1).astype(np.float32)
    Xd = padded(X, ld_x, torch.float32)  # NaN in the padding: never read into a result
    want = d[:, None].astype(np.float64) * X - A.astype(np.float64) @ X.astype(np.float64)
    tol = 1e-5 * np.abs(want).max()

    def out_buf():
        if not ld_y:
            return torch.zeros((n, C), dtype=torch.float32, device="cuda")
        buf = torch.full((n, ld_y), -7.0, dtype=torch.float32, device="cuda")
        buf[:, :C] = 0.0
        return buf[:, :C]

    Y = out_buf()
    kernels.spmm_axpy(W, Xd, a=T(d), b=-1.0, out=Y)
    np.testing.assert_allclose(Y.cpu().numpy(), want, rtol=1e-5, atol=tol)
    if ld_y:
        assert (Y.as_strided((n, ld_y), (ld_y, 1))[:, C:] == -7.0).all()
    Yu = kernels.spmm_axpy(W, padded(X, 9, torch.float32), a=T(d), b=-1.0)  # odd pitch: per-column path
    assert np.abs(Y.cpu().numpy() - Yu.cpu().numpy()).max() <= tol
    Q = np.sort(rs.choice(n, 400, replace=False)).astype(np.int32)
    Y = out_buf()
    kernels.spmm_axpy(W, Xd, a=T(d), b=-1.0, out=Y, rows=T(Q))
    Yn = Y.cpu().numpy()
    np.testing.assert_allclose(Yn[Q], want[Q], rtol=1e-5, atol=tol)
    assert (Yn[np.setdiff1d(np.arange(n), Q)] == 0).all()
    Yc = kernels.spmm_axpy(W, Xd, rows=T(Q), compact=True)
    np.testing.assert_allclose(Yc.cpu().numpy(), (A.astype(np.float64) @ X.astype(np.float64))[Q], rtol=1e-5,
                               atol=tol)
    Yc2 = kernels.spmm_axpy(W, T(X), rows=T(Q), compact=True)  # unpadded rows: the per-column path
    assert np.abs(Yc.cpu().numpy() - Yc2.cpu().numpy()).max() <= tol

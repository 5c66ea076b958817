"""The allocation-free column reduction, dlp_colreduce_noalloc (GPU).

It exists for callers that cannot allocate device memory when they need a reduction: a serving
process that reserved all of HBM for its own pool up front, a host runtime bridged through an FFI
without a device allocator, or code that must not pay the implicit synchronisation an allocation
can cause. It keeps its partial sums in a fixed array inside the library (up to 64 columns) rather
than in a caller workspace. Called through the C ABI, it must return what the workspace version
dlp_colreduce returns, on two calls in a row, and refuse wider inputs with a clear status.
This file is named to be collected last.
"""
import numpy as np
import pytest
import torch

from dynlplus_b200 import _lib, kernels
from dynlplus_b200.backend import code, ld, ptr, stream

pytestmark = pytest.mark.gpu


def _noalloc(kind, X, Y=None, diag=None, mask=None):
    n, C = X.shape
    out = torch.full((C,), float("nan"), dtype=torch.float64, device=X.device)
    _lib.call("dlp_colreduce_noalloc", kind, n, C, ptr(X), ld(X), ptr(Y), ld(Y) if Y is not None else C, ptr(diag),
              code(X), ptr(mask), ptr(out), stream())
    return out


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_noalloc_matches_workspace_version_twice(dt):
    rs = np.random.RandomState(42)
    for call in range(2):  # the second call must not see anything of the first
        for n, C in ((1, 1), (257, 3), (100_003, 9), (300_000, 33), (50_000, 64)):
            X = torch.as_tensor(rs.randn(n, C)).to(dt).cuda()
            Y = torch.as_tensor(rs.randn(n, C)).to(dt).cuda()
            d = torch.as_tensor(rs.rand(n) + 0.5).to(dt).cuda()
            mask = torch.as_tensor((rs.rand(n) < 0.5).astype(np.uint8)).cuda()
            for kind, kw in ((0, dict(diag=d)), (1, dict(Y=Y)), (2, {}), (3, dict(mask=mask))):
                want = kernels.colreduce(kind, X, **kw).cpu().numpy()
                got = _noalloc(kind, X, **kw).cpu().numpy()
                np.testing.assert_allclose(got, want, rtol=1e-12, atol=0, err_msg=f"call {call} kind {kind} C {C}")


def test_noalloc_refuses_more_columns_than_its_scratch():
    X = torch.zeros((10, 65), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.DLPError) as e:
        _noalloc(2, X)
    assert e.value.status == 9


def _numpy_reference(kind, X, Y=None, diag=None, mask=None):
    """The reduction in fp64 NumPy, independent of the library."""
    X = X.double().cpu().numpy()
    rows = np.ones(X.shape[0], bool) if mask is None else mask.cpu().numpy().astype(bool)
    X = X[rows]
    if kind == 0:
        return (np.abs(X) / diag.double().cpu().numpy()[rows][:, None]).max(axis=0, initial=0.0)
    if kind == 1:
        return (X * Y.double().cpu().numpy()[rows]).sum(axis=0)
    if kind == 2:
        return (X * X).sum(axis=0)
    return np.abs(X).max(axis=0, initial=0.0)


@pytest.mark.parametrize("dt", [torch.float32, torch.float64])
def test_noalloc_matches_numpy_up_to_its_column_limit(dt):
    """Every kind, with and without a row mask, at the widest input the fixed scratch takes (64
    columns) and at sizes that leave partial blocks, on two calls in a row."""
    rs = np.random.RandomState(7)
    for call in range(2):
        for n, C in ((5, 64), (1_000, 64), (123_457, 64), (70_001, 17)):
            X = torch.as_tensor(rs.randn(n, C)).to(dt).cuda()
            Y = torch.as_tensor(rs.randn(n, C)).to(dt).cuda()
            d = torch.as_tensor(rs.rand(n) + 0.5).to(dt).cuda()
            mask = torch.as_tensor((rs.rand(n) < 0.3).astype(np.uint8)).cuda()
            for m in (None, mask):
                for kind, kw in ((0, dict(diag=d)), (1, dict(Y=Y)), (2, {}), (3, {})):
                    got = _noalloc(kind, X, mask=m, **kw).cpu().numpy()
                    want = _numpy_reference(kind, X, mask=m, **kw)
                    # maxima of |x| exact; |x| / d is formed as |x| * (1 / d), one rounding from
                    # NumPy's quotient; sums accumulate in fp64 in a different order
                    tol = {3: dict(rtol=0, atol=0), 0: dict(rtol=1e-15, atol=0)}.get(kind, dict(rtol=1e-10, atol=1e-10))
                    np.testing.assert_allclose(got, want, **tol, err_msg=f"call {call} n {n} kind {kind}")

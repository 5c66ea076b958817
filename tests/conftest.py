import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and libdlp.so")


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_csr(g, prefix):
    import scipy.sparse as ssp
    shape = tuple(int(x) for x in g[f"{prefix}_shape"])
    return ssp.csr_matrix((g[f"{prefix}_data"], g[f"{prefix}_indices"], g[f"{prefix}_indptr"]), shape=shape)


def direct_solve(A, rhs):
    """Reference solution of A X = rhs for the checks: sparse LU on small systems; on larger random
    graphs (where LU fill-in explodes) fp64 CG to a relative residual of 1e-14 per column."""
    import scipy.sparse.linalg as sla
    rhs = np.asarray(rhs, dtype=np.float64)
    one = rhs.ndim == 1
    R = rhs.reshape(rhs.shape[0], -1)
    if A.shape[0] <= 4000:
        X = sla.spsolve(A.tocsc(), R).reshape(R.shape)
    else:
        X = np.zeros_like(R)
        Minv = 1.0 / A.diagonal()
        M = sla.LinearOperator(A.shape, matvec=lambda v: Minv * v)
        for c in range(R.shape[1]):
            X[:, c], _ = sla.cg(A, R[:, c], rtol=1e-14, atol=0.0, maxiter=20000, M=M)
    return X[:, 0] if one else X


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def dev():
    import torch
    return torch.device("cuda", 0)

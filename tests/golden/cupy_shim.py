"""Test-only CuPy stand-in: lets the reference package (pure Python over CuPy) run on the CPU.

`install()` registers modules named `cupy`, `cupyx` and `cupyx.scipy.sparse` that forward to
NumPy / SciPy, then patches the three reference entry points that need NVRTC kernels:

* `kernels.spmm_axpy` -> SciPy `a*X + b*(W@X)` (the kernel's definition, dynlp/kernels.py:140-166);
* `kernels.FrontierOps.use_kernel` -> False after construction, so the reference's own
  vectorised fallbacks run (dynlp/kernels.py:473-474, :483-486, :492);
* `solvers.IncrementalLP._push` -> the synchronous vectorised `push` (dynlp/solvers.py:386-389),
  which is the branch the reference itself takes when the fused GPU kernel is unavailable.

Used only by `make_golden.py` in this folder to produce the committed fixtures. Nothing on the
product path imports it.
"""
from __future__ import annotations

import sys
import types

import numpy as np
import scipy.sparse as ssp


class _Device:
    def __init__(self, *_a, **_k):
        self.attributes = {"MultiProcessorCount": 8}

    def synchronize(self):
        return None


class _Pool:
    def used_bytes(self):
        return 0

    def free_all_blocks(self):
        return None


def _make_cupy():
    cp = types.ModuleType("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.ndarray = np.ndarray
    cp.asnumpy = np.asarray
    cp.get_default_memory_pool = lambda: _Pool()
    cuda = types.SimpleNamespace(Device=_Device, runtime=types.SimpleNamespace(runtimeGetVersion=lambda: 0))
    cp.cuda = cuda

    def _raw_module(*_a, **_k):
        raise RuntimeError("NVRTC kernels are not available under the CPU shim")

    cp.RawModule = _raw_module
    cp.testing = np.testing
    cp.random = np.random
    cp.linalg = np.linalg
    return cp


def _make_cupyx():
    cx = types.ModuleType("cupyx")
    cx.scatter_add = lambda a, idx, v: np.add.at(a, idx, v)
    cx.scatter_max = lambda a, idx, v: np.maximum.at(a, idx, v)
    cx.scatter_min = lambda a, idx, v: np.minimum.at(a, idx, v)
    scipy_mod = types.ModuleType("cupyx.scipy")
    scipy_mod.sparse = ssp
    cx.scipy = scipy_mod
    return cx, scipy_mod


def install(reference_root: str):
    """Register the shim and import the reference package from `reference_root`."""
    if "cupy" not in sys.modules:
        sys.modules["cupy"] = _make_cupy()
        cx, sc = _make_cupyx()
        sys.modules["cupyx"] = cx
        sys.modules["cupyx.scipy"] = sc
        sys.modules["cupyx.scipy.sparse"] = ssp
    if reference_root not in sys.path:
        sys.path.insert(0, reference_root)
    import dynlp.kernels as K
    import dynlp.solvers as S

    def spmm_axpy(W, X, a=None, b=1.0, group="auto"):
        Y = b * (W @ X)
        if a is not None:
            Y = Y + a[:, None] * X
        return np.ascontiguousarray(Y.astype(X.dtype))

    K.spmm_axpy = spmm_axpy
    orig_init = K.FrontierOps.__init__

    def ops_init(self, *a, **k):
        orig_init(self, *a, **k)
        self.use_kernel = False

    K.FrontierOps.__init__ = ops_init

    def inc_push(self, s64, eps, st):
        ops = K.FrontierOps(s64.W, self.Z.shape[1], self.group)
        ok = S.push(s64, self.Z, self.R, eps, ops, st, max_iter=self.max_rounds)[2]
        st.edges += int(ops.edges)
        return ok

    S.IncrementalLP._push = inc_push
    import dynlp
    return dynlp

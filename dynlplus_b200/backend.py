"""Device runtime: PyTorch tensors for memory and streams, libdlp for compute.

Mirrors the reference's backend module (dynlp/backend.py:1-56): `sync`, `csr`, `Timer`,
`mem_used_gb`, plus the helpers the C ABI needs (raw pointers, leading dimensions, precision
codes, the current stream and a reusable workspace).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import torch

from . import _lib

DTYPES = {torch.float32: _lib.DLP_F32, torch.float64: _lib.DLP_F64, torch.bfloat16: _lib.DLP_BF16}
NP2TORCH = {"float32": torch.float32, "float64": torch.float64, "bfloat16": torch.bfloat16}


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("dynlplus_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def to_dtype(dt) -> torch.dtype:
    if isinstance(dt, torch.dtype):
        return dt
    return NP2TORCH[str(getattr(dt, "name", dt))]


def code(t: torch.Tensor) -> int:
    try:
        return DTYPES[t.dtype]
    except KeyError:
        raise TypeError(f"unsupported dtype {t.dtype}") from None


def ptr(t):
    """Raw device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    if t.device.type != "cuda":
        raise ValueError("libdlp takes CUDA tensors only")
    return t.data_ptr()


def ld(t: torch.Tensor) -> int:
    """Leading dimension (row stride in elements) of a row-major 2-D tensor."""
    if t.dim() == 1:
        return 1
    if t.stride(1) != 1:
        raise ValueError("matrices must be row-major with unit column stride")
    return t.stride(0)


def stream():
    return torch.cuda.current_stream().cuda_stream


def sync():
    """Wait for the current stream (not the whole device: another thread may be capturing a CUDA
    graph on its own stream, and a device-wide synchronisation would invalidate that capture)."""
    torch.cuda.current_stream().synchronize()


def mem_used_gb() -> float:
    return torch.cuda.memory_allocated() / 1e9 if torch.cuda.is_available() else 0.0


class Timer:
    """Wall-clock timer that synchronizes the current stream on enter and exit (dynlp/backend.py:43-56
    synchronizes the device; per-stream keeps concurrent workers independent)."""

    def __init__(self):
        self.ms = 0.0

    def __enter__(self):
        if torch.cuda.is_available():
            sync()
        self._t = time.perf_counter()
        return self

    def __exit__(self, *exc):
        if torch.cuda.is_available():
            sync()
        self.ms += (time.perf_counter() - self._t) * 1e3


class Workspace:
    """Grow-only scratch buffer handed to the kernels (they never allocate themselves)."""

    def __init__(self):
        self._buf = None

    def get(self, nbytes: int) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        if self._buf is None or self._buf.numel() < nbytes:
            self._buf = torch.empty(nbytes + (nbytes >> 2), dtype=torch.uint8, device=device())
        return self._buf


_WS: dict = {}


def workspace(tag: str = "default") -> Workspace:
    """Scratch buffer per (tag, device, current stream): work on different streams (the serving
    loop's workers) never shares a buffer."""
    key = (tag, torch.cuda.current_device() if torch.cuda.is_available() else -1,
           torch.cuda.current_stream().cuda_stream if torch.cuda.is_available() else 0)
    if key not in _WS:
        _WS[key] = Workspace()
    return _WS[key]


@dataclass
class CSR:
    """Compressed sparse rows on the device: int32 indptr/indices and float data.

    Stands in for cupyx.scipy.sparse.csr_matrix on the hot path (dynlp/backend.py:35-36).
    """

    data: torch.Tensor
    indices: torch.Tensor
    indptr: torch.Tensor
    shape: tuple

    @property
    def nnz(self) -> int:
        return int(self.indices.numel())

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def rbeg(self) -> torch.Tensor:
        return self.indptr[:-1]

    @property
    def rend(self) -> torch.Tensor:
        return self.indptr[1:]

    def avg_deg(self) -> float:
        return self.nnz / max(self.shape[0], 1)

    def astype(self, dtype) -> "CSR":
        dt = to_dtype(dtype)
        if dt == self.data.dtype:
            return self
        return CSR(self.data.to(dt), self.indices, self.indptr, self.shape)

    def to(self, dev) -> "CSR":
        return CSR(self.data.to(dev), self.indices.to(dev), self.indptr.to(dev), self.shape)

    def to_scipy(self):
        import scipy.sparse as ssp
        return ssp.csr_matrix((self.data.float().cpu().numpy() if self.data.dtype == torch.bfloat16
                               else self.data.cpu().numpy(), self.indices.cpu().numpy(),
                               self.indptr.cpu().numpy()), shape=self.shape)

    @classmethod
    def from_scipy(cls, A, dev=None, dtype=None) -> "CSR":
        A = A.tocsr()
        dev = dev or device()
        data = torch.as_tensor(A.data)
        if dtype is not None:
            data = data.to(to_dtype(dtype))
        return cls(data.to(dev), torch.as_tensor(A.indices.astype("int32")).to(dev),
                   torch.as_tensor(A.indptr.astype("int32")).to(dev), tuple(A.shape))


def csr(data, indices, indptr, shape) -> CSR:
    return CSR(data, indices, indptr, tuple(shape))


_CANCEL = None  # the registered cancel word (kept alive while registered)


def set_cancel_word(word):
    """Register a one-element int32 tensor that the device-side solve loops poll (dlp_set_cancel_word):
    while it holds a non-zero value, a running PCG stops at its next stop decision and a running push
    at its next round, and the call raises `_lib.Cancelled`. The tensor lives in device memory or in
    pinned host memory (`torch.zeros(1, dtype=torch.int32).pin_memory()`, writable from the host
    while the solve runs). None unregisters."""
    global _CANCEL
    from . import _lib
    if word is not None:
        if word.dtype != torch.int32 or word.numel() < 1:
            raise ValueError("the cancel word is a one-element int32 tensor")
        if not (word.is_cuda or word.is_pinned()):
            raise ValueError("the cancel word must be in device memory or pinned host memory")
    # pinned host memory is addressed by the same pointer on the device (unified addressing)
    _lib.call("dlp_set_cancel_word", word.data_ptr() if word is not None else None)
    _CANCEL = word

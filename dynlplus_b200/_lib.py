"""ctypes binding of libdlp.so (the C ABI declared in include/dlp.h).

The library is the only compute path: if it is missing, every call raises. There is no CPU
fallback. `python -m dynlplus_b200.build` (or `__graft_entry__.build()`) creates it in-tree.
"""
from __future__ import annotations

import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdlp.so")

DLP_F32, DLP_F64, DLP_BF16 = 0, 1, 2
STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported precision combination", 3: "CUDA runtime error",
          4: "iteration cap reached", 5: "cancelled", 6: "workspace too small", 7: "row capacity exceeded",
          8: "device-side check failed", 9: "size exceeds the fixed scratch of an allocation-free entry point"}

_P, _I, _Q, _D, _Z = ct.c_void_p, ct.c_int32, ct.c_int64, ct.c_double, ct.c_size_t
_CODES = {"p": _P, "i": _I, "q": _Q, "d": _D, "z": _Z}

# name -> (argument codes, return type). Kept in the order of include/dlp.h.
SIGNATURES: dict[str, tuple[str, object]] = {
    "dlp_version": ("", ct.c_int),
    "dlp_status_string": ("i", ct.c_char_p),
    "dlp_last_cuda_error": ("", ct.c_int),
    "dlp_sm_count": ("", ct.c_int),
    "dlp_launch_count": ("", ct.c_ulonglong),
    "dlp_set_cancel_word": ("p", ct.c_int),
    "dlp_spmm": ("ppppiipipqipddpqdpqiiidp", ct.c_int),
    "dlp_spmm_lowp": ("ppppiipqpqpddpqidp", ct.c_int),
    "dlp_frontier_jacobi": ("ppppipiipqpqpdpqipppidp", ct.c_int),
    "dlp_push_scatter": ("ppppipiipqpqipidp", ct.c_int),
    "dlp_mark_neighbors": ("ppppipp", ct.c_int),
    "dlp_push_take": ("piipqpqppqipp", ct.c_int),
    "dlp_violating": ("piipqpipppp", ct.c_int),
    "dlp_compact_workspace_bytes": ("i", ct.c_size_t),
    "dlp_compact": ("ppipppzp", ct.c_int),
    "dlp_colreduce_workspace_bytes": ("i", ct.c_size_t),
    "dlp_colreduce": ("iiipqpqpipppzp", ct.c_int),
    "dlp_colreduce_noalloc": ("iiipqpqpippp", ct.c_int),
    "dlp_cc_edges": ("ippqppp", ct.c_int),
    "dlp_cc_graph_workspace_bytes": ("", ct.c_size_t),
    "dlp_cc_graph": ("ippppipppppzp", ct.c_int),
    "dlp_cc_graph_warm_workspace_bytes": ("i", ct.c_size_t),
    "dlp_cc_graph_warm": ("ippppippppzp", ct.c_int),
    "dlp_ground_reach_workspace_bytes": ("i", ct.c_size_t),
    "dlp_ground_reach": ("ippppippppppppzp", ct.c_int),
    "dlp_cc_mask_labels_workspace_bytes": ("i", ct.c_size_t),
    "dlp_cc_mask_labels": ("ippppppzp", ct.c_int),
    "dlp_cc_relabel": ("ippppzp", ct.c_int),
    "dlp_residual_stats_workspace_bytes": ("i", ct.c_size_t),
    "dlp_residual_stats": ("iipqpqppqippzp", ct.c_int),
    "dlp_pcg_workspace_bytes": ("i", ct.c_size_t),
    "dlp_pcg": ("ppppiiippqpqpqpqpqippdiiiiidpzpppppppq", ct.c_int),
    "dlp_graph_delete": ("ipppppppipppippppppp", ct.c_int),
    "dlp_graph_insert_workspace_bytes": ("i", ct.c_size_t),
    "dlp_graph_insert": ("ipppppppppipppipppppppzp", ct.c_int),
    "dlp_class_sum_rhs": ("iipqppqp", ct.c_int),
    "dlp_class_sum_update": ("iipqppqpp", ct.c_int),
    "dlp_predict_workspace_bytes": ("i", ct.c_size_t),
    "dlp_predict": ("iipqiippppppzp", ct.c_int),
    "dlp_label_update": ("pidpppppipppp", ct.c_int),
    "dlp_new_dissim": ("pipppidpp", ct.c_int),
    "dlp_graph_toggle": ("ppppppippppp", ct.c_int),
    "dlp_graph_to_csr_workspace_bytes": ("i", ct.c_size_t),
    "dlp_graph_to_csr": ("ippppppppzp", ct.c_int),
    "dlp_graph_rowsum": ("ppppipp", ct.c_int),
    "dlp_system_rows": ("pippipdpiiippqppqp", ct.c_int),
    "dlp_park_rows": ("pipiipdpqpqp", ct.c_int),
    "dlp_cols_scale": ("iipqipipqip", ct.c_int),
    "dlp_fused_push_workspace_bytes": ("ii", ct.c_size_t),
    "dlp_fused_push": ("ppppiiippqpqippiiiipzpppp", ct.c_int),
    "dlp_fused_push_counts": ("ppp", ct.c_int),
    "dlp_amg_match_workspace_bytes": ("i", ct.c_size_t),
    "dlp_amg_match": ("ipppipppzp", ct.c_int),
    "dlp_amg_members_workspace_bytes": ("i", ct.c_size_t),
    "dlp_amg_members": ("iippppzp", ct.c_int),
    "dlp_amg_coarse_plan": ("ipppppzp", ct.c_int),
    "dlp_amg_coarsen": ("ipppppppppqppppppzp", ct.c_int),
    "dlp_amg_coarse_keys": ("ippppippp", ct.c_int),
    "dlp_amg_coarse_reduce_workspace_bytes": ("qi", ct.c_size_t),
    "dlp_amg_coarse_reduce": ("qppipppppppppzp", ct.c_int),
    "dlp_sort_pairs_workspace_bytes": ("q", ct.c_size_t),
    "dlp_sort_pairs": ("qqpppppzp", ct.c_int),
    "dlp_amg_restrict": ("iipppqpqip", ct.c_int),
    "dlp_amg_prolong_add": ("iippqpqip", ct.c_int),
    "dlp_amg_scale_rows": ("iidpqppqip", ct.c_int),
    "dlp_amg_jacobi_sweep": ("iippppqpqpdpqip", ct.c_int),
    "dlp_dense_apply": ("iippqpqip", ct.c_int),
    "dlp_amg_vcycle_workspace_bytes": ("piii", ct.c_size_t),
    "dlp_amg_vcycle": ("pipidiiipqpqpzp", ct.c_int),
    "dlp_pcg_amg_workspace_bytes": ("piii", ct.c_size_t),
    "dlp_pcg_amg": ("ppppiippqpqpqpqpqpqippdiiiidpipidipzppppppq", ct.c_int),
    "dlp_dense_spd_inverse_workspace_bytes": ("i", ct.c_size_t),
    "dlp_dense_spd_inverse": ("ippzp", ct.c_int),
    "dlp_pcg_batched_workspace_bytes": ("iii", ct.c_size_t),
    "dlp_pcg_batched": ("pppiippqpqpqpqpqiiippppppdiiiiiidpzpppp", ct.c_int),
    "dlp_ground_update": ("ipppppp", ct.c_int),
}

_lib = None


class AmgLevel(ct.Structure):
    """dlp_amg_level (include/dlp.h): one level of an AMG hierarchy."""
    _fields_ = [("n", ct.c_int32), ("nnz", ct.c_int64), ("indptr", ct.c_void_p), ("col", ct.c_void_p),
                ("w", ct.c_void_p), ("diag", ct.c_void_p), ("agg", ct.c_void_p), ("off", ct.c_void_p),
                ("members", ct.c_void_p)]


class DLPError(RuntimeError):
    """A libdlp entry point returned a non-zero status."""

    def __init__(self, name: str, status: int, cuda: int = 0):
        msg = f"{name} failed: {STATUS.get(status, status)} (status {status}"
        msg += f", cudaError {cuda})" if status == 3 else ")"
        super().__init__(msg)
        self.status = status


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libdlp.so is missing at {LIB_PATH}: build it with `python -m dynlplus_b200.build`")
        L = ct.CDLL(LIB_PATH)
        for name, (codes, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = [_CODES[c] for c in codes]
            fn.restype = res
        _lib = L
    return _lib


class Cancelled(DLPError):
    """A device-side loop stopped because the registered cancel word was set (DLP_ERR_CANCELLED)."""


DLP_ERR_CAP, DLP_ERR_CANCELLED = 4, 5


def call(name: str, *args, allow: tuple = ()) -> int:
    """Call an int-returning entry point; returns its status when it is 0 or listed in `allow`,
    raises Cancelled for DLP_ERR_CANCELLED and DLPError for any other non-zero status."""
    st = getattr(lib(), name)(*args)
    if st != 0 and st not in allow:
        if st == DLP_ERR_CANCELLED:
            raise Cancelled(name, st)
        raise DLPError(name, st, lib().dlp_last_cuda_error() if st == 3 else 0)
    return st


def exported_symbols() -> list[str]:
    return list(SIGNATURES)

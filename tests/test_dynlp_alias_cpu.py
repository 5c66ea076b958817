"""The reference's import name (CPU): `dynlp` and its modules are this implementation's."""
import importlib


def test_from_dynlp_import_modules():
    from dynlp import amg, cc, graphs, kernels, solvers, stream  # noqa: F401
    import dynlplus_b200.solvers
    assert solvers is dynlplus_b200.solvers


def test_dotted_imports_resolve_to_the_same_modules():
    for name in ("backend", "kernels", "graphs", "cc", "amg", "stream", "solvers", "bench"):
        assert importlib.import_module(f"dynlp.{name}") is importlib.import_module(f"dynlplus_b200.{name}")
    from dynlp.solvers import SOLVERS, make  # noqa: F401
    from dynlp.stream import IncrementalStream, Stream, System  # noqa: F401
    from dynlp.kernels import FrontierOps, FusedPush, spmm_axpy  # noqa: F401
    assert "dynlp+inc" in SOLVERS

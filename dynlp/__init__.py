"""The reference's import name: `import dynlp` / `from dynlp import solvers, stream, ...` resolve to
this implementation, so code written against the reference runs unchanged on the B200 path.

Each module of the reference's package (dynlp/__init__.py lists none; its modules are backend,
kernels, graphs, cc, amg, stream, solvers, bench) is the module of the same name in dynlplus_b200,
registered under both names: `dynlp.solvers is dynlplus_b200.solvers`.
"""
import importlib
import sys

_MODULES = ("backend", "kernels", "graphs", "cc", "amg", "stream", "solvers", "bench")

for _name in _MODULES:
    _mod = importlib.import_module(f"dynlplus_b200.{_name}")
    sys.modules[f"{__name__}.{_name}"] = _mod
    globals()[_name] = _mod

__all__ = list(_MODULES)

"""The drop-in boundary (CPU): every public name of the reference's modules graphs, stream, solvers,
amg, cc and kernels exists here with its parameters in the same order (positional) or among ours
(keyword-only), as recorded from the reference's source in tests/golden/api.json. The IMDB review
pipeline (downloads, TF-IDF over sparse rows) is the one part left out."""
import ast
import importlib
import inspect
import json
import os

from conftest import GOLDEN

OUT_OF_SCOPE = {("graphs", "tfidf")}  # the IMDB pipeline's document vectoriser


def _params(obj):
    sig = inspect.signature(obj)
    pos = [p.name for p in sig.parameters.values() if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]
    kw = [p.name for p in sig.parameters.values() if p.kind == p.KEYWORD_ONLY]
    var_kw = any(p.kind == p.VAR_KEYWORD for p in sig.parameters.values())
    return pos, kw, var_kw


def _check(where, obj, want, problems):
    pos, kw, var_kw = _params(obj)
    if pos[: len(want["args"])] != want["args"]:
        problems.append(f"{where}: positional {want['args']} != ours {pos}")
    missing = [k for k in want["kwonly"] if k not in kw and k not in pos and not var_kw]
    if missing:
        problems.append(f"{where}: keyword arguments {missing} missing")


def test_public_api_matches_the_reference():
    with open(os.path.join(GOLDEN, "api.json")) as f:
        api = json.load(f)
    problems = []
    for m, spec in api.items():
        if m.startswith(("bench_", "kernelbench_")):
            continue
        ours = importlib.import_module(f"dynlplus_b200.{m}")
        for c in spec["constants"]:
            if not hasattr(ours, c):
                problems.append(f"{m}.{c} missing")
        for name, want in spec["functions"].items():
            if (m, name) in OUT_OF_SCOPE:
                continue
            if not hasattr(ours, name):
                problems.append(f"{m}.{name} missing")
                continue
            _check(f"{m}.{name}", getattr(ours, name), want, problems)
        for cls, methods in spec["classes"].items():
            if not hasattr(ours, cls):
                problems.append(f"{m}.{cls} missing")
                continue
            for meth, want in methods.items():
                if not hasattr(getattr(ours, cls), meth):
                    problems.append(f"{m}.{cls}.{meth} missing")
                    continue
                _check(f"{m}.{cls}.{meth}", getattr(getattr(ours, cls), meth), want, problems)
    assert not problems, "\n".join(problems)


def test_streaming_benchmark_flags_and_columns_match_the_reference():
    """dynlp/bench.py:21-38: the same flags (switches as switches, the same defaults except the
    dataset, whose reference default is the IMDB graph) and the same CSV columns in order."""
    from dynlplus_b200 import bench
    with open(os.path.join(GOLDEN, "api.json")) as f:
        api = json.load(f)
    assert bench.FIELDS == api["bench_fields"]
    ours = {flag: (typ is None, default) for flag, typ, default, _ in bench.ARGS}
    for a in api["bench_args"]:
        assert a["flag"] in ours, a["flag"]
        switch, default = ours[a["flag"]]
        assert switch == a["switch"], a["flag"]
        if a["flag"] == "--dataset":
            assert default == "sbm"  # imdb needs downloads; the synthetic graphs stay available
        elif a["flag"] == "--data-dir":
            from dynlplus_b200 import graphs
            assert default == graphs.DATA_DIR
        else:
            assert default == ast.literal_eval(a["default"]), a["flag"]

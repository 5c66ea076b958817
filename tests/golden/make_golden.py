"""Generate the golden fixtures by running the REFERENCE (shishir9159/DynLPlus) on the CPU.

    python tests/golden/make_golden.py --reference <reference checkout>   (or DLP_REFERENCE=<path>)

The reference is pure Python over CuPy; `cupy_shim.install` maps CuPy onto NumPy/SciPy and routes
its three NVRTC-kernel entry points to its own vectorised fallbacks (see cupy_shim.py). Each
fixture stores small seeded inputs and the reference's outputs for them; the oracle (oracle/) is
pinned against these, and the GPU tests compare the CUDA path with both. The reference tree is
not needed at test time: only these .npz files are read.
"""
from __future__ import annotations

import argparse
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def csr_parts(prefix, A):
    return {f"{prefix}_indptr": np.asarray(A.indptr, dtype=np.int32), f"{prefix}_indices": np.asarray(A.indices, dtype=np.int32),
            f"{prefix}_data": np.asarray(A.data), f"{prefix}_shape": np.asarray(A.shape, dtype=np.int64)}


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path) / 1e3:.0f} kB)")


def gen_cc(dl):
    from dynlp.cc import connected_components
    out = {}
    rnd = random.Random(0)  # the reference's own test case (tests/test_dynlp.py:41-46)
    pairs = [(rnd.randrange(400), rnd.randrange(400)) for _ in range(300)]
    cases = [(400, np.array([a for a, _ in pairs]), np.array([b for _, b in pairs]))]
    rs = np.random.RandomState(11)
    cases.append((5000, rs.randint(0, 5000, 4000), rs.randint(0, 5000, 4000)))   # many components
    cases.append((3000, rs.randint(0, 3000, 30000), rs.randint(0, 3000, 30000)))  # one giant
    path = np.arange(2047)
    cases.append((2048, path[::-1], path[::-1] + 1))  # a long path, hooked from the far end
    cases.append((17, np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64)))  # no edges
    for i, (n, r, c) in enumerate(cases):
        lab, nc = connected_components(n, np.asarray(r), np.asarray(c))
        out.update({f"c{i}_n": np.int64(n), f"c{i}_rows": np.asarray(r, np.int32), f"c{i}_cols": np.asarray(c, np.int32),
                    f"c{i}_labels": np.asarray(lab, np.int32), f"c{i}_ncomp": np.int64(nc)})
    out["ncases"] = np.int64(len(cases))
    save("cc.npz", **out)


def gen_kernels(dl):
    from dynlp import graphs, kernels, solvers
    out = {}
    # the reference's kernel-test graph family (tests/test_dynlp.py:199,249), at n=1500 to keep
    # the fixture small; inputs are float32-representable so they compress
    ds = graphs.sbm(1500, K=2, deg=12, seed=8, dtype="float64")
    W, n = ds.A, ds.n
    out.update(csr_parts("W", W))
    rs = np.random.RandomState(0)
    f32 = lambda x: x.astype(np.float32).astype(np.float64)  # noqa: E731
    frontier = np.sort(rs.choice(n, 350, replace=False)).astype(np.int32)
    out["frontier"] = frontier
    diag = (W @ np.ones(n) + 1)
    out["diag"] = diag
    for C in (1, 3, 9, 17):
        X, rhs = f32(rs.random_sample((n, C))), f32(rs.random_sample((n, C)))
        a = f32(rs.random_sample(n))
        D = f32(rs.standard_normal((frontier.size, C)))
        ops = kernels.FrontierOps(W, C, 8)
        Y, ch = ops.jacobi(frontier, X, rhs, diag, 1e-2)
        R = np.zeros((n, C))
        mark = np.zeros(n, dtype=np.uint8)
        ops.push(frontier, D, R, mark)
        mk = np.zeros(n, dtype=np.uint8)
        ops.mark_neighbors(frontier, mk)
        out.update({f"C{C}_X": X, f"C{C}_rhs": rhs, f"C{C}_a": a, f"C{C}_D": D, f"C{C}_jacY": Y,
                    f"C{C}_jacch": np.asarray(ch, np.uint8), f"C{C}_pushR": R, f"C{C}_pushmark": mark,
                    f"C{C}_marknb": mk, f"C{C}_edges": np.int64(int(ops.edges)),
                    f"C{C}_spmm": solvers.spmm(W, X),
                    f"C{C}_applyA": solvers.apply_A(type("S", (), {"W": W, "diag": a})(), X)})
    save("kernels.npz", **out)


def _stream_system(dl, n=3000, K=3, deg=8, seed=3, init_frac=0.2, label_frac=0.02, dtype="float64", batch=0):
    from dynlp import graphs
    from dynlp.stream import Stream
    ds = graphs.sbm(n, K=K, deg=deg, seed=seed, dtype=dtype)
    st = Stream(ds, init_frac=init_frac, n_batches=3, label_frac=label_frac, dtype=dtype)
    active = np.zeros(ds.n, dtype=bool)
    for t, sys_ in enumerate(st.batches()):
        ins, dele = st.schedule[t]
        active[ins], active[dele] = True, False
        if t == batch:
            return ds, st, sys_, active.copy()
    raise ValueError(batch)


def gen_system(dl):
    out = {}
    for b in (0, 2):
        ds, st, s, active = _stream_system(dl, batch=b)
        p = f"b{b}"
        out.update(csr_parts(f"{p}_A", ds.A))
        out.update(csr_parts(f"{p}_W", s.W))
        out.update({f"{p}_y": np.asarray(ds.y, np.int32), f"{p}_K": np.int64(ds.K),
                    f"{p}_active": active, f"{p}_labeled": np.asarray(st.labeled),
                    f"{p}_U": np.asarray(s.U, np.int64), f"{p}_s": s.s, f"{p}_diag": s.diag, f"{p}_B": s.B,
                    f"{p}_rhs": s.rhs, f"{p}_n_ungrounded": np.int64(s.n_ungrounded)})
    save("system.npz", **out)


def gen_solvers(dl):
    from dynlp import kernels, solvers
    out = {}
    ds, st, s, active = _stream_system(dl, n=3000, K=3, deg=8, seed=3, batch=1)
    out.update(csr_parts("W", s.W))
    out.update({"diag": s.diag, "rhs": s.rhs})
    # pcg with the Jacobi preconditioner (dynlp/solvers.py:66-97)
    for tag, eps in (("pcg_loose", [1e-4] * 3), ("pcg_tight", [1e-10] * 3)):
        st_ = solvers.Stats()
        Z = solvers.pcg(s, np.zeros((s.n_u, 3)), s.rhs.copy(), eps, solvers.jacobi_M(s), 10_000, st_)
        out.update({f"{tag}_eps": np.asarray(eps), f"{tag}_Z": Z, f"{tag}_iters": np.int64(st_.iters)})
    # synchronous push from a perturbed warm start, with every round's candidate set recorded
    Zstar = solvers.pcg(s, np.zeros((s.n_u, 3)), s.rhs.copy(), [1e-12] * 3, solvers.jacobi_M(s), 10_000,
                        solvers.Stats())
    rs = np.random.RandomState(5)
    Z0 = Zstar.copy()
    hit = rs.choice(s.n_u, 40, replace=False)
    Z0[hit] += rs.standard_normal((40, 3)) * 0.05
    R0 = s.rhs - solvers.apply_A(s, Z0)
    rounds = []
    orig = kernels.FrontierOps.push

    def rec(self, frontier, D, R, mark):
        rounds.append(np.asarray(frontier).copy())
        return orig(self, frontier, D, R, mark)

    kernels.FrontierOps.push = rec
    try:
        ops = kernels.FrontierOps(s.W, 3)
        Z1, R1, ok = solvers.push(s, Z0.copy(), R0.copy(), [1e-7] * 3, ops, solvers.Stats())
    finally:
        kernels.FrontierOps.push = orig
    out.update({"push_Z0": Z0, "push_R0": R0, "push_eps": np.asarray([1e-7] * 3), "push_Z": Z1, "push_R": R1,
                "push_ok": np.int64(ok), "push_rounds": np.int64(len(rounds)),
                "push_cand": np.concatenate(rounds).astype(np.int32),
                "push_cand_off": np.cumsum([0] + [len(r) for r in rounds]).astype(np.int64)})
    save("solvers.npz", **out)


def gen_amg(dl):
    """AMG setup and one V-cycle of the reference (dynlp/amg.py) on a float32 system."""
    from dynlp.amg import AMG, _handshake, _coarsen
    from dynlp.graphs import csr_rows
    out = {}
    ds, st, s, active = _stream_system(dl, n=3000, K=3, deg=8, seed=3, batch=2, dtype="float32")
    out.update(csr_parts("W", s.W))
    out["s"] = np.asarray(s.s, dtype=np.float64)
    W = s.W
    a2, nc2 = _handshake(W.shape[0], csr_rows(W), W.indices, W.data, 3)
    out.update({"match_agg": np.asarray(a2, np.int32), "match_nc": np.int64(nc2)})
    Wc, sc = _coarsen(W, s.s, a2, nc2)
    out.update(csr_parts("match_Wc", Wc))
    out["match_sc"] = np.asarray(sc, np.float64)
    amg = AMG(W, s.s, max_coarse=50)
    out["sizes"] = np.asarray(amg.sizes, np.int64)
    for i, L in enumerate(amg.levels):
        out[f"L{i}_agg"] = np.asarray(L.agg, np.int32)
    rs = np.random.RandomState(4)
    R = rs.standard_normal((W.shape[0], 3)).astype(np.float32)
    out["R"] = R
    out["MR"] = np.asarray(amg(R), np.float64)
    save("amg.npz", **out)


def gen_stream(dl):
    """The vertex-arrival streams (dynlp/stream.py:84-346): the schedule drawn up front, every
    batch's system from Stream._build (U, is_new, seed, the new vertices' tau and FH components)
    and from IncrementalStream (solved/changed rows, global-index diag and rhs), and the warm
    starts supernode_init / init_h (dynlp/solvers.py:128-163) on those systems."""
    from dynlp import graphs, solvers
    from dynlp.stream import IncrementalStream, Stream
    out = {}
    ds = graphs.sbm(2000, K=3, deg=8, seed=3, dtype="float64")
    kw = dict(init_frac=0.2, n_batches=4, label_frac=0.02, del_frac=0.1, seed=1, dtype="float64")
    st = Stream(ds, **kw)
    out.update(csr_parts("A", ds.A))
    out.update({"y": np.asarray(ds.y, np.int32), "K": np.int64(ds.K), "order_in": np.asarray(ds.order, np.int64),
                "order": np.asarray(st.order, np.int64), "labeled": np.asarray(st.labeled), "n0": np.int64(st.n0),
                "tau": np.float64(st.tau), "wmax": np.float64(st.wmax), "eta": np.float64(st.eta),
                "nbatches": np.int64(len(st.schedule))})
    for t, (ins, dele) in enumerate(st.schedule):
        out[f"t{t}_ins"], out[f"t{t}_del"] = np.asarray(ins, np.int64), np.asarray(dele, np.int64)
    rs = np.random.RandomState(9)
    for t, s in enumerate(st.batches()):
        p = f"s{t}"
        out.update({f"{p}_U": np.asarray(s.U, np.int64), f"{p}_is_new": np.asarray(s.is_new),
                    f"{p}_seed": np.asarray(s.seed), f"{p}_diag": s.diag, f"{p}_rhs": s.rhs,
                    f"{p}_n_ungrounded": np.int64(s.n_ungrounded)})
        for name in ("tau", "fh"):
            lab, nc = s.comps[name]
            out[f"{p}_{name}"], out[f"{p}_{name}_nc"] = np.asarray(lab, np.int32), np.int64(nc)
        # warm starts on this system: DynLP's rule (known=None) and DynLP+'s (known = old rows)
        X = rs.random_sample((s.n_u, s.C))
        H = 1.0 + rs.random_sample((s.n_u, 1))
        out[f"{p}_X"], out[f"{p}_H"] = X, H
        out[f"{p}_sn_tau"] = solvers.supernode_init(s, X.copy(), comp="tau")
        known = ~np.asarray(s.is_new)
        out[f"{p}_sn_fh"] = solvers.supernode_init(s, X.copy(), known, comp="fh")
        out[f"{p}_ih"] = solvers.init_h(s, H.copy(), known, 7.0)
    # the resident form on the same graph with float32 weights (the resident graph keeps fp32 edge
    # weights; its fp64 system is built from them, as the reference's W64 is from a float32 A)
    ds32 = graphs.sbm(2000, K=3, deg=8, seed=3, dtype="float32")
    out.update(csr_parts("A32", ds32.A))
    out.update({"tau32": np.float64(float(ds32.A.data.mean())), "wmax32": np.float64(float(ds32.A.data.max()))})
    ist = IncrementalStream(ds32, ball_hops=3, **{**kw, "dtype": "float32"})
    for t, s in enumerate(ist.batches()):
        p = f"i{t}"
        out.update({f"{p}_solved": np.asarray(s.solved), f"{p}_changed": np.asarray(s.changed, np.int64),
                    f"{p}_is_new": np.asarray(s.is_new), f"{p}_seed": np.asarray(s.seed),
                    f"{p}_diag": np.asarray(s.astype("float64").diag), f"{p}_rhs": np.asarray(s.astype("float64").rhs),
                    f"{p}_n_ungrounded": np.int64(s.n_ungrounded)})
        for name in ("tau", "fh"):
            lab, nc = s.comps[name]
            out[f"{p}_{name}"], out[f"{p}_{name}_nc"] = np.asarray(lab, np.int32), np.int64(nc)
    out["inc_counters"] = np.asarray([ist.counters["ball_checks"], ist.counters["full_ground"]], np.int64)
    save("stream.npz", **out)


def gen_graphs(dl):
    """The synthetic kNN family (dynlp/graphs.py:78-143): two synth datasets (the reference's AMG
    test parameters, tests/test_dynlp.py:160, and a 3-class one) and a kNN graph of random rows."""
    from dynlp import graphs
    out = {}
    for i, kw in enumerate([dict(n=1200, K=2, k=6, subs=2, seed=7, dtype="float64"),
                            dict(n=3000, K=3, k=5, dim=16, subs=5, seed=1, dtype="float32")]):
        ds = graphs.synth(**kw)
        out.update(csr_parts(f"s{i}_A", ds.A))
        out.update({f"s{i}_y": np.asarray(ds.y, np.int32), f"s{i}_order": np.asarray(ds.order, np.int64),
                    f"s{i}_K": np.int64(ds.K), f"s{i}_name": np.asarray(ds.name)})
    rs = np.random.RandomState(5)
    X = rs.standard_normal((700, 8)).astype(np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    out["knn_X"] = X
    out.update(csr_parts("knn_A", graphs.knn_graph(X, 4, "float32")))
    save("graphs.npz", **out)


def gen_api(dl):
    """The reference's public API (the drop-in boundary): for the modules graphs, stream, solvers,
    amg, cc and kernels, every public function's parameters, every public class's constructor and
    public methods' parameters, and the public upper-case constants; read from the source (ast)."""
    import ast
    import json
    ref = os.path.join(os.path.dirname(os.path.dirname(__import__("dynlp").__file__)), "dynlp")

    def params(fn):
        a = fn.args
        return {"args": [x.arg for x in a.posonlyargs + a.args], "kwonly": [x.arg for x in a.kwonlyargs]}

    api = {}
    for m in ("graphs", "stream", "solvers", "amg", "cc", "kernels"):
        tree = ast.parse(open(os.path.join(ref, m + ".py")).read())
        mod = {"functions": {}, "classes": {}, "constants": []}
        for node in tree.body:
            if isinstance(node, ast.FunctionDef) and not node.name.startswith("_"):
                mod["functions"][node.name] = params(node)
            elif isinstance(node, ast.ClassDef) and not node.name.startswith("_"):
                mod["classes"][node.name] = {sub.name: params(sub) for sub in node.body
                                             if isinstance(sub, ast.FunctionDef)
                                             and (sub.name == "__init__" or not sub.name.startswith("_"))}
            elif isinstance(node, ast.Assign):
                mod["constants"] += [t.id for t in node.targets
                                     if isinstance(t, ast.Name) and t.id.isupper() and not t.id.startswith("_")]
        api[m] = mod
    # the streaming benchmark's command line and CSV columns (dynlp/bench.py:21-38)
    tree = ast.parse(open(os.path.join(ref, "bench.py")).read())
    for node in tree.body:
        if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name):
            if node.targets[0].id == "ARGS":
                api["bench_args"] = [{"flag": e.elts[0].value, "switch": isinstance(e.elts[1], ast.Constant),
                                      "default": ast.unparse(e.elts[2])} for e in node.value.elts]
            elif node.targets[0].id == "FIELDS":
                api["bench_fields"] = [e.value for e in node.value.elts]
    # the kernel micro-benchmark's flags and CSV columns (dynlp/kernelbench.py:21-63)
    tree = ast.parse(open(os.path.join(ref, "kernelbench.py")).read())
    api["kernelbench_args"] = [{"flag": t.elts[0].value, "default": ast.unparse(t.elts[2])} for t in ast.walk(tree)
                               if isinstance(t, ast.Tuple) and len(t.elts) == 3 and isinstance(t.elts[0], ast.Constant)
                               and isinstance(t.elts[0].value, str) and t.elts[0].value.startswith("--")]
    api["kernelbench_fields"] = next([k.arg for k in c.keywords] for c in ast.walk(tree)
                                     if isinstance(c, ast.Call) and isinstance(c.func, ast.Name)
                                     and c.func.id == "dict" and c.keywords)
    path = os.path.join(HERE, "api.json")
    with open(path, "w") as f:
        json.dump(api, f, indent=1, sort_keys=True)
    print(f"wrote {path}")


def gen_matrix(dl):
    """The reference's results matrix (scripts/matrix.py) on a synthetic results directory: CSV rows
    of the streaming benchmark's FIELDS for two datasets and five solvers; stores the inputs and the
    matrix.csv / matrix.md the reference's script writes for them."""
    import importlib.util
    import shutil
    import tempfile
    from dynlp.bench import FIELDS
    rs = np.random.RandomState(3)
    out_dir = os.path.join(HERE, "matrix")
    shutil.rmtree(out_dir, ignore_errors=True)
    os.makedirs(out_dir)
    with tempfile.TemporaryDirectory() as d:
        for tag, nb in (("sbm-20k", 3), ("er-50k", 4)):
            rows = []
            for solver in ("dynlp", "itlp", "dynlp+auto", "dynlp-fh", "dynlp+inc"):
                for b in range(nb):
                    r = {f: "" for f in FIELDS}
                    r.update(tag=tag, dataset=tag.split("-")[0], K=3, batch=b, solver=solver, n_active=1000 * (b + 5),
                             n_u=900 * (b + 5), nnz=8000 * (b + 5), inserted=500, deleted=50,
                             iters=int(rs.randint(5, 400)), edges=int(rs.randint(10**5, 10**7)),
                             sweeps=float(rs.randint(1, 90)), ms=round(float(rs.uniform(1, 300)), 3),
                             setup_ms=round(float(rs.uniform(0, 5)), 3),
                             path=["inc-push", "inc-pcg"][int(rs.randint(0, 2))] if solver == "dynlp+inc" else "pcg",
                             err_max=float(rs.uniform(1e-6, 1e-2)) if solver != "itlp" or b else "",
                             cert_self=float(rs.uniform(1e-5, 1e-3)), cert_post=float(rs.uniform(1e-5, 1e-3)),
                             hmax=float(rs.uniform(1, 50)), hmax_ref=float(rs.uniform(1, 50)),
                             agree=float(rs.uniform(0.9, 1)), acc_true=round(float(rs.uniform(0.6, 0.99)), 4),
                             build_ms=round(float(rs.uniform(5, 50)), 3), ref_ms=round(float(rs.uniform(10, 90)), 3),
                             run_s=round(float(rs.uniform(20, 40)), 2), delta=1e-4, tol=1e-3, dtype="float32",
                             group="auto")
                    rows.append(r)
            path = os.path.join(d, f"{tag}.csv")
            import csv as _csv
            with open(path, "w", newline="") as fh:
                w = _csv.DictWriter(fh, fieldnames=FIELDS)
                w.writeheader()
                w.writerows(rows)
            shutil.copy(path, os.path.join(out_dir, f"{tag}.csv"))
        root = os.path.dirname(os.path.dirname(os.path.abspath(dl.__file__)))
        spec = importlib.util.spec_from_file_location("ref_matrix", os.path.join(root, "scripts", "matrix.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        import contextlib
        with open(os.devnull, "w", encoding="utf-8") as sink, contextlib.redirect_stdout(sink):
            mod.main(d)
        for name in ("matrix.csv", "matrix.md"):
            text = open(os.path.join(d, name), encoding="utf-8").read().replace(d, "RESULTS_DIR")
            open(os.path.join(out_dir, "expected_" + name), "w", encoding="utf-8").write(text)
    print(f"wrote {out_dir}")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--reference", default=os.environ.get("DLP_REFERENCE"),
                    help="the reference checkout (default: $DLP_REFERENCE)")
    ap.add_argument("--only", default="")
    a = ap.parse_args(argv)
    import cupy_shim
    if not a.reference:
        ap.error("--reference (or DLP_REFERENCE) names the reference checkout")
    dl = cupy_shim.install(a.reference)
    gens = {"cc": gen_cc, "kernels": gen_kernels, "system": gen_system, "solvers": gen_solvers, "amg": gen_amg,
            "stream": gen_stream, "graphs": gen_graphs, "api": gen_api, "matrix": gen_matrix}
    for name, fn in gens.items():
        if not a.only or name in a.only.split(","):
            fn(dl)


if __name__ == "__main__":
    main()

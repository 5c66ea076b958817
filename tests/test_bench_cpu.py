"""bench.py without a GPU: the roofline inputs (the algorithmic bytes of one fused PCG iteration at
the headline size, the committed ncu traffic file), the flags of the profiling runs, and the
reference arm's JSON line."""
import json
import os

import pytest

import bench


def test_pcg_iteration_bytes_at_the_headline_size():
    # n = 1M rows, 9,901,056 entries of the compact W_UU, C = 9 fp32 columns: 735.6 MB
    assert bench.pcg_iteration_bytes(1_000_000, 9_901_056, 9) == 735_646_468
    # the class-sum corrections' 8 columns on the bench's compact W_UU (9,901,194 entries): 664.0 MB
    assert bench.pcg_iteration_bytes(1_000_000, 9_901_194, 8) == 664_047_764
    # the model's pieces: row pointers, per entry (index, weight, gathered row), AP, diag, own row,
    # the six vector passes and the diagonal of the sweep
    n, nnz, C, s = 1_000_000, 9_901_194, 8, 4
    assert bench.pcg_iteration_bytes(n, nnz, C) == (4 * (n + 1) + nnz * (4 + s + C * s) + n * C * s + n * s
                                                    + n * C * s + 6 * n * C * s + n * s)


def test_refine_share_reaches_the_solver():
    from dynlplus_b200 import solvers
    assert solvers.IncrementalLP(10, 4, "float32", refine_share=0.35).refine_share == 0.35
    assert solvers.IncrementalLP(10, 4, "float32").refine_share == 0.2
    assert bench.parse([]).refine_share == 0.2


def test_traffic_file_is_consistent():
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles",
                     "pcg_iteration_traffic.json")
    t = json.load(open(p))
    assert (t["n"], t["C"]) == (1_000_000, 8)  # class-sum corrections: 7 class columns and h
    assert t["dram_bytes_per_iteration"] == sum(t["per_kernel"].values())
    assert set(t["per_kernel"]) == {"k_pcg_apply", "k_pcg_fused"}  # the two-kernel iteration


def test_profiling_flags_parse():
    a = bench.parse(["--steps", "1", "--warmup", "3", "--no-cpu-baseline", "--no-clocks", "--no-graphs"])
    assert a.no_graphs and a.no_clocks and a.no_cpu_baseline and a.steps == 1
    assert not bench.parse([]).no_graphs


def test_reference_arm_prints_the_contract_line(capsys, monkeypatch):
    """--impl reference on rank 0: the oracle port over a small graph prints one JSON line with the
    arm's metric, config, cpu_baseline and a zero-copy e2e."""
    monkeypatch.delenv("RANK", raising=False)
    a = bench.parse(["--impl", "reference", "--n", "3000", "--batch", "200", "--steps", "3", "--warmup", "1",
                     "--label-frac", "0.02"])
    assert bench.reference_arm(a) == 0
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["metric"] == bench.METRIC and rec["unit"] == "edge-updates/s"
    assert rec["higher_is_better"] is True and rec["config"] == bench.config(a)
    assert 1 <= rec["steps"] <= 3 and rec["value"] > 0
    assert rec["ms_per_step"] == pytest.approx(1e3 * 200 / rec["value"], rel=1e-9)
    cb = rec["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == rec["value"] and cb["cores"] >= 1 and cb["sample"]
    assert rec["e2e"] == {"value": rec["value"], "unit": "edge-updates/s", "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    assert rec["latency_ms"]["p50"] <= rec["latency_ms"]["p99"]

"""bench.py's roofline inputs without a GPU: the algorithmic bytes of one fused PCG iteration at the
headline size, the committed ncu traffic file, and the flags of the profiling runs."""
import json
import os

import bench


def test_pcg_iteration_bytes_at_the_headline_size():
    # n = 1M rows, 9,901,056 entries of the compact W_UU, C = 9 fp32 columns: 815.6 MB
    assert bench.pcg_iteration_bytes(1_000_000, 9_901_056, 9) == 815_646_464


def test_traffic_file_is_consistent():
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles",
                     "pcg_iteration_traffic.json")
    t = json.load(open(p))
    assert (t["n"], t["C"]) == (1_000_000, 9)
    assert t["dram_bytes_per_iteration"] == sum(t["per_kernel"].values())
    assert set(t["per_kernel"]) == {"k_pcg_apply", "k_pcg_update", "k_pcg_dir"}


def test_profiling_flags_parse():
    a = bench.parse(["--steps", "1", "--warmup", "3", "--no-cpu-baseline", "--no-clocks", "--no-graphs"])
    assert a.no_graphs and a.no_clocks and a.no_cpu_baseline and a.steps == 1
    assert not bench.parse([]).no_graphs

"""bench.py with N > 1 (replicas only, one process per GPU): the cross-rank step of its timing, on
CPU ranks over gloo (world size 2). The slowest rank's times set the whole-job throughput of all
ranks' units, and every rank gets the same figures; the reference arm runs on rank 0 alone."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        dev_ms, e2e_ms = times[rank]
        out[rank] = bench.aggregate_replicas(dev_ms, e2e_ms, 10_000, world, "cpu")
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    times = {0: ([6.0, 6.2, 5.8], [6.5, 6.4]), 1: ([6.1, 7.0, 6.3], [6.6, 6.9])}
    with mp.get_context("spawn").Manager() as m:  # no fork: the ranks themselves are spawned too
        out = m.dict()
        mp.spawn(_rank, args=(2, _free_port(), times, out), nprocs=2, join=True)
        res = dict(out)
    t_dev = max(sum(times[r][0]) for r in times)
    t_e2e = max(sum(times[r][1]) for r in times)
    for r in (0, 1):
        td, te, value, e2e = res[r]
        assert td == pytest.approx(t_dev) and te == pytest.approx(t_e2e)
        assert value == pytest.approx(2 * 10_000 * 3 / (t_dev * 1e-3))
        assert e2e == pytest.approx(2 * 10_000 * 2 / (t_e2e * 1e-3))


def test_one_replica_needs_no_process_group():
    td, te, value, e2e = bench.aggregate_replicas([5.0, 5.0], [6.0], 10_000, 1)
    assert (td, te) == (10.0, 6.0)
    assert value == pytest.approx(2 * 10_000 / 0.010) and e2e == pytest.approx(10_000 / 0.006)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    assert bench.reference_arm(bench.parse(["--impl", "reference"])) == 0

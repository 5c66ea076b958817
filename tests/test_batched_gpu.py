"""Batched independent solves (GPU): each instance in the batch gets what it gets alone."""
import numpy as np
import pytest
import scipy.sparse as ssp
import scipy.sparse.linalg as sla
import torch

from conftest import direct_solve

from dynlplus_b200 import batched, graphs, stream
from oracle import ref_np as O

pytestmark = pytest.mark.gpu


def _systems(count, seed, n_range=(500, 8_000)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        k = int(rng.choice([2, 4, 8]))
        deg = float(rng.uniform(8, 24))
        ds = graphs.planted_partition(n, k, 0.75 * deg, 0.25 * deg, seed=int(seed * 1000 + i))
        lab = graphs.label_mask(n, 0.02, seed=int(seed * 1000 + i))
        out.append(stream.build_system(ds, torch.ones(n, dtype=torch.bool, device="cuda"), lab, dtype="float32"))
    return out


def _check(S, F, target):
    S64 = S.astype(torch.float64)
    A = S64.W.to_scipy().astype(np.float64)
    rel = O.relres(A, S64.diag.cpu().numpy(), F.double().cpu().numpy(), S64.rhs.cpu().numpy())
    assert rel <= target * 1.0001, rel
    Ad = ssp.diags(S64.diag.cpu().numpy()) - A
    Fd = direct_solve(Ad, S64.rhs.cpu().numpy())
    Fd = Fd.reshape(-1, 1) if Fd.ndim == 1 else Fd
    return np.abs(F.double().cpu().numpy() - Fd).max()


@pytest.mark.parametrize("graph", [True, False])
def test_batched_solves_reach_target_and_match_alone(graph):
    systems = _systems(12, seed=1)
    by_c = {}
    for s in systems:
        by_c.setdefault(s.C, []).append(s)
    for C, group in by_c.items():
        bs = batched.BatchedSystems(group, tile_rows=512)
        Z, it, st, rel = bs.solve(target_relres=1e-8, use_graph=graph)
        assert (st == 5).all(), st
        Fs = bs.split(Z)
        for S, F, r in zip(group, Fs, rel):
            _check(S, F, 1e-8)
        # alone: the same instance in a batch of one gives the same scores and iteration count
        for j in (0, len(group) - 1):
            one = batched.BatchedSystems([group[j]], tile_rows=512)
            Z1, it1, st1, _ = one.solve(target_relres=1e-8, use_graph=graph)
            assert it1[0] == it[j]
            np.testing.assert_allclose(one.split(Z1)[0].cpu().numpy(), Fs[j].cpu().numpy(), rtol=1e-12, atol=1e-14)


def test_solve_many_groups_and_autotunes():
    systems = _systems(9, seed=2)
    Fs, info = batched.solve_many(systems, target_relres=1e-6, autotune=True)
    for S, F, (it, st, rel) in zip(systems, Fs, info):
        assert st == 5 and rel <= 1e-6
        err = _check(S, F, 1e-6)
        assert err < 1e-3

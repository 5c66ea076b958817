"""CPU port of the edge-batch hot path (TEST INFRASTRUCTURE / CPU BASELINE ONLY).

Per batch, in NumPy/SciPy: the edge patch (ref_np.apply_edges), the grounded system rebuilt from the
updated graph (ref_np.build_system = Stream._build, dynlp/stream.py:142-177), and a fp64 block
Jacobi-PCG correction (the reference's pcg loop, dynlp/solvers.py:66-97, with the relative-residual
stop rule) from the previous scores until max_c ||rhs_c - A F_c|| / ||rhs_c|| <= target; the h
column (A h = diag) rides along as in DynLP+ (solvers.py:312-313). Scores are kept for all n
vertices; rows outside U hold their exact inert values (F = 0, h = 1).
"""
from __future__ import annotations

import numpy as np

from . import ref_np as O


def pcg_relres(W, diag, rhs, Z, target, rhs_norm, max_iter=10_000):
    """Jacobi block PCG from Z until ||R_c|| <= target * rhs_norm_c for every column."""
    M = lambda R: R / diag[:, None]  # noqa: E731
    R = rhs - O.apply_A(W, diag, Z)
    lim = target * rhs_norm

    def done(R):
        return bool((np.sqrt((R * R).sum(axis=0)) <= lim).all())

    if done(R):
        return Z, 0
    P = Y = M(R)
    rz = (R * Y).sum(axis=0)
    it = 0
    for it in range(1, max_iter + 1):
        AP = O.apply_A(W, diag, P)
        pAp = (P * AP).sum(axis=0)
        alpha = np.where(pAp > 0, rz / np.where(pAp > 0, pAp, 1), 0)
        Z += alpha[None, :] * P
        R -= alpha[None, :] * AP
        if done(R):
            R = rhs - O.apply_A(W, diag, Z)
            if done(R):
                break
        Y = M(R)
        rz_new = (R * Y).sum(axis=0)
        P = Y + np.where(rz > 0, rz_new / np.where(rz > 0, rz, 1), 0)[None, :] * P
        rz = rz_new
    return Z, it


def _system(A, y, lab, K):
    n = A.shape[0]
    S = O.build_system(A, y, K, np.ones(n, dtype=bool), lab)
    rhs_h = np.concatenate([S["rhs"], S["diag"][:, None]], axis=1)
    return S, rhs_h


def _norms(rhs_h, C):
    rn = np.sqrt((rhs_h * rhs_h).sum(axis=0))
    rn[C] = rn[C] * 1e3  # the h column only needs a loose solve (eps_h)
    return rn


def static_solve(A, y, lab, K, target):
    """Scores (n x (C+1)) of the initial graph, solved from the prior to the target."""
    A = A.astype(np.float64)
    n = A.shape[0]
    C = 1 if K == 2 else K
    S, rhs_h = _system(A, y, lab, K)
    Z = np.zeros((S["U"].shape[0], C + 1))
    Z[:, :C] = S["prior"][None, :]
    Z, _ = pcg_relres(S["W"], S["diag"], rhs_h, Z, target, _norms(rhs_h, C))
    out = np.zeros((n, C + 1))
    out[:, C] = 1.0
    out[S["U"]] = Z
    return out


class EdgeSolverCPU:
    def __init__(self, A, y, lab, K, Z0, target_relres=1e-6):
        self.A = A.astype(np.float64).tocsr()
        self.y, self.lab, self.K = y, lab, K
        self.C = 1 if K == 2 else K
        self.Z = np.array(Z0[:, : self.C + 1], dtype=np.float64)
        self.target = target_relres
        self.prior = np.full(self.C, 0.5 if K == 2 else 1.0 / K)
        self.last_iters = 0

    def step(self, b):
        self.A = O.apply_edges(self.A, b["ins_u"], b["ins_v"], b["ins_w"].astype(np.float64), b["del_u"], b["del_v"])
        S, rhs_h = _system(self.A, self.y, self.lab, self.K)
        U = S["U"]
        C = self.C
        inU = np.zeros(self.A.shape[0], dtype=bool)
        inU[U] = True
        Z = self.Z[U]
        new = Z[:, C] == 1.0  # rows parked at the previous batch start from the prior
        Z[new, :C] = self.prior
        Z, self.last_iters = pcg_relres(S["W"], S["diag"], rhs_h, Z, self.target, _norms(rhs_h, C))
        self.Z[U] = Z
        self.Z[~inU, :C] = 0.0
        self.Z[~inU, C] = 1.0
        return S

"""ORACLE -- test infrastructure only: numpy restatement of the reference's
AKM/KSS firm-system solver, the checker of the B200 KSS solver.

kss_structure restates TwoWaySolver::build (src/akm_kss.cpp:1045-1092): match
weights, worker/firm weight sums Dw/Df, worker CSR w_ptr, firm CSR f_ptr with
f_matches (match ids in firm order, stable), and the Jacobi preconditioner
inv_diagS = 1/(Df - sum_m c_m^2/Dw[w_m]) with the ground firm J-1 at 0.

kss_pcg restates the grounded Jacobi-PCG of TwoWaySolver::solve_S
(src/akm_kss.cpp:1340-1385) and of its CUDA twin akm_cuda_solve_S_multi
(src/akm_kss_cuda.cu:560-650): x0 = 0, rhs ground entry zeroed, stop after the
update when ||r||^2 <= tol^2 ||rhs||^2, fail when p'Ap is not positive and
finite or max_iter steps pass.  The iteration count follows the same rule.

Only tests/ import this module, and only as the checker.
"""

from __future__ import annotations

import numpy as np


def kss_structure(worker, firm, weight, n_workers, n_firms):
    """Matches (must be sorted by worker) -> the arrays akm_cuda_create takes."""
    mw = np.ascontiguousarray(worker, dtype=np.int32)
    mf = np.ascontiguousarray(firm, dtype=np.int32)
    mc = np.ascontiguousarray(weight, dtype=np.float64)
    assert np.all(np.diff(mw) >= 0), "matches must be sorted by worker"
    N, J = int(n_workers), int(n_firms)
    Dw = np.bincount(mw, weights=mc, minlength=N).astype(np.float64)
    Df = np.bincount(mf, weights=mc, minlength=J).astype(np.float64)
    w_ptr = np.zeros(N + 1, dtype=np.int64)
    w_ptr[1:] = np.cumsum(np.bincount(mw, minlength=N))
    f_ptr = np.zeros(J + 1, dtype=np.int64)
    f_ptr[1:] = np.cumsum(np.bincount(mf, minlength=J))
    f_matches = np.argsort(mf, kind="stable").astype(np.int64)
    diagS = Df.copy()
    np.subtract.at(diagS, mf, mc * mc / Dw[mw])
    Jr = max(J - 1, 0)
    inv_diagS = np.zeros(J)
    ok = (np.arange(J) < Jr) & (diagS > 0.0)
    inv_diagS[ok] = 1.0 / diagS[ok]
    return {"N": N, "J": J, "m_w": mw, "m_f": mf, "m_c": mc, "w_ptr": w_ptr, "f_ptr": f_ptr,
            "f_matches": f_matches, "Dw": Dw, "Df": Df, "inv_diagS": inv_diagS}


def apply_S(st, p):
    """Grounded S p: t = (B p)/Dw, Ap = Df p - B' t, Ap[ground] = 0."""
    t = np.bincount(st["m_w"], weights=st["m_c"] * p[st["m_f"]], minlength=st["N"]) / st["Dw"]
    Ap = st["Df"] * p - np.bincount(st["m_f"], weights=st["m_c"] * t[st["m_w"]], minlength=st["J"])
    Ap[st["J"] - 1] = 0.0
    return Ap


def kss_pcg(st, rhs, tol=1e-10, max_iter=1000):
    """One grounded solve; returns (z, iterations) or (zeros, -1) on failure."""
    J = st["J"]
    r = np.array(rhs, dtype=np.float64)
    r[J - 1] = 0.0
    x = np.zeros(J)
    rn2 = float(r @ r)
    if rn2 == 0.0:
        return x, 0
    tol2 = tol * tol * rn2
    z = st["inv_diagS"] * r
    p = z.copy()
    rz = float(r @ z)
    its = 0
    while True:
        Ap = apply_S(st, p)
        pAp = float(p @ Ap)
        if not (pAp > 0.0) or not (pAp < 1e300):
            return np.zeros(J), -1
        a = rz / pAp
        x += a * p
        r -= a * Ap
        its += 1
        if float(r @ r) <= tol2:
            x[J - 1] = 0.0
            return x, its
        if its >= max_iter:
            return np.zeros(J), -1
        z = st["inv_diagS"] * r
        rz_new = float(r @ z)
        beta = rz_new / rz if rz != 0.0 else 0.0
        p = z + beta * p
        rz = rz_new


def grounded_direct(st, rhs):
    """Exact solution of the grounded system (dense, small J only)."""
    J = st["J"]
    S = np.zeros((J, J))
    for f in range(J):
        e = np.zeros(J)
        e[f] = 1.0
        S[:, f] = apply_S(st, e)
    Jr = J - 1
    z = np.zeros(J)
    z[:Jr] = np.linalg.solve(S[:Jr, :Jr], np.asarray(rhs, dtype=np.float64)[:Jr])
    return z

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


# ---------------------------------------------------------------------------
# JLA leverages: restatement of the draw loop of akm_kss_decompose
# (src/akm_kss.cpp:2753-3160) and of its ratio estimator with the
# nonlinearity correction (:3275-3289), at the match level (working rows =
# matches in the library's order, row weight sqrt(c_m)).
# ---------------------------------------------------------------------------
_U64 = np.uint64


def _splitmix64(x):
    """SplitMix64 (src/akm_kss.cpp:212-217) on uint64 arrays, wrapping mod 2^64."""
    with np.errstate(over="ignore"):
        x = x + _U64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> _U64(27))) * _U64(0x94D049BB133111EB)
        return x ^ (x >> _U64(31))


def stream_seed(seed, tag, units):
    """The stream of (seed, draw tag, unit) for every unit (src/akm_kss.cpp:219-222)."""
    with np.errstate(over="ignore"):
        s = _splitmix64(np.array([seed], dtype=np.uint64) ^ (_U64(0xA24BAED4963EE407) * _U64(tag + 1)))
        u = np.asarray(units, dtype=np.uint64)
        return _splitmix64(s ^ (_U64(0x9FB21C651E98DF25) * (u + _U64(1))))


def row_signs(seed, draw, R):
    """The +-1 of every working row of draw d: bit r % 64 of stream (seed, 3d, r // 64)."""
    words = stream_seed(seed, 3 * draw, np.arange((R + 63) // 64))
    r = np.arange(R)
    bits = (words[r // 64] >> (r % 64).astype(np.uint64)) & _U64(1)
    return np.where(bits == 1, 1.0, -1.0)


def rademacher_sums(seed, draw, cnt):
    """Per match, the sum of cnt_m signs of stream (seed, 3d + 1, m), 64 per
    state advance (src/akm_kss.cpp:224-238)."""
    cnt = np.asarray(cnt, dtype=np.int64)
    st = stream_seed(seed, 3 * draw + 1, np.arange(cnt.size))
    acc = np.zeros(cnt.size, dtype=np.int64)
    rem = cnt.copy()
    while np.any(rem > 0):
        st = _splitmix64(st)
        k = np.minimum(rem, 64)
        live = rem > 0
        mask = np.where(k >= 64, ~_U64(0), (_U64(1) << k.clip(0, 63).astype(np.uint64)) - _U64(1))
        pc = np.bitwise_count(st & mask).astype(np.int64)
        acc += np.where(live, 2 * pc - k, 0)
        rem -= np.where(live, k, 0)
    return acc.astype(np.float64)


def solve_K(st, tw, tf):
    """K z = (tw, tf) with the ground firm pinned (src/akm_kss.cpp:1390-1403),
    the firm system solved exactly."""
    xw = tw / st["Dw"]
    rhs = tf - np.bincount(st["m_f"], weights=st["m_c"] * xw[st["m_w"]], minlength=st["J"])
    rhs[st["J"] - 1] = 0.0
    zf = grounded_direct(st, rhs)
    zw = (tw - np.bincount(st["m_w"], weights=st["m_c"] * zf[st["m_f"]], minlength=st["N"])) / st["Dw"]
    return zw, zf


def jla_leverages(st, seed, draws):
    """Match-level JLA: per row (match) pii, mii, corr and the sums bfe, bpe,
    bcov of the draws (rows are the matches of st, m_c their person-years)."""
    mw, mf, mc = st["m_w"], st["m_f"], st["m_c"]
    R = mw.size
    N, J = st["N"], st["J"]
    sw = np.sqrt(mc)
    cnt = mc.astype(np.int64)
    n_py = float(cnt.sum())
    pd = float(draws)
    scale = 1.0 / np.sqrt(pd)
    acc = {k: np.zeros(R) for k in ("Pacc", "Psq", "Macc", "Msq", "PM", "Bfe", "Bpe", "Bcov")}
    for d in range(draws):
        g = row_signs(seed, d, R)
        v = sw * g
        tw1 = np.bincount(mw, weights=v, minlength=N)
        tf1 = np.bincount(mf, weights=v, minlength=J)
        msum = rademacher_sums(seed, d, cnt)
        vbar = (msum.sum() / n_py) * scale
        su = msum * scale - vbar * cnt
        tw2 = np.bincount(mw, weights=su, minlength=N)
        tf2 = np.bincount(mf, weights=su, minlength=J)
        zw, zf = solve_K(st, tw1, tf1)
        zwf, zff = solve_K(st, np.zeros(N), tf2)
        zwp, zfp = solve_K(st, tw2, np.zeros(J))
        Z = sw * (zw[mw] + zf[mf])
        diff = g - Z
        z2, m2 = Z * Z, diff * diff
        acc["Pacc"] += z2 / pd
        acc["Psq"] += z2 * z2 / pd
        acc["Macc"] += m2 / pd
        acc["Msq"] += m2 * m2 / pd
        acc["PM"] += z2 * m2 / pd
        W2 = sw * (zwf[mw] + zff[mf])
        W1 = sw * (zwp[mw] + zfp[mf])
        acc["Bfe"] += W2 * W2
        acc["Bpe"] += W1 * W1
        acc["Bcov"] += W1 * W2
    denom = acc["Pacc"] + acc["Macc"]
    Ph = np.where(denom > 0.0, acc["Pacc"] / np.where(denom > 0.0, denom, 1.0), 0.0)
    Mh = 1.0 - Ph
    safe = np.where(Mh > 0.0, Mh, 1.0)
    Vi = (Mh * Mh * acc["Psq"] + Ph * Ph * acc["Msq"] - 2.0 * Mh * Ph * acc["PM"]) / pd
    Bi = (Mh * acc["Psq"] - Ph * acc["Msq"] + 2.0 * (Mh - Ph) * acc["PM"]) / pd
    corr = np.where(Mh > 0.0, 1.0 - Vi / (safe * safe) + Bi / safe, 0.0)
    return {"pii": Ph, "mii": Mh, "corr": corr, "bfe": acc["Bfe"], "bpe": acc["Bpe"], "bcov": acc["Bcov"]}


def match_system_from_rows(row_worker, row_firm, row_weight):
    """The match system of the reference's working rows (match level), in their
    order: workers and firms numbered by first appearance."""
    rw = np.asarray(row_worker)
    rf = np.asarray(row_firm)
    _, wi, winv = np.unique(rw, return_index=True, return_inverse=True)
    wrank = np.empty(wi.size, dtype=np.int64)
    wrank[np.argsort(wi, kind="stable")] = np.arange(wi.size)
    _, fi, finv = np.unique(rf, return_index=True, return_inverse=True)
    frank = np.empty(fi.size, dtype=np.int64)
    frank[np.argsort(fi, kind="stable")] = np.arange(fi.size)
    mw = wrank[winv].astype(np.int32)
    mf = frank[finv].astype(np.int32)
    return kss_structure(mw, mf, np.asarray(row_weight, dtype=np.float64), wi.size, fi.size)

"""Host mirror of the reference's AKM/KSS GPU solver interface.

The reference reaches its CUDA firm-system solver through
hdfe::akm::akm_cuda_* (include/hdfe/akm_kss_cuda.hpp:17-74), called from
TwoWaySolver (src/akm_kss.cpp:1154, 1323, 1675).  KssSolver wraps the same
operations of libb200fe.so: build once from the match structure, then grounded
Jacobi-PCG solves of S z = rhs, S = Df - B' Dw^{-1} B, singly or in batches of
up to max_lanes() right-hand sides.  kss_system() builds the structure from
matches exactly as TwoWaySolver::build does (src/akm_kss.cpp:1045-1092).

Failure semantics follow the reference: a lane that does not converge returns
iteration count -1 and a zero solution; CUDA or argument errors raise
AbsorberError.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .absorber import AbsorberError


def kss_system(worker, firm, weight, n_workers=None, n_firms=None) -> dict:
    """Match arrays (sorted by worker) -> the inputs of KssSolver.

    weight is the match weight (person-years of the match).  Returns m_w, m_f,
    m_c, w_ptr, f_ptr, f_matches (match ids in firm order, stable), Dw, Df and
    the Jacobi preconditioner inv_diagS (0 at the ground firm J-1).
    """
    mw = np.ascontiguousarray(worker, dtype=np.int32)
    mf = np.ascontiguousarray(firm, dtype=np.int32)
    mc = np.ascontiguousarray(weight, dtype=np.float64)
    if mw.size and np.any(np.diff(mw) < 0):
        raise ValueError("matches must be sorted by worker")
    N = int(n_workers if n_workers is not None else (mw.max() + 1 if mw.size else 0))
    J = int(n_firms if n_firms is not None else (mf.max() + 1 if mf.size else 1))
    Dw = np.bincount(mw, weights=mc, minlength=N).astype(np.float64)
    Df = np.bincount(mf, weights=mc, minlength=J).astype(np.float64)
    w_ptr = np.zeros(N + 1, dtype=np.int64)
    w_ptr[1:] = np.cumsum(np.bincount(mw, minlength=N))
    f_ptr = np.zeros(J + 1, dtype=np.int64)
    f_ptr[1:] = np.cumsum(np.bincount(mf, minlength=J))
    f_matches = np.argsort(mf, kind="stable").astype(np.int64)
    diag = Df.copy()
    np.subtract.at(diag, mf, mc * mc / Dw[mw])
    inv = np.zeros(J)
    ok = (np.arange(J) < J - 1) & (diag > 0.0)
    inv[ok] = 1.0 / diag[ok]
    return {"n_workers": N, "n_firms": J, "m_w": mw, "m_f": mf, "m_c": mc, "w_ptr": w_ptr,
            "f_ptr": f_ptr, "f_matches": f_matches, "Dw": Dw, "Df": Df, "inv_diagS": inv}


def max_lanes() -> int:
    """akm_cuda_max_lanes."""
    return int(_lib.load().b200fe_kss_max_lanes())


def stable_sort_u64(keys) -> np.ndarray:
    """akm_cuda_stable_sort_u64: input rows in ascending key order, ties stable."""
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    order = np.empty(k.size, dtype=np.int64)
    rc = _lib.load().b200fe_stable_sort_u64(k.ctypes.data, order.ctypes.data, k.size)
    if rc != _lib.OK:
        raise AbsorberError(rc, "stable sort failed")
    return order


class KssSolver:
    """akm_cuda_create / _solve_S / _solve_S_multi / _destroy over the B200 solver."""

    def __init__(self, system: dict):
        lib = _lib.load()
        self._lib = lib
        self.n_firms = int(system["n_firms"])
        self._keep = {k: np.ascontiguousarray(v) for k, v in system.items()
                      if isinstance(v, np.ndarray)}
        a = self._keep
        h = ctypes.c_void_p()
        rc = lib.b200fe_kss_create(int(system["n_workers"]), self.n_firms, a["m_w"].ctypes.data,
                                   a["m_f"].ctypes.data, a["m_c"].ctypes.data, a["m_c"].size,
                                   a["w_ptr"].ctypes.data, a["f_ptr"].ctypes.data,
                                   a["f_matches"].ctypes.data, a["Dw"].ctypes.data,
                                   a["Df"].ctypes.data, a["inv_diagS"].ctypes.data,
                                   ctypes.byref(h))
        if rc != _lib.OK:
            raise AbsorberError(rc, "b200fe_kss_create failed")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.b200fe_kss_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self) -> str:
        msg = self._lib.b200fe_kss_last_error(self._h)
        return msg.decode() if msg else ""

    def solve(self, rhs, tol: float = 1e-10, max_iter: int = 1000):
        """One grounded solve -> (z, iterations); iterations -1 if not converged."""
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        if b.shape != (self.n_firms,):
            raise ValueError("rhs must have n_firms entries")
        z = np.zeros(self.n_firms)
        it = ctypes.c_int(-1)
        rc = self._lib.b200fe_kss_solve(self._h, b.ctypes.data, z.ctypes.data, tol, max_iter,
                                        ctypes.byref(it))
        if rc not in (_lib.OK, _lib.NOT_CONVERGED):
            raise AbsorberError(rc, self._err())
        return z, int(it.value)

    def solve_multi(self, rhs_pack, tol: float = 1e-10, max_iter: int = 1000):
        """nb solves at once: rhs_pack (nb, J) -> (Z (nb, J), iterations (nb,))."""
        B = np.ascontiguousarray(rhs_pack, dtype=np.float64)
        if B.ndim != 2 or B.shape[1] != self.n_firms:
            raise ValueError("rhs_pack must be (nb, n_firms)")
        nb = B.shape[0]
        Z = np.zeros_like(B)
        its = np.full(nb, -1, dtype=np.int32)
        rc = self._lib.b200fe_kss_solve_multi(self._h, B.ctypes.data, Z.ctypes.data, nb, tol,
                                              max_iter, its.ctypes.data)
        if rc != _lib.OK:
            raise AbsorberError(rc, self._err())
        return Z, its

    def jla(self, row_w, row_f, m_cnt, n_py, *, row_sw=None, seed: int = 20260705, draws: int = 200,
            block: int = 8, tol: float = 1e-10, max_iter: int = 1000) -> dict:
        """JLA leverages of the leave-out decomposition on the device (the draw
        loop of akm_kss_decompose, src/akm_kss.cpp:2753-3160, with the ratio
        estimator :3275-3289): rows given by their worker / firm in this
        solver's numbering, in the reference's row order (it indexes the
        Rademacher streams); m_cnt the person-years of every match, n_py their
        total; row_sw the rows' sqrt match weights at match level (None: 1).
        Returns pii, mii, corr, bfe, bpe, bcov (one entry per row), the number
        of solve lanes that did not converge and the summed PCG iterations."""
        rw = np.ascontiguousarray(row_w, dtype=np.int32)
        rf = np.ascontiguousarray(row_f, dtype=np.int32)
        cnt = np.ascontiguousarray(m_cnt, dtype=np.int64)
        if rw.shape != rf.shape or rw.ndim != 1 or cnt.shape != (self._keep["m_c"].size,):
            raise ValueError("row_w / row_f must have one entry per row, m_cnt one per match")
        sw = None if row_sw is None else np.ascontiguousarray(row_sw, dtype=np.float64)
        if sw is not None and sw.shape != rw.shape:
            raise ValueError("row_sw must have one entry per row")
        R = rw.size
        out = {k: np.zeros(R) for k in ("pii", "mii", "corr", "bfe", "bpe", "bcov")}
        failed = ctypes.c_int(0)
        iters = ctypes.c_longlong(0)
        rc = self._lib.b200fe_kss_jla(
            self._h, R, rw.ctypes.data, rf.ctypes.data, None if sw is None else sw.ctypes.data,
            cnt.ctypes.data, float(n_py), int(seed) & 0xFFFFFFFFFFFFFFFF, int(draws), int(block), tol, max_iter,
            out["pii"].ctypes.data, out["mii"].ctypes.data, out["corr"].ctypes.data, out["bfe"].ctypes.data,
            out["bpe"].ctypes.data, out["bcov"].ctypes.data, ctypes.byref(failed), ctypes.byref(iters))
        if rc not in (_lib.OK, _lib.NOT_CONVERGED):
            raise AbsorberError(rc, self._err())
        out["failed_lanes"] = int(failed.value)
        out["iterations"] = int(iters.value)
        return out

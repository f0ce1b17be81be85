"""ORACLE -- test infrastructure only.

Python front of the two checkers built by oracle/Makefile:

* ``liboracle.so``          -- the plain-C restatement of the reference's
  absorber (demean_oracle.c): Irons-Tuck MAP with the honest stop, a tight
  projection for pinning, and the normal-equation certificate;
* ``_ref/libxhdfe_ref.so``  -- the reference's own CPU core compiled from its
  unmodified sources, behind ref_driver.cpp;
* ``_ref/libxhdfe_ref_cuda.so`` -- the same core with the reference's own CUDA
  backend compiled for sm_100a (target ``ref_cuda``), timed as the GPU bar;
* ``_ref/libxhdfe_ref_b200.so`` -- the same core over this repository's
  reference-side binding (the drop-in check).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, and only as the checker (never as the measured or shipped path).
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libxhdfe_ref.so"
# the reference core built with -DHDFE_USE_CUDA over the B200 library (drop-in check)
REF_B200_SO = HERE / "_ref" / "libxhdfe_ref_b200.so"
# the reference core with its own CUDA backend built for sm_100a (GPU bar)
REF_CUDA_SO = HERE / "_ref" / "libxhdfe_ref_cuda.so"

_vp, _i64, _int, _dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
_olib = None
_rlib = {}


def build_oracle() -> Path:
    if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < (HERE / "demean_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    return ORACLE_SO


def olib() -> ctypes.CDLL:
    global _olib
    if _olib is None:
        build_oracle()
        lib = ctypes.CDLL(str(ORACLE_SO))
        lib.oracle_demean_map.argtypes = [_i64, _int, _vp, _int, _vp, _vp, _vp, _vp, _dbl, _int,
                                          _int, ctypes.POINTER(_int)]
        lib.oracle_demean_map.restype = _int
        lib.oracle_sweep.argtypes = [_i64, _int, _vp, _int, _vp, _vp, _vp, _vp]
        lib.oracle_sweep.restype = None
        lib.oracle_certify.argtypes = [_i64, _int, _vp, _vp, _int, _vp, _vp, _vp,
                                       ctypes.POINTER(_dbl), ctypes.POINTER(_dbl)]
        lib.oracle_certify.restype = None
        _olib = lib
    return _olib


def _pack(y, X, fes, G, weights):
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = y.shape[0]
    X = np.zeros((n, 0)) if X is None else np.asarray(X, dtype=np.float64).reshape(n, -1)
    V = np.empty((n, 1 + X.shape[1]), dtype=np.float64, order="F")
    V[:, 0] = y
    V[:, 1:] = X
    g = np.ascontiguousarray(np.stack([np.asarray(f, dtype=np.int32) for f in fes]) if fes
                             else np.zeros((0, n), np.int32))
    Ga = np.ascontiguousarray(G, dtype=np.int32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    return V, g, Ga, w


def map_demean(y, X, fes, G, weights=None, *, tol=1e-8, max_iter=100000, accel=True,
               order=None):
    """Reference-style IT-MAP demeaning.  Returns (V~ [n, C] Fortran, iters, converged)."""
    V, g, Ga, w = _pack(y, X, fes, G, weights)
    it = _int()
    o = None if order is None else np.ascontiguousarray(order, dtype=np.int32)
    conv = olib().oracle_demean_map(V.shape[0], V.shape[1], V.ctypes.data, len(fes),
                                    g.ctypes.data, Ga.ctypes.data,
                                    None if w is None else w.ctypes.data,
                                    None if o is None else o.ctypes.data, float(tol),
                                    int(max_iter), 1 if accel else 0, ctypes.byref(it))
    return V, int(it.value), bool(conv)


def project(y, X, fes, G, weights=None, *, tol=1e-14, max_iter=200000):
    """Tightly converged within transform (the near-exact projection)."""
    return map_demean(y, X, fes, G, weights, tol=tol, max_iter=max_iter, accel=True)


def certify(V_orig, V_tilde, fes, G, weights=None):
    """(abs_residual, abs_residual_rel) of the reference's certificate."""
    Vo = np.asfortranarray(V_orig, dtype=np.float64)
    Vt = np.asfortranarray(V_tilde, dtype=np.float64)
    g = np.ascontiguousarray(np.stack([np.asarray(f, dtype=np.int32) for f in fes]))
    Ga = np.ascontiguousarray(G, dtype=np.int32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    a, r = _dbl(), _dbl()
    olib().oracle_certify(Vo.shape[0], Vo.shape[1], Vo.ctypes.data, Vt.ctypes.data, len(fes),
                          g.ctypes.data, Ga.ctypes.data, None if w is None else w.ctypes.data,
                          ctypes.byref(a), ctypes.byref(r))
    return float(a.value), float(r.value)


# ---------------------------------------------------------------------------
# The reference's own CPU core (oracle/_ref), when it was built here.
# ---------------------------------------------------------------------------
class XrefOptions(ctypes.Structure):
    _fields_ = [("tol", _dbl), ("tolerance_mode", _int), ("absorption_method", _int),
                ("num_threads", _int), ("max_iter", _int), ("drop_singletons", _int),
                ("se_type", _int), ("fit_intercept", _int), ("gpu_backend", _int),
                ("use_krylov", _int)]


TOLERANCE_MODES = {"xhdfe-fast": 0, "reghdfe-comparable": 1, "strict-residual": 2}
METHODS = {"auto": 0, "gauss-seidel": 1, "symmetric-gauss-seidel": 2, "jacobi": 3}
# "krylov": the reference's coefficient-space Jacobi-PCG absorber
# (HdfeOptions::use_krylov, src/fe_absorption.cpp:10110), CPU only
SE_TYPES = {"unadjusted": 0, "robust": 1, "cluster": 2}


def ref_available() -> bool:
    return REF_SO.exists()


def rlib(path: Path = REF_SO) -> ctypes.CDLL:
    if path not in _rlib:
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (oracle/Makefile targets 'ref', 'ref_b200')")
        lib = ctypes.CDLL(str(path))
        P = ctypes.POINTER
        lib.xref_absorb.argtypes = [_vp, _vp, _i64, _int, _vp, _int, _vp, P(XrefOptions), _vp, _vp,
                                    P(_int), P(_dbl), ctypes.c_char_p, _int]
        lib.xref_absorb.restype = _int
        lib.xref_partial_out.argtypes = [_vp, _vp, _i64, _int, _vp, _int, _vp, P(XrefOptions), _vp,
                                         _vp, _vp, P(_int), P(_dbl), ctypes.c_char_p, _int]
        lib.xref_partial_out.restype = _int
        lib.xref_fit.argtypes = [_vp, _vp, _i64, _int, _vp, _int, _vp, _vp, P(XrefOptions), _vp,
                                 _vp, P(_int), P(_dbl), ctypes.c_char_p, _int]
        lib.xref_fit.restype = _int
        if hasattr(lib, "xref_absorb_slopes"):
            lib.xref_absorb_slopes.argtypes = [_vp, _vp, _i64, _int, _vp, _int, _vp, _vp, _vp,
                                               P(XrefOptions), _vp, _vp, P(_int), P(_dbl),
                                               ctypes.c_char_p, _int]
            lib.xref_absorb_slopes.restype = _int
        if hasattr(lib, "xref_absorb_gi"):
            lib.xref_absorb_gi.argtypes = [_vp, _vp, _i64, _int, _vp, _int, _vp, _vp, _vp, _vp,
                                           _vp, _vp, _int, _i64, P(XrefOptions), _vp, _vp,
                                           P(_int), P(_dbl), ctypes.c_char_p, _int]
            lib.xref_absorb_gi.restype = _int
        if hasattr(lib, "xref_recover_fe"):
            lib.xref_recover_fe.argtypes = [_vp, _i64, _vp, _int, _vp, P(XrefOptions), _dbl, _vp,
                                            P(_int), P(_dbl), ctypes.c_char_p, _int]
            lib.xref_recover_fe.restype = _int
        if hasattr(lib, "xref_run_ols"):
            lib.xref_run_ols.argtypes = [_vp, _vp, _i64, _int, _vp, _vp, _int, _dbl, _dbl, _dbl, _int,
                                         _vp, _vp, _vp, _vp, ctypes.c_char_p, _int]
            lib.xref_run_ols.restype = _int
        if hasattr(lib, "xref_components"):
            lib.xref_components.argtypes = [_vp, _vp, _i64, _vp, P(_int), P(ctypes.c_longlong),
                                            P(_dbl), ctypes.c_char_p, _int]
            lib.xref_components.restype = _int
        if hasattr(lib, "xref_schwarz_demean_raw"):
            lib.xref_schwarz_demean_raw.argtypes = [_vp, _vp, _i64, _int, _vp, _int, _vp, _int, _dbl,
                                                    _int, P(_int)]
            lib.xref_schwarz_demean_raw.restype = _int
        if hasattr(lib, "xref_akm_kss"):
            lib.xref_akm_kss.argtypes = [_vp, _vp, _vp, _i64, _vp, ctypes.c_uint64, _dbl, _vp, P(_int),
                                         P(ctypes.c_longlong), ctypes.c_char_p, _int]
            lib.xref_akm_kss.restype = _int
        _rlib[path] = lib
    return _rlib[path]


GPU_BACKENDS = {"default": 0, "cpu": 1, "cuda": 2}


def _xopts(tol, tolerance_mode, method, threads, max_iter=0, drop_singletons=True,
           se_type="unadjusted", fit_intercept=True, gpu_backend="default"):
    o = XrefOptions()
    o.tol = tol
    o.tolerance_mode = TOLERANCE_MODES[tolerance_mode]
    o.absorption_method = METHODS["auto" if method == "krylov" else method]
    o.use_krylov = 1 if method == "krylov" else 0
    o.num_threads = threads
    o.max_iter = max_iter
    o.drop_singletons = 1 if drop_singletons else 0
    o.se_type = SE_TYPES[se_type]
    o.fit_intercept = 1 if fit_intercept else 0
    o.gpu_backend = GPU_BACKENDS[gpu_backend]
    return o


def ref_absorb(y, X, fes, weights=None, *, tol=1e-8, tolerance_mode="reghdfe-comparable",
               method="auto", threads=1, max_iter=0, gpu_backend="default", lib_path=REF_SO):
    """Reference absorb_fixed_effects_v6 (raw ids, no singleton drop)."""
    V, g, _, w = _pack(y, X, fes, [1] * len(fes), weights)
    n, C = V.shape
    Vo = np.empty_like(V, order="F")
    info = (_int * 8)()
    dinfo = (_dbl * 2)()
    err = ctypes.create_string_buffer(512)
    o = _xopts(tol, tolerance_mode, method, threads, max_iter, gpu_backend=gpu_backend)
    rc = rlib(lib_path).xref_absorb(V[:, 0].ctypes.data, V[:, 1:].ctypes.data if C > 1 else None, n, C - 1,
                            g.ctypes.data, len(fes), None if w is None else w.ctypes.data,
                            ctypes.byref(o), Vo[:, 0].ctypes.data,
                            Vo[:, 1:].ctypes.data if C > 1 else None, info, dinfo, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return {"V": Vo, "iterations": info[0], "converged": bool(info[1]),
            "precision_certified": bool(info[2]), "gpu_status_code": info[3],
            "abs_residual": dinfo[0], "abs_residual_rel": dinfo[1]}


def ref_absorb_slopes(y, X, fes, slopes, weights=None, *, tol=1e-8,
                      tolerance_mode="reghdfe-comparable", method="auto", threads=1, max_iter=0,
                      gpu_backend="default", lib_path=REF_SO):
    """Reference absorb_fixed_effects_v6 with heterogeneous slopes.

    ``slopes``: list of (fe_index, values, include_intercept), the fields of
    the reference's HeterogeneousSlopeTerm (include/fe_absorption.hpp:49-53).
    """
    V, g, _, w = _pack(y, X, fes, [1] * len(fes), weights)
    n, C = V.shape
    kind = np.zeros(len(fes), dtype=np.int32)
    zf = np.zeros((len(fes), n), dtype=np.float64)
    for d, z, icpt in slopes:
        kind[d] = 2 if icpt else 1
        zf[d] = np.asarray(z, dtype=np.float64)
    Vo = np.empty_like(V, order="F")
    info = (_int * 8)()
    dinfo = (_dbl * 2)()
    err = ctypes.create_string_buffer(512)
    o = _xopts(tol, tolerance_mode, method, threads, max_iter, gpu_backend=gpu_backend)
    rc = rlib(lib_path).xref_absorb_slopes(
        V[:, 0].ctypes.data, V[:, 1:].ctypes.data if C > 1 else None, n, C - 1, g.ctypes.data,
        len(fes), None if w is None else w.ctypes.data, zf.ctypes.data, kind.ctypes.data,
        ctypes.byref(o), Vo[:, 0].ctypes.data, Vo[:, 1:].ctypes.data if C > 1 else None, info,
        dinfo, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return {"V": Vo, "iterations": info[0], "converged": bool(info[1]),
            "precision_certified": bool(info[2]), "gpu_status_code": info[3],
            "abs_residual": dinfo[0], "abs_residual_rel": dinfo[1]}


def ref_absorb_gi(y, X, fes, gi, weights=None, *, tol=1e-8, tolerance_mode="reghdfe-comparable",
                  method="auto", threads=1, max_iter=0, gpu_backend="default", lib_path=REF_SO):
    """Reference absorb_fixed_effects_group_individual.  ``gi`` has the fields of
    the reference's GroupIndividualStructure (group_ptr, group_individual,
    individual_ptr, individual_group, group_scale, num_individuals)."""
    V, g, _, w = _pack(y, X, fes, [1] * len(fes), weights)
    n, C = V.shape
    a = [np.ascontiguousarray(x, dtype=np.int32) for x in
         (gi.group_ptr, gi.group_individual, gi.individual_ptr, gi.individual_group)]
    sc = np.ascontiguousarray(gi.group_scale, dtype=np.float64)
    Vo = np.empty_like(V, order="F")
    info = (_int * 8)()
    dinfo = (_dbl * 2)()
    err = ctypes.create_string_buffer(512)
    o = _xopts(tol, tolerance_mode, method, threads, max_iter, gpu_backend=gpu_backend)
    rc = rlib(lib_path).xref_absorb_gi(
        V[:, 0].ctypes.data, V[:, 1:].ctypes.data if C > 1 else None, n, C - 1, g.ctypes.data,
        len(fes), None if w is None else w.ctypes.data, *[x.ctypes.data for x in a],
        sc.ctypes.data, int(gi.num_individuals), int(a[1].shape[0]), ctypes.byref(o),
        Vo[:, 0].ctypes.data, Vo[:, 1:].ctypes.data if C > 1 else None, info, dinfo, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return {"V": Vo, "iterations": info[0], "converged": bool(info[1]),
            "precision_certified": bool(info[2]), "gpu_status_code": info[3],
            "abs_residual": dinfo[0], "abs_residual_rel": dinfo[1]}


def ref_partial_out(y, X, fes, weights=None, *, tol=1e-8, tolerance_mode="reghdfe-comparable",
                    threads=1, drop_singletons=True, gpu_backend="default", lib_path=REF_SO):
    V, g, _, w = _pack(y, X, fes, [1] * len(fes), weights)
    n, C = V.shape
    Vo = np.zeros_like(V, order="F")
    idx = np.zeros(n, dtype=np.int32)
    info = (_int * 8)()
    dinfo = (_dbl * 2)()
    err = ctypes.create_string_buffer(512)
    o = _xopts(tol, tolerance_mode, "auto", threads, 0, drop_singletons, gpu_backend=gpu_backend)
    rc = rlib(lib_path).xref_partial_out(V[:, 0].ctypes.data, V[:, 1:].ctypes.data if C > 1 else None, n,
                                 C - 1, g.ctypes.data, len(fes),
                                 None if w is None else w.ctypes.data, ctypes.byref(o),
                                 Vo[:, 0].ctypes.data, Vo[:, 1:].ctypes.data if C > 1 else None,
                                 idx.ctypes.data, info, dinfo, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    kept = info[3]
    # partial_out writes kept rows contiguously into each output column of length n
    Vk = np.empty((kept, C), order="F")
    Vk[:, 0] = Vo[:kept, 0]
    if C > 1:
        flat = Vo[:, 1:].ravel(order="F")[: kept * (C - 1)]
        Vk[:, 1:] = flat.reshape((kept, C - 1), order="F")
    return {"V": Vk, "sample_index": idx[:kept].copy(), "iterations": info[0],
            "converged": bool(info[1]), "precision_certified": bool(info[2]),
            "gpu_status_code": info[4],
            "abs_residual": dinfo[0], "abs_residual_rel": dinfo[1]}


def ref_fit(y, X, fes, weights=None, cluster=None, *, tol=1e-8,
            tolerance_mode="reghdfe-comparable", threads=1, se_type=None, fit_intercept=False,
            drop_singletons=True, gpu_backend="default", lib_path=REF_SO):
    V, g, _, w = _pack(y, X, fes, [1] * len(fes), weights)
    n, C = V.shape
    k = C - 1
    coef = np.zeros(k + 2)
    se = np.zeros(k + 2)
    info = (_int * 8)()
    dinfo = (_dbl * 4)()
    err = ctypes.create_string_buffer(512)
    st = se_type or ("cluster" if cluster is not None else "unadjusted")
    o = _xopts(tol, tolerance_mode, "auto", threads, 0, drop_singletons, st, fit_intercept,
               gpu_backend)
    cl = None if cluster is None else np.ascontiguousarray(cluster, dtype=np.int32)
    rc = rlib(lib_path).xref_fit(V[:, 0].ctypes.data, V[:, 1:].ctypes.data, n, k, g.ctypes.data, len(fes),
                         None if w is None else w.ctypes.data,
                         None if cl is None else cl.ctypes.data, ctypes.byref(o),
                         coef.ctypes.data, se.ctypes.data, info, dinfo, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    p = info[5]
    return {"coef": coef[:p].copy(), "se": se[:p].copy(), "iterations": info[0],
            "converged": bool(info[1]), "precision_certified": bool(info[2]), "nobs": info[3],
            "num_singletons": info[4], "gpu_status_code": info[6],
            "abs_residual_rel": dinfo[0], "rss": dinfo[1],
            "r2_within": dinfo[2], "df_a": dinfo[3]}


LEVERAGE = {"auto": 0, "exact": 1, "jla": 2}


def ref_akm_kss(y, worker, firm, *, leverages="auto", jla_draws=0, seed=20260705, cg_tol=1e-10,
                direct_max_firms=-1, use_gpu=False, threads=0, cg_max_iter=0, lib_path=REF_SO):
    """The reference's hdfe::akm::akm_kss_decompose (include/hdfe/akm_kss.hpp:227-233)
    on raw worker/firm ids, no controls.  use_gpu routes its PCG solves to the
    CUDA backend the library was linked with (only the ref_b200 build has one)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    w = np.ascontiguousarray(worker, dtype=np.int32)
    f = np.ascontiguousarray(firm, dtype=np.int32)
    opts = np.array([LEVERAGE[leverages], jla_draws, direct_max_firms, int(use_gpu), threads,
                     cg_max_iter], dtype=np.int32)
    out = np.zeros(16)
    info = (_int * 8)()
    iters = ctypes.c_longlong(0)
    err = ctypes.create_string_buffer(512)
    rc = rlib(lib_path).xref_akm_kss(y.ctypes.data, w.ctypes.data, f.ctypes.data, len(y),
                                    opts.ctypes.data, seed, cg_tol, out.ctypes.data, info,
                                    ctypes.byref(iters), err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    names = ["var_alpha", "var_psi", "cov_alpha_psi"]
    return {"plugin": dict(zip(names, out[0:3])), "agsu": dict(zip(names, out[3:6])),
            "kss": dict(zip(names, out[6:9])), "var_y": out[9], "sigma2_ho": out[10],
            "mean_pii": out[11], "max_pii": out[12], "n_obs": int(out[13]),
            "n_workers": info[0], "n_firms": info[1], "n_matches": info[2],
            "gpu_used": bool(info[3]), "gpu_status_code": info[4], "solver_direct": bool(info[5]),
            "converged": bool(info[6]), "jla_draws_used": info[7],
            "solver_iterations": int(iters.value)}


def ref_akm_kss_rows(y, worker, firm, *, leverages="jla", jla_draws=0, seed=20260705, cg_tol=1e-10,
                     direct_max_firms=-1, threads=0, cg_max_iter=0, lib_path=REF_SO):
    """The working rows of the reference's akm_kss_decompose
    (include/hdfe/akm_kss.hpp:120-124, 227-233), in its row order: pii,
    original worker and firm ids, person-year weight."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    w = np.ascontiguousarray(worker, dtype=np.int32)
    f = np.ascontiguousarray(firm, dtype=np.int32)
    opts = np.array([LEVERAGE[leverages], jla_draws, direct_max_firms, 0, threads, cg_max_iter],
                    dtype=np.int32)
    cap = len(y)
    pii = np.zeros(cap)
    rw = np.zeros(cap, dtype=np.int32)
    rf = np.zeros(cap, dtype=np.int32)
    wt = np.zeros(cap)
    nr = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(512)
    lib = rlib(lib_path)
    lib.xref_akm_kss_rows.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_void_p, ctypes.c_uint64,
                                      ctypes.c_double, ctypes.c_int64] + [ctypes.c_void_p] * 5 + \
        [ctypes.c_char_p, ctypes.c_int]
    lib.xref_akm_kss_rows.restype = ctypes.c_int
    rc = lib.xref_akm_kss_rows(y.ctypes.data, w.ctypes.data, f.ctypes.data, len(y), opts.ctypes.data, seed,
                               cg_tol, cap, pii.ctypes.data, rw.ctypes.data, rf.ctypes.data, wt.ctypes.data,
                               ctypes.byref(nr), err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    R = nr.value
    return {"pii": pii[:R].copy(), "row_worker": rw[:R].copy(), "row_firm": rf[:R].copy(),
            "row_weight": wt[:R].copy()}


def ref_recover_fe(partial, fes, weights=None, *, tol=1e-8, fe_tolerance=0.0, threads=1,
                   gpu_backend="default", lib_path=REF_SO):
    """The reference's recover_fixed_effects (include/fe_absorption.hpp:127-130):
    per-dim FE contributions of ``partial`` (n x dims), iterations, converged,
    max_delta."""
    pv = np.ascontiguousarray(partial, dtype=np.float64)
    n = pv.shape[0]
    g = np.ascontiguousarray(np.stack([np.asarray(f, dtype=np.int32) for f in fes]))
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    contrib = np.zeros((len(fes), n))
    info = (_int * 2)()
    dinfo = (_dbl * 1)()
    err = ctypes.create_string_buffer(512)
    o = _xopts(tol, "reghdfe-comparable", "auto", threads, gpu_backend=gpu_backend)
    rc = rlib(lib_path).xref_recover_fe(pv.ctypes.data, n, g.ctypes.data, len(fes),
                                        None if w is None else w.ctypes.data, ctypes.byref(o),
                                        fe_tolerance, contrib.ctypes.data, info, dinfo, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return {"contributions": contrib, "iterations": info[0], "converged": bool(info[1]),
            "max_delta": dinfo[0]}


SE_CODES = {"unadjusted": 0, "robust": 1, "cluster": 2}


def ref_run_ols(y, X, weights=None, clusters=None, *, se_type="unadjusted", tss=0.0,
                within_tss=0.0, n_effective=-1.0, weights_are_frequencies=False, lib_path=REF_SO):
    """The reference's hdfe::detail::run_ols (include/ols.hpp:40-51)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    X = np.asfortranarray(X, dtype=np.float64)
    n, p = X.shape
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    c = None if clusters is None else np.ascontiguousarray(clusters, dtype=np.int32)
    coef, se = np.zeros(p), np.zeros(p)
    cov = np.zeros((p, p), order="F")
    sc = np.zeros(8)
    err = ctypes.create_string_buffer(512)
    rc = rlib(lib_path).xref_run_ols(y.ctypes.data, X.ctypes.data, n, p,
                                    None if w is None else w.ctypes.data,
                                    None if c is None else c.ctypes.data, SE_CODES[se_type], tss,
                                    within_tss, n_effective, int(weights_are_frequencies),
                                    coef.ctypes.data, se.ctypes.data, cov.ctypes.data,
                                    sc.ctypes.data, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return {"coef": coef, "se": se, "cov": cov, "rss": sc[0], "sigma2": sc[1], "df_resid": sc[2],
            "cov_scale": sc[3], "cluster_u2": sc[4], "r2": sc[5], "r2_within": sc[6],
            "num_clusters": int(sc[7])}


def ref_schwarz_demean_raw(y, X, fes, levels, *, tol=1e-10, max_iter=10000, threads=1,
                           lib_path=REF_SO):
    """xhdfe::schwarz_demean_raw of the given build (the reference's CPU block
    PCG in libxhdfe_ref.so; the B200 absorber through the binding in
    libxhdfe_ref_b200.so).  Returns (ok, V (n x (1+k)), iterations)."""
    y = np.array(y, dtype=np.float64, copy=True)
    X = np.asfortranarray(np.array(X, dtype=np.float64, copy=True))
    n, k = y.size, X.shape[1]
    g = np.ascontiguousarray(np.concatenate([np.asarray(f, dtype=np.int32) for f in fes]))
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    its = _int(0)
    ok = rlib(lib_path).xref_schwarz_demean_raw(y.ctypes.data, X.ctypes.data if k else None, n, k,
                                                g.ctypes.data, len(fes), lv.ctypes.data, threads,
                                                tol, max_iter, ctypes.byref(its))
    return bool(ok), np.column_stack([y, X]), int(its.value)


def ref_components(fe1, fe2, weights=None, lib_path=REF_SO):
    """The reference's compute_first_pair_component_stats."""
    a = np.ascontiguousarray(fe1, dtype=np.int32)
    b = np.ascontiguousarray(fe2, dtype=np.int32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    oi = (_int * 1)()
    ol = (ctypes.c_longlong * 1)()
    od = (_dbl * 2)()
    err = ctypes.create_string_buffer(512)
    rc = rlib(lib_path).xref_components(a.ctypes.data, b.ctypes.data, a.size,
                                       None if w is None else w.ctypes.data, oi, ol, od, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return {"num_components": oi[0], "largest_component_n_obs": int(ol[0]),
            "largest_component_obs_share": od[0], "largest_component_weight_share": od[1]}

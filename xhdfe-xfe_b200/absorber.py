"""Host-side absorber interface, mirroring the reference's absorber calls.

Reference counterparts (reisportela/xhdfe-xfe):

* ``Absorber.absorb``         -> hdfe::detail::absorb_fixed_effects_cuda
                                 (include/fe_absorption_cuda.hpp:127-134)
* ``HeterogeneousSlopeTerm``  -> the struct of the same name (include/fe_absorption.hpp:49-53);
                                 ``Absorber.absorb(slopes=...)`` is the is_slope path of
                                 absorb_fixed_effects_cuda (src/fe_absorption_cuda.cu:2316)
* ``Absorber.absorb_group_individual`` -> absorb_fixed_effects_group_individual_cuda
                                 (include/fe_absorption_cuda.hpp:136-145);
                                 ``GroupIndividualStructure`` / ``build_group_individual``
                                 -> the reference's structure and its builder
                                 (src/hdfe_regressor_v11.cpp:5780-5920)
* ``absorb_fixed_effects``    -> hdfe::detail::absorb_fixed_effects_v6 with the
                                 CUDA backend (src/fe_absorption.cpp:8750, GPU
                                 dispatch :9203-9237): raw ids are ranked densely
                                 as build_indexer does (:845-940)
* ``partial_out``             -> HdfeRegressorV11::partial_out
                                 (src/hdfe_regressor_v11.cpp:10275): singleton
                                 drop, then absorption
* ``demean_raw``              -> xhdfe::schwarz_demean_raw (include/schwarz_demean.hpp:30)
* ``fe_recovery_max_delta``   -> fe_recovery_max_delta_cuda (fe_absorption_cuda.hpp:152)
* ``cuda_backend_available``  -> cuda_backend_available (fe_absorption_cuda.hpp:125)

Failure semantics follow the reference: a CUDA or argument failure raises
(the reference returns false and its callers fail closed); non-convergence
returns a result with ``converged == False``.  Nothing here computes on the
CPU: every call goes through libb200fe.so.
"""

from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _lib

TOLERANCE_MODES = {"xhdfe-fast": 0, "reghdfe-comparable": 1, "strict-residual": 2}
PRECISIONS = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}


@dataclass
class HeterogeneousSlopeTerm:
    """A slope on FE dimension ``fe_index`` with per-observation ``values``;
    ``include_intercept`` keeps the group intercept in the same block
    (the reference's struct of the same name, include/fe_absorption.hpp:49-53).
    Tuples (fe_index, values, include_intercept) are accepted wherever a list
    of terms is."""
    fe_index: int
    values: np.ndarray
    include_intercept: bool = False


@dataclass
class GroupIndividualStructure:
    """The reference's GroupIndividualStructure (include/fe_absorption.hpp:13-21):
    rows of the data are groups; CSR lists of the individuals of every group
    and of the groups of every individual; group_scale per group (1 for sum
    aggregation, 1 / group size for mean)."""
    num_groups: int
    num_individuals: int
    group_ptr: np.ndarray
    group_individual: np.ndarray
    individual_ptr: np.ndarray
    individual_group: np.ndarray
    group_scale: np.ndarray


def build_group_individual(group_ids, individual_ids, aggregation: str = "mean"
                           ) -> tuple[GroupIndividualStructure, np.ndarray, np.ndarray]:
    """Build the structure from edge-level data, one (group, individual) pair
    per edge, as the reference's builder does (src/hdfe_regressor_v11.cpp:
    5780-5920): groups and individuals ranked densely by value, edges sorted by
    (group, individual), a repeated pair is an error, mean aggregation scales
    a group by 1 / its number of individuals.  Returns the structure and the
    group and individual values in dense order."""
    g_raw = np.asarray(group_ids)
    i_raw = np.asarray(individual_ids)
    if g_raw.shape != i_raw.shape or g_raw.ndim != 1 or g_raw.size == 0:
        raise ValueError("group_ids and individual_ids must be non-empty vectors of one length")
    g_vals, g = np.unique(g_raw, return_inverse=True)
    i_vals, ind = np.unique(i_raw, return_inverse=True)
    G, I = g_vals.size, i_vals.size
    key = g.astype(np.int64) * I + ind
    order = np.argsort(key, kind="stable")
    ks = key[order]
    if np.any(ks[1:] == ks[:-1]):
        raise ValueError("group_ids and individual_ids do not uniquely identify the observations")
    ge, ie = (ks // I).astype(np.int32), (ks % I).astype(np.int32)
    group_ptr = np.zeros(G + 1, dtype=np.int32)
    np.cumsum(np.bincount(ge, minlength=G), out=group_ptr[1:])
    individual_ptr = np.zeros(I + 1, dtype=np.int32)
    np.cumsum(np.bincount(ie, minlength=I), out=individual_ptr[1:])
    by_ind = np.argsort(ie, kind="stable")  # groups ascending within an individual
    if aggregation == "mean":
        scale = 1.0 / np.diff(group_ptr).astype(np.float64)
    elif aggregation == "sum":
        scale = np.ones(G)
    else:
        raise ValueError("aggregation must be 'mean' or 'sum'")
    gi = GroupIndividualStructure(G, I, group_ptr, ie.copy(), individual_ptr,
                                  ge[by_ind].copy(), scale)
    return gi, g_vals, i_vals


def _slope_table(slopes, num_dims: int, n: int):
    """Per-dim slope values (or None) and intercept flags from a term list."""
    vals = [None] * num_dims
    icpt = np.ones(num_dims, dtype=np.uint8)
    for t in slopes:
        d, z, inc = (t.fe_index, t.values, t.include_intercept) if isinstance(
            t, HeterogeneousSlopeTerm) else t
        d = int(d)
        if d < 0 or d >= num_dims:
            raise ValueError("Heterogeneous slope FE index out of range")
        if vals[d] is not None:
            raise ValueError("at most one slope term per FE dimension")
        z = np.ascontiguousarray(z, dtype=np.float64)
        if z.shape != (n,):
            raise ValueError("slope values must have the same length as y")
        vals[d] = z
        icpt[d] = 1 if inc else 0
    return vals, icpt


class AbsorberError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"b200fe: {_lib.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


@dataclass
class AbsorptionResult:
    """Fields of hdfe::detail::AbsorptionResult (include/fe_absorption.hpp:23-47)."""
    y_tilde: np.ndarray
    X_tilde: np.ndarray
    iterations: int = 0
    converged: bool = True
    abs_residual: float = 0.0
    abs_residual_rel: float = 0.0
    precision_certified: bool = True
    fe_levels: list = field(default_factory=list)
    gpu_used: bool = True
    gpu_status_code: int = 1
    gpu_attempted: bool = True
    gpu_absorption_converged: bool = True
    gpu_absorption_iterations: int = 0
    # diagnostics of this implementation
    outer_iterations: int = 0
    rel_residual: float = 0.0
    primary_dim: int = -1
    setup_ms: float = 0.0
    solve_ms: float = 0.0
    h2d_ms: float = 0.0
    d2h_ms: float = 0.0
    kernel_launches: int = 0
    # options.profile: per kernel category (_lib.PROF_NAMES) CUDA-event ms,
    # algorithmic bytes and launches
    prof_ms: list = field(default_factory=list)
    prof_bytes: list = field(default_factory=list)
    prof_launches: list = field(default_factory=list)
    sample_index: np.ndarray | None = None
    # saved FEs (save_fe=True): per dim, [G_d, 1 + k] coefficients, column 0 for
    # y -- the fe_alpha_y / fe_alpha_X of the reference's retain_fixed_effects
    fe: list | None = None

    @property
    def fe_alpha_y(self):
        return None if self.fe is None else [a[:, 0] for a in self.fe]

    @property
    def fe_alpha_X(self):
        return None if self.fe is None else [a[:, 1:] for a in self.fe]


def cuda_backend_available() -> bool:
    return bool(_lib.load().b200fe_device_available())


def make_options(*, tol=1e-8, tolerance_mode="reghdfe-comparable", precision="mixed",
                 max_iter=10000, certify=True, check_interval=4, reuse_structure=False,
                 inner_tol=1e-5, max_outer=12, profile=False,
                 pass_kernel=0, fe_linf_tol=0.0) -> _lib.Options:
    o = _lib.default_options()
    o.tol = float(tol)
    o.tolerance_mode = TOLERANCE_MODES[tolerance_mode] if isinstance(tolerance_mode, str) \
        else int(tolerance_mode)
    o.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    o.max_iter = int(max_iter)
    o.certify = 1 if certify else 0
    o.check_interval = int(check_interval)
    o.reuse_structure = 1 if reuse_structure else 0
    o.inner_tol = float(inner_tol)
    o.max_outer = int(max_outer)
    o.profile = 1 if profile else 0
    # "auto": the form tuned for the call's dims and rows (autotune.py's table),
    # resolved by Absorber.absorb / absorb_device before the library is called
    o.pass_kernel = PASS_KERNEL_AUTO if pass_kernel == "auto" else int(pass_kernel)
    o.fe_linf_tol = float(fe_linf_tol)
    return o


PASS_KERNEL_AUTO = -1


def _resolve_options(o, num_dims: int, n: int):
    """A copy of options o with pass_kernel "auto" replaced by the tuned form."""
    if o is None or o.pass_kernel != PASS_KERNEL_AUTO:
        return o
    from .autotune import choose_pass_kernel
    r = _lib.Options()
    ctypes.pointer(r)[0] = o
    r.pass_kernel = choose_pass_kernel(num_dims, n)
    return r


def _ptr_array(ptrs):
    arr = (ctypes.c_void_p * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


def dense_ids(ids: np.ndarray) -> tuple[np.ndarray, int]:
    """Dense 0..G-1 ranking of nonnegative ids (build_indexer's rule)."""
    ids = np.asarray(ids)
    if ids.size and ids.min() < 0:
        raise ValueError("fixed-effect IDs must be nonnegative")
    if ids.size == 0:
        return ids.astype(np.int32), 0
    mx = int(ids.max())
    if mx < 4 * ids.size + 1024:
        present = np.bincount(ids.astype(np.int64), minlength=mx + 1) > 0
        remap = np.cumsum(present) - 1
        return remap[ids].astype(np.int32), int(present.sum())
    uniq, inv = np.unique(ids, return_inverse=True)
    return inv.astype(np.int32), int(uniq.size)


class Absorber:
    """One CUDA context (stream + device workspace), like the reference's
    thread-local CUDA workspace (src/fe_absorption_cuda.cu:1536)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self.lib.b200fe_context_create(int(device), ctypes.byref(h))
        if rc != _lib.OK:
            raise AbsorberError(rc, "cannot create a CUDA context")
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.b200fe_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc):
        msg = self.lib.b200fe_last_error(self.handle)
        return AbsorberError(rc, msg.decode() if msg else "")

    @property
    def stream_handle(self) -> int:
        return int(self.lib.b200fe_context_stream(self.handle) or 0)

    def absorb(self, y, X, group_ids, num_groups, weights=None, options=None,
               y_out=None, X_out=None, save_fe=False, slopes=None) -> AbsorptionResult:
        """Absorb host arrays with dense ids (absorb_fixed_effects_cuda).  With
        save_fe the result carries the FE coefficients (``fe``).  ``slopes``:
        heterogeneous slope terms (GpuFeInput.is_slope); saved FEs are not
        available with slopes."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.shape[0]
        X = np.zeros((n, 0)) if X is None else np.asarray(X, dtype=np.float64)
        if X.ndim == 1:
            X = X[:, None]
        X = np.asfortranarray(X)
        k = X.shape[1]
        if X.shape[0] != n:
            raise ValueError("X must have the same number of rows as y")
        gids = [np.ascontiguousarray(g, dtype=np.int32) for g in group_ids]
        for g in gids:
            if g.shape[0] != n:
                raise ValueError("each fixed-effect vector must have the same length as y")
        G = np.ascontiguousarray(num_groups, dtype=np.int32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        if y_out is None:
            y_out = np.empty_like(y)
        if X_out is None:
            X_out = np.empty((n, k), dtype=np.float64, order="F")
        o = _resolve_options(options or make_options(), len(gids), n)
        r = _lib.Result()
        if slopes:
            if save_fe:
                raise ValueError("saved fixed effects are not available with heterogeneous slopes")
            zv, icpt = _slope_table(slopes, len(gids), n)
            for z in zv:
                if z is not None:
                    _check_finite(z, "slope values")
            rc = self.lib.b200fe_absorb_slopes(
                self.handle, y.ctypes.data, X.ctypes.data if k else None, n, k, len(gids),
                _ptr_array([g.ctypes.data for g in gids]), G.ctypes.data,
                _ptr_array([z.ctypes.data if z is not None else None for z in zv]),
                icpt.ctypes.data, None if w is None else w.ctypes.data, ctypes.byref(o),
                y_out.ctypes.data, X_out.ctypes.data if k else None, ctypes.byref(r))
            if rc not in (_lib.OK, _lib.NOT_CONVERGED):
                raise self._err(rc)
            return _to_result(r, y_out, X_out, G)
        fe = [np.zeros((int(g), k + 1), order="F") for g in G] if save_fe else None
        rc = self.lib.b200fe_absorb_fe(
            self.handle, y.ctypes.data, X.ctypes.data if k else None, n, k, len(gids),
            _ptr_array([g.ctypes.data for g in gids]), G.ctypes.data,
            None if w is None else w.ctypes.data, ctypes.byref(o), y_out.ctypes.data,
            X_out.ctypes.data if k else None,
            _ptr_array([a.ctypes.data for a in fe]) if fe else None, ctypes.byref(r))
        if rc not in (_lib.OK, _lib.NOT_CONVERGED):
            raise self._err(rc)
        res = _to_result(r, y_out, X_out, G)
        res.fe = fe
        return res

    def absorb_device(self, v, group_ids, num_groups, weights=None, options=None, out=None,
                      stream=None):
        """Absorb device tensors (torch, float64 (cols, n) contiguous = column-major
        n x cols; int32 group ids).  Returns (out, _lib.Result)."""
        import torch
        if v.dtype != torch.float64 or not v.is_cuda or v.dim() != 2 or not v.is_contiguous():
            raise ValueError("v must be a contiguous float64 CUDA tensor of shape (cols, n)")
        cols, n = v.shape
        if out is None:
            out = torch.empty_like(v)
        for g in group_ids:
            if g.dtype != torch.int32 or not g.is_cuda or g.numel() != n:
                raise ValueError("group ids must be int32 CUDA tensors of length n")
        G = np.ascontiguousarray(num_groups, dtype=np.int32)
        o = _resolve_options(options or make_options(), len(group_ids), n)
        r = _lib.Result()
        rc = self.lib.b200fe_absorb_device(
            self.handle, v.data_ptr(), n, cols, len(group_ids),
            _ptr_array([g.data_ptr() for g in group_ids]), G.ctypes.data,
            None if weights is None else weights.data_ptr(), ctypes.byref(o), out.data_ptr(),
            ctypes.byref(r), stream)
        if rc not in (_lib.OK, _lib.NOT_CONVERGED):
            raise self._err(rc)
        return out, r

    def absorb_group_individual(self, y, X, group_ids, num_groups, gi, weights=None,
                                options=None, y_out=None, X_out=None) -> AbsorptionResult:
        """Absorb the standard FE dims (dense ids; may be empty) and the
        individual FEs of ``gi`` (a GroupIndividualStructure; rows = groups),
        absorb_fixed_effects_group_individual_cuda."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.shape[0]
        X = np.zeros((n, 0)) if X is None else np.asarray(X, dtype=np.float64)
        if X.ndim == 1:
            X = X[:, None]
        X = np.asfortranarray(X)
        k = X.shape[1]
        if X.shape[0] != n or int(gi.num_groups) != n:
            raise ValueError("y, X and the group/individual structure must have one row per group")
        gids = [np.ascontiguousarray(g, dtype=np.int32) for g in group_ids]
        G = np.ascontiguousarray(num_groups, dtype=np.int32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in
                (gi.group_ptr, gi.group_individual, gi.individual_ptr, gi.individual_group)]
        sc = np.ascontiguousarray(gi.group_scale, dtype=np.float64)
        _check_finite(sc, "group_scale")
        st = _lib.GroupIndividual(int(gi.num_individuals), int(arrs[1].shape[0]),
                                  *[a.ctypes.data for a in arrs], sc.ctypes.data)
        if y_out is None:
            y_out = np.empty_like(y)
        if X_out is None:
            X_out = np.empty((n, k), dtype=np.float64, order="F")
        o = _resolve_options(options or make_options(), len(group_ids), n)
        r = _lib.Result()
        rc = self.lib.b200fe_absorb_group_individual(
            self.handle, y.ctypes.data, X.ctypes.data if k else None, n, k, len(gids),
            _ptr_array([g.ctypes.data for g in gids]), G.ctypes.data, ctypes.byref(st),
            None if w is None else w.ctypes.data, ctypes.byref(o), y_out.ctypes.data,
            X_out.ctypes.data if k else None, ctypes.byref(r))
        if rc not in (_lib.OK, _lib.NOT_CONVERGED):
            raise self._err(rc)
        res = _to_result(r, y_out, X_out, G)
        res.fe_levels = [int(x) for x in G] + [int(gi.num_individuals)]
        return res

    def absorb_slopes_device(self, v, group_ids, num_groups, slopes, weights=None,
                             options=None, out=None, stream=None):
        """absorb_device with heterogeneous slopes; the terms' values are
        float64 CUDA tensors of length n.  Returns (out, _lib.Result)."""
        import torch
        if v.dtype != torch.float64 or not v.is_cuda or v.dim() != 2 or not v.is_contiguous():
            raise ValueError("v must be a contiguous float64 CUDA tensor of shape (cols, n)")
        cols, n = v.shape
        if out is None:
            out = torch.empty_like(v)
        for g in group_ids:
            if g.dtype != torch.int32 or not g.is_cuda or g.numel() != n:
                raise ValueError("group ids must be int32 CUDA tensors of length n")
        zp = [None] * len(group_ids)
        icpt = np.ones(len(group_ids), dtype=np.uint8)
        for t in slopes:
            d, z, inc = (t.fe_index, t.values, t.include_intercept) if isinstance(
                t, HeterogeneousSlopeTerm) else t
            if not 0 <= int(d) < len(group_ids):
                raise ValueError("Heterogeneous slope FE index out of range")
            if (z.dtype != torch.float64 or not z.is_cuda or z.numel() != n
                    or not z.is_contiguous()):
                raise ValueError("slope values must be contiguous float64 CUDA tensors of length n")
            zp[int(d)] = z.data_ptr()
            icpt[int(d)] = 1 if inc else 0
        G = np.ascontiguousarray(num_groups, dtype=np.int32)
        o = _resolve_options(options or make_options(), len(group_ids), n)
        r = _lib.Result()
        rc = self.lib.b200fe_absorb_slopes_device(
            self.handle, v.data_ptr(), n, cols, len(group_ids),
            _ptr_array([g.data_ptr() for g in group_ids]), G.ctypes.data, _ptr_array(zp),
            icpt.ctypes.data, None if weights is None else weights.data_ptr(), ctypes.byref(o),
            out.data_ptr(), ctypes.byref(r), stream)
        if rc not in (_lib.OK, _lib.NOT_CONVERGED):
            raise self._err(rc)
        return out, r

    def fe_recovery_max_delta(self, residual, group_ids, num_groups, weights=None,
                              sweep_order=None) -> float:
        res = np.ascontiguousarray(residual, dtype=np.float64)
        gids = [np.ascontiguousarray(g, dtype=np.int32) for g in group_ids]
        G = np.ascontiguousarray(num_groups, dtype=np.int32)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        so = None if sweep_order is None else np.ascontiguousarray(sweep_order, dtype=np.int32)
        out = ctypes.c_double()
        rc = self.lib.b200fe_fe_recovery_max_delta(
            self.handle, res.ctypes.data, res.shape[0], len(gids),
            _ptr_array([g.ctypes.data for g in gids]), G.ctypes.data,
            None if w is None else w.ctypes.data, None if so is None else so.ctypes.data,
            ctypes.byref(out))
        if rc != _lib.OK:
            raise self._err(rc)
        return float(out.value)


def _to_result(r: _lib.Result, y_out, X_out, G) -> AbsorptionResult:
    return AbsorptionResult(
        y_tilde=y_out, X_tilde=X_out, iterations=int(r.iterations),
        converged=bool(r.converged), abs_residual=float(r.abs_residual),
        abs_residual_rel=float(r.abs_residual_rel),
        precision_certified=bool(r.precision_certified),
        fe_levels=[int(g) for g in G], gpu_used=True,
        gpu_status_code=1 if r.converged else 3, gpu_attempted=True,
        gpu_absorption_converged=bool(r.converged),
        gpu_absorption_iterations=int(r.iterations),
        outer_iterations=int(r.outer_iterations), rel_residual=float(r.rel_residual),
        primary_dim=int(r.primary_dim), setup_ms=float(r.setup_ms),
        solve_ms=float(r.solve_ms), h2d_ms=float(r.h2d_ms), d2h_ms=float(r.d2h_ms),
        kernel_launches=int(r.kernel_launches), prof_ms=list(r.prof_ms),
        prof_bytes=list(r.prof_bytes), prof_launches=list(r.prof_launches))


_tls = threading.local()


def _thread_absorber(device: int = 0) -> Absorber:
    a = getattr(_tls, "absorber", None)
    if a is None or a.device != device:
        a = Absorber(device)
        _tls.absorber = a
    return a


def absorb_many(jobs, *, workers: int = 4, device: int = 0, options=None, ols=None):
    """Independent absorptions of device-resident panels, run concurrently.

    jobs: a sequence of (v, group_ids, num_groups, weights) with v a float64
    CUDA tensor (cols, n) as absorb_device takes.  Each of ``workers`` host
    threads owns an Absorber context and a CUDA stream and takes the jobs
    i = w, w + workers, ...; the GPU overlaps their kernels, which for small
    (launch- and latency-bound) panels raises the batch's throughput.  Every
    panel is solved exactly as by one absorb_device call, so each answer is
    bitwise that of the sequential call.  ols: optional keyword arguments of
    run_ols, run per panel on its within transform (clusters given as the 5th
    element of the job).  Returns [(out, Result, OlsResult or None)] in job order.
    """
    import torch
    from concurrent.futures import ThreadPoolExecutor
    jobs = list(jobs)
    workers = max(1, min(int(workers), len(jobs) or 1))
    o = options or make_options()
    results = [None] * len(jobs)

    def run(w):
        torch.cuda.set_device(device)
        ab = _thread_absorber(device)
        st = torch.cuda.Stream(device=device)
        with torch.cuda.stream(st):
            for i in range(w, len(jobs), workers):
                job = jobs[i]
                v, g, G, wt = job[0], job[1], job[2], job[3]
                out, r = ab.absorb_device(v, g, G, wt, o, stream=st.cuda_stream)
                o_r = None
                if ols is not None:
                    cl = job[4] if len(job) > 4 else None
                    o_r = run_ols(out[0], out[1:], wt, cl, device=device, **ols)
                results[i] = (out, r, o_r)
        st.synchronize()

    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(run, w) for w in range(workers)]:
            f.result()
    return results


def _check_finite(a, name):
    if not np.all(np.isfinite(a)):
        raise ValueError(f"{name} contains non-finite values")


def absorb_fixed_effects(y, X, fes, weights=None, *, device=0, save_fe=False, slopes=None,
                         **options) -> AbsorptionResult:
    """Demean y and X on the FE dims ``fes`` (raw nonnegative ids), no singleton
    drop (absorb_fixed_effects_v6 with the GPU backend).  save_fe: also return
    the FE coefficients per dim, indexed by the dense ids (``fe``), as the
    reference's retain_fixed_effects.  slopes: heterogeneous slope terms
    (fe_index, values, include_intercept), the v6 call's ``slopes``."""
    y = np.asarray(y, dtype=np.float64)
    _check_finite(y, "y")
    if X is not None:
        _check_finite(np.asarray(X), "X")
    dense = [dense_ids(f) for f in fes]
    o = make_options(**options)
    return _thread_absorber(device).absorb(
        y, X, [d for d, _ in dense], [g for _, g in dense], weights, o, save_fe=save_fe,
        slopes=slopes)


@dataclass
class FeRecoveryResult:
    """hdfe::detail::FeRecoveryResult (include/fe_absorption.hpp:55-60)."""
    contributions: list
    iterations: int = 0
    max_delta: float = 0.0
    converged: bool = True


def recover_fixed_effects(partial, fes, weights=None, *, tol=1e-8, fe_tolerance=0.0, device=0,
                          **options) -> FeRecoveryResult:
    """The reference's recover_fixed_effects on its GPU path
    (src/fe_absorption.cpp:15453-15540): absorb ``partial`` (y - X b) with
    saved FEs, the per-dim contributions alpha_d[gid_d], then the orthogonality
    check max_delta of partial - sum_d contributions; converged when
    max_delta <= fe_tolerance (or tol).  ``fes`` are dense ids."""
    partial = np.asarray(partial, dtype=np.float64)
    _check_finite(partial, "partial")
    gids = [np.ascontiguousarray(f, dtype=np.int32) for f in fes]
    G = [int(g.max()) + 1 if g.size else 1 for g in gids]
    ab = _thread_absorber(device)
    fe_tol = fe_tolerance if fe_tolerance > 0.0 else tol
    # the check below is absolute (the largest group mean of the residual): the
    # solve runs two orders tighter than the tolerance it must meet and stops
    # only when every group mean is within half of it
    solve_tol = max(min(tol, fe_tol) * 1e-2, 1e-14)
    res = ab.absorb(partial, None, gids, G, weights,
                    make_options(tol=solve_tol, fe_linf_tol=0.5 * fe_tol, **options),
                    save_fe=True)
    contrib = [res.fe[d][gids[d], 0] for d in range(len(gids))]
    out = FeRecoveryResult(contributions=contrib, iterations=res.iterations)
    if res.converged and fe_tol > 0.0:
        resid = partial - np.sum(contrib, axis=0)
        out.max_delta = ab.fe_recovery_max_delta(resid, gids, G, weights)
        out.converged = out.max_delta <= fe_tol
    else:
        out.converged = bool(res.converged)
    return out


def drop_singletons_mask(fes) -> np.ndarray:
    """Rows kept after iteratively dropping singleton groups in any FE dim
    (the reference's pre-absorption rule, src/hdfe_regressor_v11.cpp:4056)."""
    n = len(fes[0])
    keep = np.ones(n, dtype=bool)
    dense = [dense_ids(f)[0] for f in fes]
    while True:
        changed = False
        for fe in dense:
            idx = fe[keep]
            cnt = np.bincount(idx)
            single = cnt[idx] == 1
            if single.any():
                kidx = np.flatnonzero(keep)
                keep[kidx[single]] = False
                changed = True
        if not changed:
            return keep


def dense_ids_device(raw, device=0):
    """build_indexer on the device (src/fe_absorption.cpp:845-940): raw int32
    ids (numpy or torch) -> (int32 CUDA tensor of dense ids, num_groups,
    num_levels_present)."""
    import torch
    ab = _thread_absorber(device)
    r = torch.as_tensor(np.asarray(raw, dtype=np.int32) if not isinstance(raw, torch.Tensor) else raw,
                        dtype=torch.int32).to(f"cuda:{device}").contiguous()
    out = torch.empty_like(r)
    G, present = ctypes.c_int32(), ctypes.c_int32()
    rc = ab.lib.b200fe_dense_ids_device(ab.handle, r.data_ptr(), r.numel(), out.data_ptr(),
                                        ctypes.byref(G), ctypes.byref(present))
    if rc != _lib.OK:
        raise ab._err(rc)
    return out, int(G.value), int(present.value)


def drop_singletons_device(ids, num_groups, device=0, max_iter=100):
    """Singleton cascade on the device (compute_keep_mask_drop_singletons,
    src/hdfe_regressor_v11.cpp:4056-4290): dense int32 CUDA tensors ->
    (bool CUDA tensor keep, dropped, rounds)."""
    import torch
    ab = _thread_absorber(device)
    n = ids[0].numel()
    keep = torch.empty(n, dtype=torch.uint8, device=ids[0].device)
    G = np.ascontiguousarray(num_groups, dtype=np.int32)
    dropped, rounds = ctypes.c_int64(), ctypes.c_int()
    rc = ab.lib.b200fe_drop_singletons_device(
        ab.handle, len(ids), _ptr_array([g.data_ptr() for g in ids]), G.ctypes.data, n,
        keep.data_ptr(), max_iter, ctypes.byref(dropped), ctypes.byref(rounds))
    if rc != _lib.OK:
        raise ab._err(rc)
    return keep.bool(), int(dropped.value), int(rounds.value)


@dataclass
class FeComponentStats:
    """hdfe::v11::FeComponentStats (include/hdfe/hdfe_regressor_v11.hpp:68-73)."""
    num_components: int
    largest_component_n_obs: int
    largest_component_obs_share: float
    largest_component_weight_share: float


def first_pair_component_stats(first_fe, second_fe, weights=None, device=0) -> FeComponentStats:
    """compute_first_pair_component_stats on the device: the mobility groups
    (connected components) of the first two FE dims, raw int32 ids."""
    import torch
    ab = _thread_absorber(device)
    dev = f"cuda:{device}"

    def on_device(a):  # torch CUDA tensors are used in place
        if isinstance(a, torch.Tensor):
            return a.to(device=dev, dtype=torch.int32).contiguous()
        return torch.as_tensor(np.asarray(a, dtype=np.int32)).to(dev).contiguous()

    f1 = on_device(first_fe)
    f2 = on_device(second_fe)
    if f1.numel() != f2.numel():
        raise ValueError("First-pair FE vectors must have the same length")
    w = None if weights is None else torch.as_tensor(
        np.asarray(weights, dtype=np.float64)).to(dev).contiguous()
    nc, big = ctypes.c_int(), ctypes.c_int64()
    share, wshare = ctypes.c_double(), ctypes.c_double()
    rc = ab.lib.b200fe_first_pair_components_device(
        ab.handle, f1.data_ptr(), f2.data_ptr(), f1.numel(), None if w is None else w.data_ptr(),
        ctypes.byref(nc), ctypes.byref(big), ctypes.byref(share), ctypes.byref(wshare))
    if rc != _lib.OK:
        raise ab._err(rc)
    return FeComponentStats(int(nc.value), int(big.value), float(share.value), float(wshare.value))


def partial_out(y, X, fes, weights=None, *, drop_singletons=True, device=0,
                **options) -> AbsorptionResult:
    """HdfeRegressorV11::partial_out: singleton drop, then absorption.  The
    result's ``sample_index`` holds the kept 0-based rows."""
    y = np.asarray(y, dtype=np.float64)
    if y.size == 0:
        raise ValueError("Outcome vector must be non-empty")
    X = np.zeros((y.size, 0)) if X is None else np.asarray(X, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    if X.shape[0] != y.size:
        raise ValueError("X must have the same number of rows as y")
    _check_finite(y, "y")
    _check_finite(X, "X")
    if weights is not None:
        w = np.asarray(weights, dtype=np.float64)
        if w.shape[0] != y.size or not np.all(np.isfinite(w)) or np.any(w < 0):
            raise ValueError("weights must be finite and non-negative")
    import torch
    # the columns go to the device once; preprocessing (dense ids as in
    # build_indexer, the singleton cascade), the row compaction, the
    # absorption and the within transform stay there; one copy back
    dev = torch.device("cuda", device)
    ab = _thread_absorber(device)
    dense = [dense_ids_device(f, device) for f in fes]
    G = [g for _, g, _ in dense]
    n = y.size
    idx_d = None
    if drop_singletons and fes:
        keep = drop_singletons_device([d for d, _, _ in dense], G, device)[0]
        idx_d = torch.nonzero(keep).squeeze(1)
    o = make_options(**options)
    if idx_d is not None and idx_d.numel() == 0:
        raise ValueError("no observations left after dropping singletons")
    cols = 1 + X.shape[1]
    v = torch.empty((cols, n), dtype=torch.float64, device=dev)
    v[0].copy_(torch.from_numpy(np.ascontiguousarray(y)))
    if cols > 1:
        v[1:].copy_(torch.from_numpy(np.ascontiguousarray(X.T)))
    w_d = None if weights is None else torch.from_numpy(
        np.ascontiguousarray(weights, dtype=np.float64)).to(dev)
    ids = [d for d, _, _ in dense]
    if idx_d is not None and idx_d.numel() < n:
        v = v.index_select(1, idx_d)
        ids = [d.index_select(0, idx_d) for d in ids]
        w_d = None if w_d is None else w_d.index_select(0, idx_d)
        idx = idx_d.to(torch.int32).cpu().numpy()
    else:
        idx = np.arange(n, dtype=np.int32)
    stream = torch.cuda.current_stream(dev).cuda_stream
    out, r = ab.absorb_device(v, ids, G, w_d, o, stream=stream)
    host = out.cpu().numpy()
    res = _to_result(r, host[0], host[1:].T, G)
    res.sample_index = idx
    return res


SE_TYPES = {"unadjusted": 0, "homoskedastic": 0, "robust": 1, "cluster": 2}


@dataclass
class OlsResult:
    """Fields of hdfe::detail::OlsResult (include/ols.hpp:13-34) this library
    computes (residuals stay on the device)."""
    coefficients: np.ndarray
    std_errors: np.ndarray
    covariance: np.ndarray
    xtx_inv: np.ndarray
    rss: float
    sigma2: float
    df_resid: float
    cov_scale: float
    cluster_u2: float
    num_clusters: int
    nobs: int


def run_ols(y, X, weights=None, clusters=None, *, se_type="unadjusted", n_effective=-1.0,
            weights_are_frequencies=False, device=0) -> OlsResult:
    """hdfe::detail::run_ols (include/ols.hpp:40-51) on within-transformed host
    arrays: moments on the device, the p x p algebra on the host.  ``clusters``:
    ids (made dense here); torch CUDA tensors are taken as device arrays."""
    se = SE_TYPES[se_type]
    ab = _thread_absorber(device)
    r = _lib.OlsResult()
    try:
        import torch
        on_device = isinstance(y, torch.Tensor)
    except ImportError:
        on_device = False
    if on_device:
        n, p = int(X.shape[1]), int(X.shape[0])  # X: (p, n) contiguous = column-major n x p
        cl = None if clusters is None else clusters
        G = 0 if clusters is None else int(clusters.max().item()) + 1
        rc = ab.lib.b200fe_ols_device(
            ab.handle, y.data_ptr(), X.data_ptr(), n, p,
            None if weights is None else weights.data_ptr(),
            None if cl is None else cl.data_ptr(), G, se, float(n_effective),
            int(weights_are_frequencies), ctypes.byref(r))
    else:
        y = np.ascontiguousarray(y, dtype=np.float64)
        X = np.asfortranarray(X, dtype=np.float64)
        if X.ndim == 1:
            X = X[:, None]
        n, p = X.shape
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        cl, G = (None, 0) if clusters is None else dense_ids(clusters)
        rc = ab.lib.b200fe_ols(
            ab.handle, y.ctypes.data, X.ctypes.data, n, p, None if w is None else w.ctypes.data,
            None if cl is None else cl.ctypes.data, G, se, float(n_effective),
            int(weights_are_frequencies), ctypes.byref(r))
    if rc != _lib.OK:
        raise ab._err(rc)
    cov = np.ctypeslib.as_array(r.cov)[: p * p].reshape(p, p, order="F").copy()
    inv = np.ctypeslib.as_array(r.xtx_inv)[: p * p].reshape(p, p, order="F").copy()
    return OlsResult(coefficients=np.array(r.coef[:p]), std_errors=np.array(r.se[:p]),
                     covariance=cov, xtx_inv=inv, rss=r.rss, sigma2=r.sigma2,
                     df_resid=r.df_resid, cov_scale=r.cov_scale, cluster_u2=r.cluster_u2,
                     num_clusters=int(r.num_clusters), nobs=n)


def demean_raw(Y, X, fes, nlev, tol=1e-8, max_iter=0) -> int:
    """In-place demean (schwarz_demean_raw's interface).  Returns iterations."""
    lib = _lib.load()
    Y = np.asarray(Y)
    if Y.dtype != np.float64 or not Y.flags.c_contiguous:
        raise ValueError("Y must be a contiguous float64 array (modified in place)")
    k = 0 if X is None else X.shape[1]
    if k and (X.dtype != np.float64 or not X.flags.f_contiguous):
        raise ValueError("X must be a Fortran-ordered float64 array (modified in place)")
    gids = [np.ascontiguousarray(f, dtype=np.int32) for f in fes]
    G = np.ascontiguousarray(nlev, dtype=np.int32)
    it = ctypes.c_int()
    rc = lib.b200fe_demean_raw(Y.ctypes.data, X.ctypes.data if k else None, Y.shape[0], k,
                               len(gids), _ptr_array([g.ctypes.data for g in gids]),
                               G.ctypes.data, float(tol), int(max_iter), ctypes.byref(it))
    if rc not in (_lib.OK, _lib.NOT_CONVERGED):
        raise AbsorberError(rc, "demean_raw failed")
    return int(it.value)

"""Parity at the benchmark configurations' own sizes, against the reference's CPU core.

Config 1 (the reference's CPU-runnable case): N = 1,000,000 observations, seed 0,
workers observed 1 + Poisson(9) years capped at a 10-year panel (workers are drawn
until the panel holds exactly 1,000,000 rows, about 107k workers), 10,000 firms with
Zipf(1.1) sizes, move probability 0.1, y = 0.5 x1 - 0.3 x2 + worker + firm + year FE
+ noise; singletons dropped; worker-clustered SEs.  Absorbed on {worker, firm} and on
{worker, firm, year}:

* the reference's own HdfeRegressorV11::fit (src/hdfe_regressor_v11.cpp:7522)
  dispatching its absorptions to this library through the reference-side binding,
  against the same fit on the reference's CPU core in strict-residual mode;
* this library's partial_out + run_ols (cluster) against the reference's
  partial_out (src/hdfe_regressor_v11.cpp:10275, CPU, strict-residual) + run_ols
  at the same n_effective.

Coefficients and SEs agree to 1e-8 relative in both.

Config 2's panel shape (the 50M generator's ratios: workers, firms and 36 years,
the outcome plus 12 regressors, three FE dims): this library's default
mixed-precision absorption at tol 1e-8 agrees to 1e-8 of each column's norm with
the reference CPU core's strict-residual projection (tol 1e-11) at 1M rows, and
with the reference's own CUDA absorber in strict-residual mode at 5M rows (the
reference's CPU core needs 606 alternating-projection iterations, over two minutes
on eight cores, for tol 1e-8 at 5M, and its iteration count grows with N).
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8   # coefficients, SEs, within transform (column norm)
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def config1(panels):
    return panels.akm_two_way(1_000_000, n_firms=10_000, n_years=10, seed=0, three_way=True)


def _fes(p, three_way):
    return p.fes if three_way else p.fes[:2]


@pytest.mark.parametrize("three_way", [False, True])
def test_config1_reference_fit_on_b200(oracle_mod, config1, three_way):
    if not oracle_mod.REF_B200_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_b200.so not built (needs the reference sources)")
    p, so = config1, oracle_mod.REF_B200_SO
    fes = _fes(p, three_way)
    fg = oracle_mod.ref_fit(p.y, p.X, fes, cluster=p.cluster, tol=1e-10, threads=THREADS,
                            gpu_backend="cuda", lib_path=so)
    fc = oracle_mod.ref_fit(p.y, p.X, fes, cluster=p.cluster, tol=1e-14,
                            tolerance_mode="strict-residual", threads=THREADS,
                            gpu_backend="cpu", lib_path=so)
    assert fg["gpu_status_code"] == 1 and fg["converged"]
    assert fg["nobs"] == fc["nobs"] and fg["df_a"] == fc["df_a"]
    assert np.allclose(fg["coef"], fc["coef"], rtol=REL_TOL, atol=0.0), (fg["coef"], fc["coef"])
    assert np.allclose(fg["se"], fc["se"], rtol=REL_TOL, atol=0.0), (fg["se"], fc["se"])


@pytest.mark.parametrize("three_way", [False, True])
def test_config1_partial_out_and_cluster_ols(pkg, oracle_mod, config1, three_way):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    p = config1
    fes = _fes(p, three_way)
    ours = pkg.partial_out(p.y, p.X, fes, None, tol=1e-10)
    ref = oracle_mod.ref_partial_out(p.y, p.X, fes, None, tol=1e-14,
                                     tolerance_mode="strict-residual", threads=THREADS,
                                     gpu_backend="cpu")
    assert ours.converged and ours.precision_certified
    assert np.array_equal(ours.sample_index, ref["sample_index"])
    keep = ours.sample_index
    V = np.column_stack([ours.y_tilde, ours.X_tilde])
    Vo = np.column_stack([p.y, p.X])[keep]
    err = np.linalg.norm(V - ref["V"], axis=0) / np.linalg.norm(Vo, axis=0)
    assert err.max() <= REL_TOL, err
    cl = p.cluster[keep]
    # worker FEs nest in the worker clusters: only the other dims' levels are absorbed dof
    n_eff = keep.size - sum(int(np.unique(f[keep]).size) for f in fes[1:])
    o = pkg.run_ols(ours.y_tilde, ours.X_tilde, None, cl, se_type="cluster",
                    n_effective=float(n_eff))
    r = oracle_mod.ref_run_ols(ref["V"][:, 0], ref["V"][:, 1:], None, cl, se_type="cluster",
                               n_effective=float(n_eff))
    assert np.allclose(o.coefficients, r["coef"], rtol=REL_TOL, atol=0.0)
    assert np.allclose(o.std_errors, r["se"], rtol=REL_TOL, atol=0.0)
    assert o.num_clusters == r["num_clusters"]


def _config2_shape(panels, n):
    p = panels.akm_batched(n, n_firms=max(1000, int(800_000 * n / 50_000_000)), n_years=36, seed=0)
    return panels.subset(p, panels.drop_singletons(p.fes))


def _rel_err(res, V_ref, p):
    V = np.column_stack([res.y_tilde, res.X_tilde])
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    return np.linalg.norm(V - V_ref, axis=0) / scale


def test_config2_shape_1m_against_reference_cpu_tight_projection(pkg, oracle_mod, panels):
    """The config-2 panel shape at 1M rows (about 100k workers, 16k firms, 36
    years, 13 columns): the default mixed
    absorption at tol 1e-8 against the reference CPU core's strict-residual
    projection at tol 1e-11."""
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    p = _config2_shape(panels, 1_000_000)
    res = pkg.absorb_fixed_effects(p.y, p.X, p.fes, tol=1e-8, precision="mixed")
    assert res.converged and res.precision_certified
    ref = oracle_mod.ref_absorb(p.y, p.X, p.fes, None, tol=1e-11, tolerance_mode="strict-residual",
                                threads=THREADS)
    assert ref["converged"]
    err = _rel_err(res, ref["V"], p)
    assert err.max() <= REL_TOL, err


def test_config2_shape_5m_against_reference_cuda_backend(pkg, oracle_mod, panels):
    """The config-2 panel shape at 5M rows against the reference's own CUDA
    absorber (its alternating projections, built for sm_100a from its sources)
    run in strict-residual mode at tol 1e-11: an independent solve of the same
    projection at a size the reference's CPU core does not finish in minutes."""
    if not oracle_mod.REF_CUDA_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_cuda.so not built")
    p = _config2_shape(panels, 5_000_000)
    res = pkg.absorb_fixed_effects(p.y, p.X, p.fes, tol=1e-8, precision="mixed")
    assert res.converged and res.precision_certified
    ref = oracle_mod.ref_absorb(p.y, p.X, p.fes, None, tol=1e-11, tolerance_mode="strict-residual",
                                threads=THREADS, gpu_backend="cuda", lib_path=oracle_mod.REF_CUDA_SO)
    assert ref["converged"] and ref["gpu_status_code"] == 1  # solved on the reference's GPU path
    err = _rel_err(res, ref["V"], p)
    assert err.max() <= REL_TOL, err

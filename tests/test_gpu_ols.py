"""OLS on within-transformed data on the device (b200fe_ols / b200fe_ols_device)
against the reference's own hdfe::detail::run_ols (include/ols.hpp:40-51,
src/ols.cpp:1237-1520) on the same inputs: coefficients, standard errors,
covariance, RSS, df_resid, cov_scale, cluster_u2 and the cluster count, for
homoskedastic, robust and one-way cluster inference, unweighted, with
analytic weights and with frequency weights; clusters by worker (many small)
and by firm (Zipf sizes: a cluster spans many chunks).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # FP64 moments in a different (fixed) summation order


@pytest.fixture(scope="module")
def within(pkg, panels):
    p = panels.akm_two_way(40_000, n_firms=300, seed=81, three_way=True)
    p = panels.subset(p, panels.drop_singletons(p.fes))
    r = pkg.absorb_fixed_effects(p.y, p.X, p.fes, tol=1e-10)
    return p, r.y_tilde, np.asfortranarray(r.X_tilde)


def _close(a, b, tol=REL_TOL):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b)))


@pytest.mark.parametrize("se_type", ["unadjusted", "robust", "cluster"])
@pytest.mark.parametrize("wmode", ["none", "analytic", "frequency"])
@pytest.mark.parametrize("cl_dim", [0, 1])
def test_run_ols_matches_reference(pkg, oracle_mod, within, se_type, wmode, cl_dim):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    if se_type != "cluster" and cl_dim == 1:
        pytest.skip("the cluster variable only matters for cluster inference")
    p, yt, Xt = within
    rng = np.random.default_rng(5)
    w = None
    if wmode == "analytic":
        w = rng.lognormal(0.0, 0.5, size=p.n)
    elif wmode == "frequency":
        w = rng.integers(1, 5, size=p.n).astype(np.float64)
    freq = wmode == "frequency"
    cl = np.asarray(p.fes[cl_dim]) if se_type == "cluster" else None
    n_eff = p.n - 1234.0
    ours = pkg.run_ols(yt, Xt, w, cl, se_type=se_type, n_effective=n_eff,
                       weights_are_frequencies=freq)
    ref = oracle_mod.ref_run_ols(yt, Xt, w, cl, se_type=se_type, n_effective=n_eff,
                                 weights_are_frequencies=freq)
    assert _close(ours.coefficients, ref["coef"])
    assert _close(ours.std_errors, ref["se"])
    assert _close(ours.covariance, ref["cov"])
    assert _close(ours.rss, ref["rss"])
    assert ours.df_resid == ref["df_resid"]
    assert _close(ours.cov_scale, ref["cov_scale"], 1e-14)
    if se_type == "cluster":
        assert ours.num_clusters == ref["num_clusters"]
        assert _close(ours.cluster_u2, ref["cluster_u2"], 1e-9)


def test_device_arrays_match_host(pkg, within):
    import torch
    p, yt, Xt = within
    cl = np.asarray(p.fes[1]).astype(np.int32)
    host = pkg.run_ols(yt, Xt, None, cl, se_type="cluster")
    dy = torch.from_numpy(np.ascontiguousarray(yt)).cuda()
    dX = torch.from_numpy(np.ascontiguousarray(Xt.T)).cuda()  # (p, n): column-major n x p
    dc = torch.from_numpy(cl).cuda()
    dev = pkg.run_ols(dy, dX, None, dc, se_type="cluster")
    assert np.array_equal(host.coefficients, dev.coefficients)
    assert np.array_equal(host.std_errors, dev.std_errors)


def test_rank_deficient_design_like_reference(pkg, oracle_mod, within):
    # the reference's pivoted LDLT zeroes a coefficient in the null direction
    # (a zero column) instead of failing
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    p, yt, Xt = within
    X2 = np.asfortranarray(np.column_stack([Xt[:, 0], np.zeros(p.n), Xt[:, 1]]))
    ours = pkg.run_ols(yt, X2, se_type="robust")
    ref = oracle_mod.ref_run_ols(yt, X2, se_type="robust")
    assert ours.coefficients[1] == 0.0 and ours.std_errors[1] == 0.0
    assert _close(ours.coefficients, ref["coef"])
    assert _close(ours.std_errors, ref["se"])


def test_device_cluster_ids_with_gaps(pkg, within):
    """Cluster ids on the device need not be dense: ids with unused values in
    between (empty clusters) give the same inference as the dense ids."""
    import torch
    p, yt, Xt = within
    cl = np.asarray(p.fes[0]).astype(np.int32)  # workers: many clusters of a few rows
    dense = pkg.run_ols(yt, Xt, None, cl, se_type="cluster")
    dy = torch.from_numpy(np.ascontiguousarray(yt)).cuda()
    dX = torch.from_numpy(np.ascontiguousarray(Xt.T)).cuda()
    gaps = pkg.run_ols(dy, dX, None, torch.from_numpy(3 * cl + 1).cuda(), se_type="cluster")
    assert gaps.num_clusters == dense.num_clusters
    assert _close(gaps.coefficients, dense.coefficients)
    assert _close(gaps.std_errors, dense.std_errors)

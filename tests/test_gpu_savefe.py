"""Saved fixed effects (b200fe_absorb_fe): the FE coefficients behind the
within transform, the reference's retain_fixed_effects outputs
(fe_alpha_y / fe_alpha_X, src/fe_absorption_cuda.cu:4663-4690) that its
recover_fixed_effects consumes (src/fe_absorption.cpp:15484-15540).

Checked: the reconstruction identity v - v~ = sum_d fe_d[gid_d] (to rounding),
the total FE fit against the oracle's near-exact projection (REL_TOL), groups
without observations at zero, the package's recover_fixed_effects against the
reference CPU core's, and the reference's own recover_fixed_effects running on
this library through the reference-side binding.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8    # total FE fit vs the near-exact projection (tol 1e-10 solves)
IDENT_TOL = 1e-11  # v - v~ vs sum of the saved coefficients


def _panel(panels, n, three_way, seed, firms=500):
    p = panels.akm_two_way(n, n_firms=firms, seed=seed, three_way=three_way)
    return panels.subset(p, panels.drop_singletons(p.fes))


def _fe_sum(fe, fes):
    return sum(fe[d][np.asarray(fes[d])] for d in range(len(fes)))


@pytest.mark.parametrize("case", ["three_way", "two_way", "weighted", "one_way", "four_dims"])
def test_saved_fe_reconstruct_and_match_projection(absorber, pkg, oracle_mod, panels, case):
    rng = np.random.default_rng(3)
    p = _panel(panels, 30_000, case != "two_way", seed=71)
    fes, G = list(p.fes), list(p.levels)
    w = None
    if case == "weighted":
        w = rng.lognormal(0.0, 0.5, size=p.n)
    elif case == "one_way":
        fes, G = fes[:1], G[:1]
    elif case == "four_dims":
        fx = ((np.asarray(fes[1]) * 7 + np.asarray(fes[2])) % 997).astype(np.int32)
        fx, gx = pkg.dense_ids(fx)
        fes, G = fes + [fx], G + [gx]
    V = np.column_stack([p.y, p.X])
    r = absorber.absorb(p.y, p.X, fes, G, w, pkg.make_options(tol=1e-10), save_fe=True)
    assert r.converged and r.fe is not None
    assert [a.shape for a in r.fe] == [(g, V.shape[1]) for g in G]
    out = np.column_stack([r.y_tilde, r.X_tilde])
    scale = np.linalg.norm(V, axis=0)
    fit = _fe_sum(r.fe, fes)
    ident = np.linalg.norm((V - out) - fit, axis=0) / scale
    assert ident.max() <= IDENT_TOL, ident
    ref, _, ok = oracle_mod.project(p.y, p.X, fes, G, w, tol=1e-13)
    assert ok
    err = np.linalg.norm((V - ref) - fit, axis=0) / scale
    assert err.max() <= REL_TOL, err
    assert np.array_equal(r.fe_alpha_y[0], r.fe[0][:, 0])


def test_saved_fe_empty_groups_are_zero(absorber, pkg, panels):
    p = _panel(panels, 10_000, True, seed=73, firms=200)
    G = list(p.levels)
    G[1] += 5  # five firms without observations
    r = absorber.absorb(p.y, p.X, p.fes, G, None, pkg.make_options(tol=1e-10), save_fe=True)
    assert not r.fe[1][-5:].any()


def test_recover_fixed_effects_matches_reference_cpu(pkg, oracle_mod, panels):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    p = _panel(panels, 20_000, True, seed=75, firms=400)
    beta = np.array([0.5, -0.3])
    partial = p.y - p.X @ beta
    ours = pkg.recover_fixed_effects(partial, p.fes, tol=1e-10)
    ref = oracle_mod.ref_recover_fe(partial, p.fes, tol=1e-10)
    assert ours.converged and ref["converged"]
    assert ours.max_delta <= 1e-10
    tot = np.sum(ours.contributions, axis=0)
    tot_ref = ref["contributions"].sum(axis=0)
    assert np.linalg.norm(tot - tot_ref) <= REL_TOL * np.linalg.norm(partial)


def test_reference_recovery_runs_on_b200(oracle_mod, panels):
    if not oracle_mod.REF_B200_SO.exists() or not oracle_mod.ref_available():
        pytest.skip("reference libraries not built (need the reference sources)")
    p = _panel(panels, 20_000, True, seed=77, firms=400)
    partial = p.y - 0.4 * p.X[:, 0]
    gpu = oracle_mod.ref_recover_fe(partial, p.fes, tol=1e-10, gpu_backend="cuda",
                                    lib_path=oracle_mod.REF_B200_SO)
    cpu = oracle_mod.ref_recover_fe(partial, p.fes, tol=1e-10)
    assert gpu["converged"] and gpu["max_delta"] <= 1e-10
    tot = gpu["contributions"].sum(axis=0)
    assert np.linalg.norm(tot - cpu["contributions"].sum(axis=0)) <= REL_TOL * np.linalg.norm(partial)


def test_group_mean_stop_on_a_large_panel(absorber, pkg, panels):
    """fe_linf_tol: on a 2M-row panel the relative L2 stop leaves firm means of
    the within transform near 1e-7 for the smallest firms; with the option every
    group mean is within it, and recover_fixed_effects meets an absolute
    fe_tolerance of 1e-8."""
    p = panels.akm_batched(2_000_000, n_firms=32_000, n_years=36, seed=0)
    p = panels.subset(p, panels.drop_singletons(p.fes))
    rng = np.random.default_rng(3)
    partial = p.y - p.X @ (0.01 * rng.standard_normal(p.k))
    G = np.asarray(p.levels, dtype=np.int32)
    def max_means(r):
        out = []
        for d in range(len(p.fes)):
            cnt = np.bincount(p.fes[d], minlength=G[d])
            m = np.bincount(p.fes[d], weights=r.y_tilde, minlength=G[d])[cnt > 0] / cnt[cnt > 0]
            out.append(np.abs(m).max())
        return max(out)

    plain = absorber.absorb(partial, None, p.fes, G, None, pkg.make_options(tol=1e-10))
    assert plain.converged and max_means(plain) > 1e-8  # the L2 stop alone
    r = absorber.absorb(partial, None, p.fes, G, None,
                        pkg.make_options(tol=1e-10, fe_linf_tol=1e-9))
    assert r.converged and max_means(r) <= 1e-9 * (1 + 1e-6)
    # a bound below the rounding floor: the round that cannot reach it is undone
    tight = absorber.absorb(partial, None, p.fes, G, None,
                            pkg.make_options(tol=1e-10, fe_linf_tol=1e-15))
    assert tight.converged and max_means(tight) <= max_means(plain)
    rec = pkg.recover_fixed_effects(partial, p.fes, tol=1e-8, fe_tolerance=1e-8)
    assert rec.converged and rec.max_delta <= 1e-8

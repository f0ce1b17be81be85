"""Drop-in check: the reference's own core, built with -DHDFE_USE_CUDA over the
reference-side binding (xhdfe-xfe_b200/shim/fe_absorption_b200.cpp), runs its
absorptions on the B200 library.

oracle/_ref/libxhdfe_ref_b200.so is the reference's unmodified CPU sources
compiled with CUDA on, its host certificate, the shim and the test driver
(oracle/Makefile target ref_b200).  Through it the reference's own
absorb_fixed_effects_v6, HdfeRegressorV11::partial_out and ::fit dispatch to
libb200fe.so exactly as they would to the reference's CUDA absorber, certify
the result with the reference's host certificate, and report GPU status 1.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


@pytest.fixture(scope="module")
def ref_b200(oracle_mod):
    if not oracle_mod.REF_B200_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_b200.so not built (needs the reference sources)")
    return oracle_mod.REF_B200_SO


def _panel(panels, seed=61):
    p = panels.akm_two_way(30_000, n_firms=600, seed=seed, three_way=True)
    return panels.subset(p, panels.drop_singletons(p.fes))


def test_reference_absorber_dispatches_to_b200(oracle_mod, panels, ref_b200):
    p = _panel(panels)
    r = oracle_mod.ref_absorb(p.y, p.X, p.fes, None, tol=1e-10, gpu_backend="cuda",
                              lib_path=ref_b200)
    assert r["gpu_status_code"] == 1  # used, converged
    assert r["converged"] and r["precision_certified"]
    ref, _, ok = oracle_mod.project(p.y, p.X, p.fes, p.levels, tol=1e-13)
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    assert (np.linalg.norm(r["V"] - ref, axis=0) / scale).max() <= REL_TOL


def test_reference_partial_out_and_fit_on_b200(oracle_mod, panels, ref_b200):
    p = _panel(panels, seed=67)
    gpu = oracle_mod.ref_partial_out(p.y, p.X, p.fes, tol=1e-10, gpu_backend="cuda",
                                     lib_path=ref_b200)
    cpu = oracle_mod.ref_partial_out(p.y, p.X, p.fes, tol=1e-14,
                                     tolerance_mode="strict-residual", gpu_backend="cpu",
                                     lib_path=ref_b200)
    assert gpu["gpu_status_code"] == 1
    assert np.array_equal(gpu["sample_index"], cpu["sample_index"])
    scale = np.linalg.norm(cpu["V"], axis=0) + 1e-300
    Vo = np.column_stack([p.y, p.X])[cpu["sample_index"]]
    err = (np.linalg.norm(gpu["V"] - cpu["V"], axis=0) / np.linalg.norm(Vo, axis=0)).max()
    assert err <= REL_TOL
    fg = oracle_mod.ref_fit(p.y, p.X, p.fes, cluster=p.cluster, tol=1e-10, gpu_backend="cuda",
                            lib_path=ref_b200)
    fc = oracle_mod.ref_fit(p.y, p.X, p.fes, cluster=p.cluster, tol=1e-14,
                            tolerance_mode="strict-residual", gpu_backend="cpu",
                            lib_path=ref_b200)
    assert fg["gpu_status_code"] == 1 and fg["nobs"] == fc["nobs"]
    assert np.allclose(fg["coef"], fc["coef"], rtol=REL_TOL, atol=1e-12)
    assert np.allclose(fg["se"], fc["se"], rtol=REL_TOL, atol=1e-12)


def test_demean_raw_matches_oracle(pkg, oracle_mod, panels):
    """b200fe_demean_raw (the C entry behind xhdfe::schwarz_demean_raw) against
    the oracle's tight projection, unweighted, two and three FE dims."""
    p = _panel(panels, seed=71)
    ref, _, ok = oracle_mod.project(p.y, p.X, p.fes, p.levels, tol=1e-13)
    assert ok
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    for k in (2, 3):
        fes = p.fes[:k]
        ref_k = ref if k == 3 else oracle_mod.project(p.y, p.X, fes, p.levels[:k], tol=1e-13)[0]
        Y = np.array(p.y, dtype=np.float64, copy=True)
        X = np.asfortranarray(np.array(p.X, dtype=np.float64, copy=True))
        its = pkg.demean_raw(Y, X, fes, p.levels[:k], tol=1e-10)
        V = np.column_stack([Y, X])
        assert (np.linalg.norm(V - ref_k, axis=0) / scale).max() <= REL_TOL
        assert its > 0


def test_schwarz_demean_raw_binding_on_b200(oracle_mod, panels, ref_b200):
    """The reference's xhdfe::schwarz_demean_raw with the reference signature,
    defined by the binding over this library (libxhdfe_ref_b200.so, where
    src/schwarz_demean.cpp is left out), against the oracle and against the
    reference's own CPU block-PCG (libxhdfe_ref.so) on the same call."""
    p = _panel(panels, seed=73)
    ok_g, Vg, its_g = oracle_mod.ref_schwarz_demean_raw(p.y, p.X, p.fes, p.levels, tol=1e-10,
                                                        lib_path=ref_b200)
    ok_c, Vc, _ = oracle_mod.ref_schwarz_demean_raw(p.y, p.X, p.fes, p.levels, tol=1e-10, threads=4)
    ref, _, ok = oracle_mod.project(p.y, p.X, p.fes, p.levels, tol=1e-13)
    assert ok_g and ok_c and ok and its_g > 0
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    assert (np.linalg.norm(Vg - ref, axis=0) / scale).max() <= REL_TOL
    assert (np.linalg.norm(Vg - Vc, axis=0) / scale).max() <= REL_TOL
    # unsupported calls return false and leave the inputs as they were, as the
    # reference's: one FE dim, and more than 16 columns
    ok1, V1, _ = oracle_mod.ref_schwarz_demean_raw(p.y, p.X, p.fes[:1], p.levels[:1], lib_path=ref_b200)
    assert not ok1 and np.array_equal(V1, np.column_stack([p.y, p.X]))
    X16 = np.repeat(p.X, 8, axis=1)  # 1 + 16 columns
    ok2, V2, _ = oracle_mod.ref_schwarz_demean_raw(p.y, X16, p.fes, p.levels, lib_path=ref_b200)
    assert not ok2 and np.array_equal(V2, np.column_stack([p.y, X16]))

"""GPU parity of the AKM/KSS firm-system solver (b200fe_kss_*, the replacement
of the reference's akm_cuda_* backend).

* batched solves against the numpy restatement of the reference's grounded
  Jacobi-PCG (oracle/kss_oracle.py): same per-lane iteration counts at the
  reference's default tol 1e-10 (within one step: the two sum the dots in
  different orders) and, at tol 1e-12, solutions within REL_TOL of a dense
  direct solve; lane pitches 1..64, firms larger than one chunk, a zero
  right-hand side and lanes that run out of iterations;
* bitwise reproducibility of two identical calls;
* the stable key sort;
* drop-in: the reference's own akm_kss_decompose, built over the reference
  side binding, routes its PCG solves to this solver (gpu_used) and gives the
  reference CPU core's variance components (tests/golden/kss_*.npz).
"""

from pathlib import Path

import numpy as np
import pytest

from test_kss import dims, match_set

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8       # solutions at tol 1e-12 vs the dense direct solve
COMP_TOL = 1e-8      # variance components, GPU path vs the reference CPU core
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def system():
    from oracle import kss_oracle as ko
    rows = match_set(3000, 300, seed=5, zipf=1.4)
    N, J = dims(rows)
    st = ko.kss_structure(rows[:, 0], rows[:, 1], rows[:, 2], N, J)
    return rows, st


@pytest.mark.parametrize("nb", [1, 3, 32, 64])
def test_batched_solve_matches_oracle(pkg, system, nb):
    """Iteration counts at the reference's default tol 1e-10 (where they do not
    depend on the order of the dot sums; at 1e-12 the residual sits on the
    FP64 rounding floor and the step that crosses it moves with that order),
    accuracy at 1e-12 against the dense direct solve."""
    from oracle import kss_oracle as ko
    rows, st = system
    J = st["J"]
    assert np.diff(st["f_ptr"]).max() > 64  # a firm spans several chunks
    sysd = pkg.kss_system(rows[:, 0], rows[:, 1], rows[:, 2], st["N"], J)
    B = np.random.default_rng(nb).standard_normal((nb, J))
    solver = pkg.KssSolver(sysd)
    try:
        Z10, its10 = solver.solve_multi(B, tol=1e-10, max_iter=20_000)
        Z, its = solver.solve_multi(B, tol=1e-12, max_iter=20_000)
        Z2, its2 = solver.solve_multi(B, tol=1e-12, max_iter=20_000)
    finally:
        solver.close()
    assert np.array_equal(Z, Z2) and np.array_equal(its, its2)  # bitwise reproducible
    for l in range(nb):
        zo, ito = ko.kss_pcg(st, B[l], tol=1e-10, max_iter=20_000)
        assert ito > 0 and abs(int(its10[l]) - ito) <= 1, (l, its10[l], ito)
        assert np.linalg.norm(Z10[l] - zo) <= 1e-6 * np.linalg.norm(zo)
        zd = ko.grounded_direct(st, B[l])
        assert its[l] > 0 and Z[l, J - 1] == 0.0
        err = np.linalg.norm(Z[l] - zd) / np.linalg.norm(zd)
        assert err <= REL_TOL, (l, err)


def test_zero_rhs_and_failing_lanes(pkg, system):
    rows, st = system
    J = st["J"]
    sysd = pkg.kss_system(rows[:, 0], rows[:, 1], rows[:, 2], st["N"], J)
    B = np.random.default_rng(9).standard_normal((4, J))
    B[2] = 0.0
    B[3, :] = 0.0
    B[3, J - 1] = 5.0  # only the ground entry: the grounded rhs is zero
    solver = pkg.KssSolver(sysd)
    try:
        Z, its = solver.solve_multi(B, tol=1e-12, max_iter=3)
        z1, it1 = solver.solve(B[0], tol=1e-12, max_iter=3)
        z0, it0 = solver.solve(B[0], tol=1e-10, max_iter=20_000)
    finally:
        solver.close()
    assert list(its) == [-1, -1, 0, 0]
    assert not Z.any()  # failed lanes zeroed, zero lanes zero
    assert it1 == -1 and not z1.any()
    from oracle import kss_oracle as ko
    zo, ito = ko.kss_pcg(st, B[0], tol=1e-10, max_iter=20_000)
    assert abs(it0 - ito) <= 1
    assert np.linalg.norm(z0 - zo) <= 1e-6 * np.linalg.norm(zo)


def test_stable_sort_u64(pkg):
    rng = np.random.default_rng(4)
    keys = rng.integers(0, 1000, size=200_000).astype(np.uint64) << np.uint64(20)
    keys[::7] = np.uint64(2**63 + 5)  # large keys and many ties
    order = pkg.stable_sort_u64(keys)
    assert np.array_equal(order, np.argsort(keys, kind="stable"))


@pytest.fixture(scope="module")
def ref_b200(oracle_mod):
    if not oracle_mod.REF_B200_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_b200.so not built (needs the reference sources)")
    return oracle_mod.REF_B200_SO


@pytest.mark.parametrize("case", ["felsdvsimul", "akm20k"])
def test_reference_akm_kss_runs_on_b200_solver(oracle_mod, ref_b200, case):
    g = np.load(GOLDEN / f"kss_{case}.npz")
    draws = 150 if case == "felsdvsimul" else 200
    seed = 42 if case == "felsdvsimul" else 20260705
    r = oracle_mod.ref_akm_kss(g["y"], g["worker"], g["firm"], leverages="jla", jla_draws=draws,
                               seed=seed, use_gpu=True, threads=1, lib_path=ref_b200)
    assert r["gpu_used"] and r["gpu_status_code"] == 1 and r["converged"]
    got = np.array([r[k][c] for k in ("plugin", "agsu", "kss")
                    for c in ("var_alpha", "var_psi", "cov_alpha_psi")])
    want = g["jla_pcg_components"]
    err = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert err.max() <= COMP_TOL, (got, want)

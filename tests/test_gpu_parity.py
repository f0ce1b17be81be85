"""GPU parity of the absorber against the oracle, through the C ABI.

Bar: for every column c, ||v~_c - v~*_c|| <= REL_TOL * ||v_c|| where v~* is the
oracle's tightly converged projection (IT-MAP to 1e-13, pinned against the
reference core by test_oracle_golden.py).  The solver's own stopping rule is
the relative residual of the projected normal equations at 1e-10 here.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8      # relative error of the within transform vs the oracle
SOLVE_TOL = 1e-10   # solver tolerance used in these tests


def _rel_err(V, ref, Vorig):
    scale = np.linalg.norm(Vorig, axis=0)
    scale[scale == 0] = 1.0
    return float((np.linalg.norm(V - ref, axis=0) / scale).max())


def _check(absorber, pkg, oracle_mod, y, X, fes, G, w=None, precision="mixed", tol=SOLVE_TOL):
    o = pkg.make_options(tol=tol, precision=precision)
    res = absorber.absorb(y, X, fes, G, w, o)
    assert res.converged
    V = np.column_stack([res.y_tilde, res.X_tilde])
    Vorig = np.column_stack([y, X])
    ref, _, ok = oracle_mod.project(y, X, fes, G, w, tol=1e-13)
    assert ok
    err = _rel_err(V, ref, Vorig)
    assert err <= REL_TOL, f"relative error {err:.3e}"
    # certificate agrees with the oracle's certificate of the same output
    a, r = oracle_mod.certify(Vorig, V, fes, G, w)
    assert res.abs_residual_rel <= max(1e-12, 10 * r) and r <= max(1e-12, 10 * res.abs_residual_rel)
    return res, V


def _akm(panels, n, three_way, seed=0, firms=500, years=10):
    p = panels.akm_two_way(n, n_firms=firms, n_years=years, seed=seed, three_way=three_way)
    return panels.subset(p, panels.drop_singletons(p.fes))


def test_reference_packed_fixture(absorber, pkg, oracle_mod):
    # tests/test_cg_breakdown.py:_packed_fixture of the reference
    i = np.arange(120)
    f1 = (i % 20).astype(np.int32)
    f2 = ((i * 7 + i // 20) % 20).astype(np.int32)
    y = 0.7 * np.sin(i / 3) + 0.2 * (f1 - 9.5) + 0.1 * (f2 - 9.5)
    X = np.cos(i / 5)[:, None]
    _check(absorber, pkg, oracle_mod, y, X, [f1, f2], [20, 20])


def test_reference_soa_fixture_weighted(absorber, pkg, oracle_mod):
    # tests/test_cg_breakdown.py:_soa_fixture of the reference (unit weights)
    i = np.arange(40)
    f1 = (i // 2).astype(np.int32)
    f2 = ((i + 1) // 2).astype(np.int32)
    y = np.sin(i / 3) + 0.2 * f1 - 0.1 * f2
    X = np.cos(i / 5)[:, None]
    _check(absorber, pkg, oracle_mod, y, X, [f1, f2], [20, 21], w=np.ones(40))


def test_validate_backends_design(absorber, pkg, oracle_mod):
    # tests/validation/VALIDATE_PYTHON_BACKENDS.py:43-54 design (unsorted primary)
    rng = np.random.default_rng(20260605)
    n = 50000
    fe1 = (np.arange(n) % 1000).astype(np.int32)
    fe2 = (np.arange(n) % 97).astype(np.int32)
    x1 = rng.normal(size=n)
    x2 = rng.normal(size=n)
    X = np.column_stack([x1, x2])
    y = 1.25 * x1 - 0.70 * x2 + 0.01 * fe1 - 0.02 * fe2 + rng.normal(scale=0.01, size=n)
    _check(absorber, pkg, oracle_mod, y, X, [fe1, fe2], [1000, 97])


@pytest.mark.parametrize("three_way", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_akm_panel(absorber, pkg, oracle_mod, panels, three_way, precision):
    p = _akm(panels, 30_000, three_way)
    _check(absorber, pkg, oracle_mod, p.y, p.X, p.fes, p.levels, precision=precision)


def test_akm_weighted(absorber, pkg, oracle_mod, panels):
    p = _akm(panels, 30_000, True, seed=5)
    w = np.random.default_rng(1).lognormal(0.0, 0.5, size=p.n)
    _check(absorber, pkg, oracle_mod, p.y, p.X, p.fes, p.levels, w=w)


def test_akm_shuffled_rows(absorber, pkg, oracle_mod, panels):
    p = _akm(panels, 30_000, True, seed=7)
    perm = np.random.default_rng(2).permutation(p.n)
    fes = [f[perm] for f in p.fes]
    _check(absorber, pkg, oracle_mod, p.y[perm], p.X[perm], fes, p.levels)


def test_single_dimension(absorber, pkg, oracle_mod, panels):
    p = _akm(panels, 10_000, False)
    _check(absorber, pkg, oracle_mod, p.y, p.X, p.fes[:1], p.levels[:1])


def test_four_dimensions_two_large(absorber, pkg, oracle_mod, panels):
    p = _akm(panels, 30_000, True, seed=11)
    fy = p.fes[1].astype(np.int64) * p.levels[2] + p.fes[2]
    fy, gfy = pkg.dense_ids(fy)
    fes = p.fes + [fy]
    keep = panels.drop_singletons(fes)
    fes = [pkg.dense_ids(f[keep])[0] for f in fes]
    G = [int(f.max()) + 1 for f in fes]
    _check(absorber, pkg, oracle_mod, p.y[keep], p.X[keep], fes, G)


def test_many_columns_batches(absorber, pkg, oracle_mod, panels):
    p = _akm(panels, 8_000, True, seed=13)
    rng = np.random.default_rng(4)
    X = rng.standard_normal((p.n, 39))  # 40 columns with y: two column batches
    _check(absorber, pkg, oracle_mod, p.y, X, p.fes, p.levels)


def test_empty_groups_zero_and_constant_columns(absorber, pkg, oracle_mod, panels):
    p = _akm(panels, 10_000, True, seed=17)
    G = [g + 5 for g in p.levels]  # levels without observations
    X = np.column_stack([p.X, np.zeros(p.n), np.full(p.n, 3.0)])
    res, V = _check(absorber, pkg, oracle_mod, p.y, X, p.fes, G)
    assert np.all(V[:, -2] == 0.0)
    assert np.abs(V[:, -1]).max() < 1e-12


def test_bitwise_deterministic(absorber, pkg, panels):
    p = _akm(panels, 30_000, True, seed=19)
    o = pkg.make_options(tol=1e-10)
    r1 = absorber.absorb(p.y, p.X, p.fes, p.levels, None, o)
    r2 = absorber.absorb(p.y, p.X, p.fes, p.levels, None, o)
    assert np.array_equal(r1.y_tilde, r2.y_tilde)
    assert np.array_equal(r1.X_tilde, r2.X_tilde)
    assert r1.iterations == r2.iterations


def test_no_large_dimension(absorber, pkg, oracle_mod, panels):
    # worker (primary) + year (small): no run structure, bins only
    p = _akm(panels, 20_000, True, seed=23)
    fes = [p.fes[0], p.fes[2]]
    keep = panels.drop_singletons(fes)
    fes = [pkg.dense_ids(f[keep])[0] for f in fes]
    G = [int(f.max()) + 1 for f in fes]
    _check(absorber, pkg, oracle_mod, p.y[keep], p.X[keep], fes, G)


def test_all_segments_long(absorber, pkg, oracle_mod):
    # primary groups of ~515 observations: every segment takes the long path
    rng = np.random.default_rng(29)
    n = 50000
    fe1 = (np.arange(n) % 50).astype(np.int32)
    fe2 = (np.arange(n) % 97).astype(np.int32)
    X = rng.normal(size=(n, 3))
    y = X @ np.array([0.5, -0.2, 0.1]) + 0.01 * fe1 + rng.normal(size=n)
    _check(absorber, pkg, oracle_mod, y, X, [fe1, fe2], [50, 97])


def test_zipf_primary_mixed_long_and_tiles(absorber, pkg, oracle_mod, panels):
    # firm (Zipf sizes) as the largest dim with year: big firms are long segments
    p = _akm(panels, 30_000, True, seed=31, firms=3000)
    fes = [p.fes[1], p.fes[2]]
    keep = panels.drop_singletons(fes)
    fes = [pkg.dense_ids(f[keep])[0] for f in fes]
    G = [int(f.max()) + 1 for f in fes]
    w = np.random.default_rng(3).lognormal(0.0, 0.5, size=int(keep.sum()))
    _check(absorber, pkg, oracle_mod, p.y[keep], p.X[keep], fes, G, w=w)


@pytest.mark.parametrize("years", [10, 20, 36, 50])
@pytest.mark.parametrize("weighted", [False, True])
def test_block_and_tile_matvec_agree(absorber, pkg, oracle_mod, panels, weighted, years):
    # the CG matvec forms solve the same system: the explicit sparse Schur
    # block of the firm dim with the dense small-dim coupling (0, the default
    # here), the general tile pass (1), block level with per-block small-dim
    # updates (2) and block level with the dense coupling through the runs (3).
    # The year counts reach each register tile of the year-year coupling
    # (<= 12, <= 24, <= 36 levels) and the shared-memory accumulator (> 36)
    p = _akm(panels, 30_000, True, seed=37, years=years)
    w = np.random.default_rng(5).lognormal(0.0, 0.5, size=p.n) if weighted else None
    outs = []
    for pk in (0, 1, 2, 3):
        o = pkg.make_options(tol=1e-10, precision="fp64", pass_kernel=pk)
        r = absorber.absorb(p.y, p.X, p.fes, p.levels, w, o)
        assert r.converged
        outs.append(np.column_stack([r.y_tilde, r.X_tilde]))
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    for o in outs[1:]:
        assert (np.linalg.norm(outs[0] - o, axis=0) / scale).max() <= 1e-9


def test_firm_coupling_over_run_ranges_with_gapped_ids(absorber, pkg, oracle_mod, panels):
    # the firm-year coupling is summed over ranges of 512 runs in firm order,
    # across firm boundaries: firm ids without runs (every even id here, and
    # five past the last) get zero rows, and the largest firms (thousands of
    # runs) span several ranges whose pieces are joined in range order
    p = _akm(panels, 120_000, True, seed=53, firms=200, years=20)
    fes = [p.fes[0], (2 * p.fes[1] + 1).astype(np.int32), p.fes[2]]
    G = [p.levels[0], 2 * p.levels[1] + 5, p.levels[2]]
    assert np.bincount(p.fes[1]).max() > 3 * 512  # obs of the largest firm: several ranges of runs
    outs = []
    for pk in (0, 1):
        o = pkg.make_options(tol=1e-10, precision="fp64", pass_kernel=pk)
        r = absorber.absorb(p.y, p.X, fes, G, None, o)
        assert r.converged
        outs.append(np.column_stack([r.y_tilde, r.X_tilde]))
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    assert (np.linalg.norm(outs[0] - outs[1], axis=0) / scale).max() <= 1e-9
    _check(absorber, pkg, oracle_mod, p.y, p.X, fes, G)


def test_pipelined_host_copies_match_single_stream(pkg, oracle_mod, panels, monkeypatch):
    """Host-array calls with more than four columns copy column groups in and
    out on their own streams while other groups are solved; the within
    transform equals the oracle's tight projection and the single-stream call
    (B200FE_PIPELINE=0 at context creation) to 1e-9 of the column norm."""
    p = _akm(panels, 40_000, True, seed=41)
    rng = np.random.default_rng(9)
    X = np.asfortranarray(np.column_stack([p.X, rng.standard_normal((p.n, 10))]))  # 13 columns
    o = pkg.make_options(tol=1e-10)
    outs = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("B200FE_PIPELINE", flag)
        ab = pkg.Absorber(0)
        try:
            r = ab.absorb(p.y, X, p.fes, p.levels, None, o)
        finally:
            ab.close()
        assert r.converged and r.precision_certified
        outs[flag] = np.column_stack([r.y_tilde, r.X_tilde])
    ref, _, ok = oracle_mod.project(p.y, X, p.fes, p.levels, tol=1e-13)
    scale = np.linalg.norm(np.column_stack([p.y, X]), axis=0)
    assert ok and (np.linalg.norm(outs["1"] - ref, axis=0) / scale).max() <= REL_TOL
    assert (np.linalg.norm(outs["1"] - outs["0"], axis=0) / scale).max() <= 1e-9

"""Heterogeneous slopes on the CPU: the oracle (oracle/slope_oracle.py, exact
weighted projection with the reference's determinant rule) pinned against the
golden vectors of the reference's absorb_fixed_effects_v6 with
HeterogeneousSlopeTerm slopes (tests/golden/slopes_*.npz), the fixture
generators, and the host-side slope-term checks of the package.
"""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

ORACLE_TOL = 1e-10   # oracle vs the reference at tol 1e-13, relative to the column norm
DENSE_MAX_N = 5000   # the dense oracle runs on the small cases only


def load(name):
    d = np.load(GOLDEN / f"slopes_{name}.npz")
    return d, json.loads(str(d["meta"]))


@pytest.mark.parametrize("name", sorted(make_golden.SLOPE_CASES))
def test_generator_reproduces_slope_inputs(name):
    _, meta = load(name)
    c = make_golden.SLOPE_CASES[name]()
    assert make_golden.slope_digest(c) == meta["input_digest"]


@pytest.mark.parametrize("name", sorted(make_golden.SLOPE_CASES))
def test_slope_oracle_matches_reference(name):
    from oracle.slope_oracle import slope_projection
    d, meta = load(name)
    if meta["n"] > DENSE_MAX_N:
        pytest.skip("dense oracle: small cases only")
    c = make_golden.SLOPE_CASES[name]()
    V = np.column_stack([c["y"], c["X"]])
    o = slope_projection(V, c["fes"], c["slopes"], c["weights"])
    rows = d["rows"]
    err = np.abs(o[rows] - d["ref_rows"]).max(axis=0) / d["ref_colnorm"]
    assert err.max() <= ORACLE_TOL
    assert np.allclose(np.linalg.norm(o, axis=0), d["ref_colnorm"], rtol=1e-9)


def test_slope_oracle_degenerate_rule():
    """A group whose z is constant keeps its intercept alone; a slope-only
    group with z = 0 contributes nothing."""
    from oracle.slope_oracle import slope_basis
    f = np.array([0, 0, 0, 1, 1, 1], dtype=np.int32)
    z = np.array([2.0, 2.0, 2.0, 1.0, 2.0, 4.0])
    B = slope_basis([f], [(0, z, True)], None, 6)
    assert B.shape[1] == 3  # group 0: intercept; group 1: intercept + slope
    z0 = np.array([0.0, 0.0, 0.0, 1.0, 2.0, 3.0])
    B = slope_basis([f], [(0, z0, False)], None, 6)
    assert B.shape[1] == 1


def test_slope_terms_host_checks(pkg):
    import importlib
    ab = importlib.import_module(pkg.__name__ + ".absorber")
    z = np.ones(4)
    vals, icpt = ab._slope_table([(1, z, True)], 2, 4)
    assert vals[0] is None and vals[1] is not None and list(icpt) == [1, 1]
    vals, icpt = ab._slope_table([ab.HeterogeneousSlopeTerm(0, z, False)], 2, 4)
    assert list(icpt) == [0, 1]
    with pytest.raises(ValueError, match="out of range"):
        ab._slope_table([(2, z, True)], 2, 4)
    with pytest.raises(ValueError, match="at most one"):
        ab._slope_table([(0, z, True), (0, z, False)], 2, 4)
    with pytest.raises(ValueError, match="length"):
        ab._slope_table([(0, np.ones(3), True)], 2, 4)


def test_slope_oracle_matches_reference_live(oracle_mod):
    """The reference core, rebuilt here, against the oracle on a fresh case."""
    if not oracle_mod.REF_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built (needs the reference sources)")
    from oracle.slope_oracle import slope_projection
    rng = np.random.default_rng(99)
    n = 1500
    f1 = rng.integers(0, 120, n).astype(np.int32)
    f2 = rng.integers(0, 9, n).astype(np.int32)
    z = rng.uniform(0, 3, n)
    X = rng.standard_normal((n, 2))
    y = X @ np.array([0.3, -0.1]) + rng.standard_normal(n)
    w = rng.uniform(0.2, 3.0, n)
    sl = [(0, z, True), (1, rng.standard_normal(n), False)]
    r = oracle_mod.ref_absorb_slopes(y, X, [f1, f2], sl, w, tol=1e-13, threads=1)
    o = slope_projection(np.column_stack([y, X]), [f1, f2], sl, w)
    scale = np.linalg.norm(o, axis=0)
    assert (np.abs(r["V"] - o).max(axis=0) / scale).max() <= ORACLE_TOL

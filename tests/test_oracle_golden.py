"""The oracle pinned against golden vectors produced by the reference core.

The fixtures in tests/golden/ were written by tests/golden/make_golden.py from
the reference's own CPU absorber (oracle/_ref, built from its sources).  These
tests run on the CPU only.
"""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

import make_golden  # noqa: E402

CASES = sorted(make_golden.CASES)


def _load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    return z, json.loads(str(z["meta"]))


def _inputs(name):
    c = make_golden.CASES[name]()
    return c["y"], np.asarray(c["X"]), c["fes"], c["weights"], c["cluster"]


@pytest.mark.parametrize("name", CASES)
def test_generator_reproduces_golden_inputs(name):
    _, meta = _load(name)
    y, X, fes, w, _ = _inputs(name)
    d = make_golden.digest(y, X, *[np.asarray(f, dtype=np.int32) for f in fes],
                           *([w] if w is not None else []))
    assert d == meta["input_digest"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_projection_matches_reference(name, oracle_mod):
    z, meta = _load(name)
    y, X, fes, w, _ = _inputs(name)
    G = meta["levels"]
    V, it, ok = oracle_mod.project(y, X, fes, G, w, tol=1e-14)
    assert ok
    rows = z["rows"]
    scale = np.linalg.norm(np.column_stack([y, X]), axis=0)
    err = np.abs(V[rows] - z["exact_rows"]).max(axis=0) / scale
    assert err.max() <= 1e-10, err
    cn = np.linalg.norm(V, axis=0)
    assert np.all(np.abs(cn - z["exact_colnorm"]) <= 1e-9 * z["exact_colnorm"] + 1e-10 * scale)


@pytest.mark.parametrize("name", CASES)
def test_oracle_comparable_mode_certifies(name, oracle_mod):
    # reghdfe-comparable at tol 1e-8: certificate limit max(8*min(tol,1e-9), 64 eps)
    z, meta = _load(name)
    y, X, fes, w, _ = _inputs(name)
    G = meta["levels"]
    V, it, ok = oracle_mod.map_demean(y, X, fes, G, w, tol=1e-8)
    assert ok
    _, rel = oracle_mod.certify(np.column_stack([y, X]), V, fes, G, w)
    assert rel <= 8e-9
    assert meta["comparable_abs_residual_rel"] <= 8e-9


@pytest.mark.parametrize("name", CASES)
def test_oracle_ols_coefficients_match_reference_fit(name, oracle_mod):
    z, meta = _load(name)
    y, X, fes, w, _ = _inputs(name)
    V, _, ok = oracle_mod.project(y, X, fes, meta["levels"], w, tol=1e-14)
    yt, Xt = V[:, 0], V[:, 1:]
    if np.linalg.norm(Xt) <= 1e-8 * np.linalg.norm(X):
        pytest.skip("regressors absorbed by the FEs (saturated design): no coefficient")
    sw = np.ones_like(yt) if w is None else w
    beta = np.linalg.solve(Xt.T @ (Xt * sw[:, None]), Xt.T @ (yt * sw))
    coef = z["coef"][: beta.size]
    assert np.allclose(beta, coef, rtol=1e-8, atol=1e-12), (beta, coef)


def test_oracle_sweep_is_a_projection(oracle_mod):
    # the restated sweep leaves an already-absorbed vector unchanged
    y, X, fes, w, _ = _inputs("packed120")
    V, _, _ = oracle_mod.project(y, X, fes, [20, 20], w, tol=1e-15)
    V2, it, ok = oracle_mod.map_demean(V[:, 0], V[:, 1:], fes, [20, 20], w, tol=1e-12)
    assert ok and it <= 2
    assert np.abs(V2 - V).max() <= 1e-12


@pytest.mark.skipif(not (Path(__file__).resolve().parents[1] / "oracle" / "_ref" /
                         "libxhdfe_ref.so").exists(), reason="reference core not built here")
def test_oracle_matches_reference_live(oracle_mod):
    y, X, fes, w, _ = _inputs("akm3w_20k")
    G = [int(f.max()) + 1 for f in fes]
    r = oracle_mod.ref_absorb(y, X, fes, w, tol=1e-14, tolerance_mode="strict-residual",
                              method="gauss-seidel")
    V, _, ok = oracle_mod.project(y, X, fes, G, w, tol=1e-14)
    scale = np.linalg.norm(np.column_stack([y, X]), axis=0)
    assert (np.linalg.norm(V - r["V"], axis=0) / scale).max() <= 1e-10

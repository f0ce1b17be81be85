"""Heterogeneous slopes on the CPU: the oracle (oracle/slope_oracle.py, exact
weighted projection with the reference's determinant rule) pinned against the
golden vectors of the reference's absorb_fixed_effects_v6 with
HeterogeneousSlopeTerm slopes (tests/golden/slopes_*.npz), the fixture
generators, the host-side slope-term checks of the package, and the algebra of
the Schur form's block diagonal for a primary with its own slope (pair sums and
2x2 block inverses, raw and centred basis) against the dense projection.
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


def _pair_blocks(tp, fp, fd, zd, w, center):
    """Diagonal blocks of the Schur complement D_d' W (I - P_p) D_d for a
    dimension d with intercept and slope zd, the primary fp carrying an
    intercept and a slope tp, from per-(primary group, group) pair sums and
    each primary group's 2x2 block inverse -- the formulas of the device's
    pair_contrib_kernel and slope_centred_inverse_kernel -- in the raw basis
    (1, t) or the centred one (1, t - tbar)."""
    Gp, Gd = fp.max() + 1, fd.max() + 1
    W = np.bincount(fp, w, Gp)
    Z = np.bincount(fp, w * tp, Gp)
    ZZ = np.bincount(fp, w * tp * tp, Gp)
    keep = W * ZZ - Z * Z > 1e-12 * np.maximum(1.0, W * ZZ)  # the reference's rule
    t = tp - (Z / W)[fp] if center else tp
    Zt = np.bincount(fp, w * t, Gp)
    SS = np.bincount(fp, w * t * t, Gp)
    det = W * SS - Zt * Zt
    m00 = np.where(keep, SS / np.where(keep, det, 1), 1 / W)
    m01 = np.where(keep, -Zt / np.where(keep, det, 1), 0.0)
    m11 = np.where(keep, W / np.where(keep, det, 1), 0.0)
    S = np.zeros((Gd, 2, 2))
    np.add.at(S, (fd, 0, 0), w)
    np.add.at(S, (fd, 0, 1), w * zd)
    np.add.at(S, (fd, 1, 1), w * zd * zd)
    key = fp.astype(np.int64) * Gd + fd
    for k in np.unique(key):
        rows = key == k
        j, g = divmod(int(k), Gd)
        ca, cb = w[rows].sum(), (w * zd)[rows].sum()
        ta, tb = (w * t)[rows].sum(), (w * zd * t)[rows].sum()

        def qf(u0, u1, v0, v1):
            return m00[j] * u0 * v0 + m01[j] * (u0 * v1 + u1 * v0) + m11[j] * u1 * v1

        S[g, 0, 0] -= qf(ca, ta, ca, ta)
        S[g, 0, 1] -= qf(ca, ta, cb, tb)
        S[g, 1, 1] -= qf(cb, tb, cb, tb)
    S[:, 1, 0] = S[:, 0, 1]
    return S


@pytest.mark.parametrize("weighted", [False, True])
def test_schur_blocks_of_a_slope_primary(weighted):
    """The pair-sum form of the Schur complement's block diagonal, for a primary
    with intercept and slope, equals the dense D_d' W (I - P_p) D_d (P_p the
    exact W-projection on the primary's basis under the reference's rule) in
    the raw and the centred basis; one-row groups and groups of constant t
    drop the slope."""
    rng = np.random.default_rng(17)
    sizes = rng.integers(1, 8, 120)
    fp = np.repeat(np.arange(120), sizes).astype(np.int32)
    n = fp.size
    tp = rng.uniform(0.0, 5.0, n)
    tp[fp % 13 == 4] = 2.5
    fd = rng.integers(0, 9, n).astype(np.int32)
    zd = rng.uniform(-1.0, 3.0, n)
    w = rng.uniform(0.3, 3.0, n) if weighted else np.ones(n)
    # dense reference: projection on the primary basis column by column
    cols = []
    for j in range(120):
        rows = fp == j
        e = np.zeros(n)
        e[rows] = 1.0
        cols.append(e)
        W, Z, ZZ = w[rows].sum(), (w * tp)[rows].sum(), (w * tp * tp)[rows].sum()
        if W * ZZ - Z * Z > 1e-12 * max(1.0, W * ZZ):
            f = np.zeros(n)
            f[rows] = tp[rows]
            cols.append(f)
    B = np.column_stack(cols)
    sw = np.sqrt(w)
    Q, _ = np.linalg.qr(B * sw[:, None])
    Gd = int(fd.max()) + 1
    dense = np.zeros((Gd, 2, 2))
    for g in range(Gd):
        D = np.zeros((n, 2))
        rows = fd == g
        D[rows, 0] = 1.0
        D[rows, 1] = zd[rows]
        A = D * sw[:, None]
        R = A - Q @ (Q.T @ A)
        dense[g] = R.T @ R
    for center in (False, True):
        S = _pair_blocks(tp, fp, fd, zd, w, center)
        scale = np.abs(dense).max()
        assert np.abs(S - dense).max() <= 1e-10 * scale, center

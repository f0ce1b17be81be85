"""Heterogeneous slopes on the B200 (b200fe_absorb_slopes), through the C ABI.

Parity: the within transform against the reference's absorb_fixed_effects_v6
with HeterogeneousSlopeTerm slopes (golden vectors, tol 1e-13) and against the
oracle's exact projection (oracle/slope_oracle.py), at REL_TOL of each
column's norm; bitwise determinism; invariance to the row order; a plain-FE
call through the slope path equal to the main absorber; the certificate and
idempotence on a 2M-row firm x tenure panel; argument errors; and the
reference's own absorb_fixed_effects_v6 with slopes running on this library
through the reference-side binding.
"""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

REL_TOL = 1e-8  # within transform vs reference / exact projection, per column norm


def _opts(pkg, tol=1e-10, **kw):  # pass_kernel 1: block Jacobi over every dim
    return pkg.make_options(tol=tol, **kw)


def _absorb(absorber, pkg, c, tol=1e-10, **kw):
    fes = [np.asarray(f, dtype=np.int32) for f in c["fes"]]
    G = [int(f.max()) + 1 for f in fes]
    return absorber.absorb(c["y"], c["X"], fes, G, c["weights"], _opts(pkg, tol, **kw),
                           slopes=c["slopes"])


def _rel(V, ref_rows, rows, colnorm):
    return (np.abs(V[rows] - ref_rows).max(axis=0) / colnorm).max()


@pytest.mark.parametrize("name", sorted(make_golden.SLOPE_CASES))
def test_slopes_match_reference_golden(absorber, pkg, name):
    d = np.load(GOLDEN / f"slopes_{name}.npz")
    meta = json.loads(str(d["meta"]))
    c = make_golden.SLOPE_CASES[name]()
    assert make_golden.slope_digest(c) == meta["input_digest"]
    r = _absorb(absorber, pkg, c)
    assert r.converged
    V = np.column_stack([r.y_tilde, r.X_tilde])
    assert _rel(V, d["ref_rows"], d["rows"], d["ref_colnorm"]) <= REL_TOL
    assert r.precision_certified


@pytest.mark.parametrize("name", ["stata600", "mixed3kw", "degenerate2k"])
def test_slopes_match_exact_projection(absorber, pkg, name):
    from oracle.slope_oracle import slope_projection
    c = make_golden.SLOPE_CASES[name]()
    r = _absorb(absorber, pkg, c, tol=1e-12)
    V = np.column_stack([r.y_tilde, r.X_tilde])
    o = slope_projection(np.column_stack([c["y"], c["X"]]), c["fes"], c["slopes"], c["weights"])
    scale = np.linalg.norm(np.column_stack([c["y"], c["X"]]), axis=0)
    assert (np.linalg.norm(V - o, axis=0) / scale).max() <= REL_TOL * 1e-1


def test_slopes_bitwise_deterministic(absorber, pkg):
    c = make_golden.SLOPE_CASES["akm20k"]()
    a = _absorb(absorber, pkg, c)
    b = _absorb(absorber, pkg, c)
    assert np.array_equal(a.y_tilde, b.y_tilde) and np.array_equal(a.X_tilde, b.X_tilde)
    assert a.iterations == b.iterations


def test_slopes_row_order_invariant(absorber, pkg):
    c = make_golden.SLOPE_CASES["mixed3kw"]()
    rng = np.random.default_rng(4)
    perm = rng.permutation(c["y"].shape[0])
    cp = dict(y=c["y"][perm], X=c["X"][perm], fes=[f[perm] for f in c["fes"]],
              slopes=[(d, z[perm], i) for d, z, i in c["slopes"]], weights=c["weights"][perm])
    a = _absorb(absorber, pkg, c, tol=1e-12)
    b = _absorb(absorber, pkg, cp, tol=1e-12)
    Va = np.column_stack([a.y_tilde, a.X_tilde])[perm]
    Vb = np.column_stack([b.y_tilde, b.X_tilde])
    scale = np.linalg.norm(Va, axis=0)
    assert (np.linalg.norm(Va - Vb, axis=0) / scale).max() <= 1e-10


def test_slope_path_without_slopes_equals_main_absorber(absorber, pkg, libmod, panels):
    """All dims plain: the slope solver's projection equals the main solver's."""
    p = panels.akm_two_way(40_000, n_firms=800, seed=5, three_way=True)
    p = panels.subset(p, panels.drop_singletons(p.fes))
    G = np.asarray(p.levels, dtype=np.int32)
    main = absorber.absorb(p.y, p.X, p.fes, G, None, _opts(pkg, 1e-11, precision="fp64"))
    # a slope term on no dim: call the slope entry point directly with all-NULL values
    import ctypes
    n, k = p.n, p.k
    y_out = np.empty(n)
    X_out = np.empty((n, k), order="F")
    r = libmod.Result()
    o = _opts(pkg, 1e-11)
    gids = [np.ascontiguousarray(f, dtype=np.int32) for f in p.fes]
    arr = (ctypes.c_void_p * len(gids))(*[g.ctypes.data for g in gids])
    zs = (ctypes.c_void_p * len(gids))()
    X = np.asfortranarray(p.X)
    rc = absorber.lib.b200fe_absorb_slopes(absorber.handle, p.y.ctypes.data, X.ctypes.data, n, k,
                                           len(gids), arr, G.ctypes.data, zs, None, None,
                                           ctypes.byref(o), y_out.ctypes.data, X_out.ctypes.data,
                                           ctypes.byref(r))
    assert rc == libmod.OK
    Vm = np.column_stack([main.y_tilde, main.X_tilde])
    Vs = np.column_stack([y_out, X_out])
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    assert (np.linalg.norm(Vm - Vs, axis=0) / scale).max() <= REL_TOL


def test_slopes_full_panel_certificate_and_idempotence(absorber, pkg, panels):
    """2M rows, worker + firm##c.tenure + year: converged, certified, and
    absorbing the output again moves it by less than the tolerance."""
    p, sl = panels.akm_firm_tenure_slopes(2_000_000, n_firms=20_000, seed=8)
    G = np.asarray(p.levels, dtype=np.int32)
    r = absorber.absorb(p.y, p.X, p.fes, G, None, _opts(pkg, 1e-8), slopes=sl)
    assert r.converged and r.precision_certified
    r2 = absorber.absorb(r.y_tilde, r.X_tilde, p.fes, G, None, _opts(pkg, 1e-8), slopes=sl)
    V1 = np.column_stack([r.y_tilde, r.X_tilde])
    V2 = np.column_stack([r2.y_tilde, r2.X_tilde])
    scale = np.linalg.norm(np.column_stack([p.y, p.X]), axis=0)
    assert (np.linalg.norm(V1 - V2, axis=0) / scale).max() <= REL_TOL


def test_slopes_device_entry_point(absorber, pkg):
    import torch
    c = make_golden.SLOPE_CASES["mixed3kw"]()
    host = _absorb(absorber, pkg, c)
    n = c["y"].shape[0]
    v = torch.tensor(np.column_stack([c["y"], c["X"]]).T.copy(), device="cuda")
    gids = [torch.tensor(np.asarray(f, dtype=np.int32), device="cuda") for f in c["fes"]]
    G = [int(np.max(f)) + 1 for f in c["fes"]]
    sl = [(d, torch.tensor(z, device="cuda"), i) for d, z, i in c["slopes"]]
    w = torch.tensor(c["weights"], device="cuda")
    out, r = absorber.absorb_slopes_device(v, gids, G, sl, w, _opts(pkg))
    torch.cuda.synchronize()
    Vd = out.cpu().numpy().T
    assert r.converged and Vd.shape == (n, 4)
    assert np.array_equal(Vd[:, 0], host.y_tilde) and np.array_equal(Vd[:, 1:], host.X_tilde)


def test_slopes_argument_errors(absorber, pkg):
    c = make_golden.SLOPE_CASES["stata600"]()
    fes = [np.asarray(f, dtype=np.int32) for f in c["fes"]]
    z = c["slopes"][0][1].copy()
    z[5] = np.nan
    with pytest.raises(ValueError):
        absorber.absorb(c["y"], c["X"], fes, [60, 10], None, _opts(pkg), slopes=[(0, z, True)])
    with pytest.raises(pkg.AbsorberError):
        absorber.absorb(c["y"], c["X"], fes, [50, 10], None, _opts(pkg), slopes=c["slopes"])
    with pytest.raises(ValueError):
        absorber.absorb(c["y"], c["X"], fes, [60, 10], None, _opts(pkg), slopes=c["slopes"],
                        save_fe=True)


def test_reference_slopes_dispatch_to_b200(oracle_mod):
    """The reference's absorb_fixed_effects_v6 with slopes, built with CUDA on
    over the reference-side binding, runs on this library (GPU status 1) and
    matches its own CPU absorber."""
    if not oracle_mod.REF_B200_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_b200.so not built (needs the reference sources)")
    c = make_golden.SLOPE_CASES["mixed3kw"]()
    g = oracle_mod.ref_absorb_slopes(c["y"], c["X"], c["fes"], c["slopes"], c["weights"],
                                     tol=1e-10, gpu_backend="cuda", lib_path=oracle_mod.REF_B200_SO)
    assert g["gpu_status_code"] == 1 and g["converged"]
    d = np.load(GOLDEN / "slopes_mixed3kw.npz")
    assert _rel(g["V"], d["ref_rows"], d["rows"], d["ref_colnorm"]) <= REL_TOL


def test_slopes_schur_and_block_jacobi_agree(absorber, pkg):
    """Worker (plain, the most groups) eliminated exactly vs block Jacobi over
    every dimension: same projection, fewer iterations."""
    c = make_golden.SLOPE_CASES["akm20k"]()
    a = _absorb(absorber, pkg, c, tol=1e-11)
    b = _absorb(absorber, pkg, c, tol=1e-11, pass_kernel=1)
    assert a.converged and b.converged
    Va = np.column_stack([a.y_tilde, a.X_tilde])
    Vb = np.column_stack([b.y_tilde, b.X_tilde])
    scale = np.linalg.norm(np.column_stack([c["y"], c["X"]]), axis=0)
    assert (np.linalg.norm(Va - Vb, axis=0) / scale).max() <= 1e-9
    assert a.iterations < b.iterations


@pytest.mark.parametrize("weighted", [False, True])
def test_slopes_schur_matches_exact_projection(absorber, pkg, panels, weighted):
    from oracle.slope_oracle import slope_projection
    p, sl = panels.akm_firm_tenure_slopes(3000, n_firms=80, seed=12)
    w = np.random.default_rng(1).uniform(0.3, 3.0, p.n) if weighted else None
    c = dict(y=p.y, X=p.X, fes=p.fes, slopes=sl, weights=w)
    r = _absorb(absorber, pkg, c, tol=1e-12)
    assert r.converged and r.primary_dim == 0
    V0 = np.column_stack([p.y, p.X])
    o = slope_projection(V0, p.fes, sl, w)
    V = np.column_stack([r.y_tilde, r.X_tilde])
    assert (np.linalg.norm(V - o, axis=0) / np.linalg.norm(V0, axis=0)).max() <= REL_TOL * 1e-1


@pytest.mark.parametrize("weighted", [False, True])
def test_slopes_schur_long_primary_groups(absorber, pkg, weighted):
    """Primary groups longer than one chunk (the fused projection's fix-up
    path): Schur form equals block Jacobi over every dimension."""
    rng = np.random.default_rng(21)
    k = 12_000  # primary groups: mostly 2-7 rows, 2% of them 65-600 rows
    sizes = np.where(rng.random(k) < 0.02, rng.integers(65, 600, k), rng.integers(2, 8, k))
    g1 = np.repeat(np.arange(k), sizes).astype(np.int32)
    n = g1.size
    g2 = rng.integers(0, 300, n).astype(np.int32)
    g3 = rng.integers(0, 12, n).astype(np.int32)
    z = rng.uniform(0, 4, n)
    X = rng.standard_normal((n, 3))
    y = X @ np.array([0.5, -1.0, 0.2]) + 0.1 * z * (g2 % 7) + rng.standard_normal(n)
    w = rng.uniform(0.3, 3.0, n) if weighted else None
    c = dict(y=y, X=X, fes=[g1, g2, g3], slopes=[(1, z, True)], weights=w)
    assert np.bincount(g1).max() > 64 and int(g1.max()) + 1 > 300
    a = _absorb(absorber, pkg, c, tol=1e-11)
    b = _absorb(absorber, pkg, c, tol=1e-11, pass_kernel=1)
    assert a.converged and b.converged and a.primary_dim == 0
    Va = np.column_stack([a.y_tilde, a.X_tilde])
    Vb = np.column_stack([b.y_tilde, b.X_tilde])
    scale = np.linalg.norm(np.column_stack([y, X]), axis=0)
    assert (np.linalg.norm(Va - Vb, axis=0) / scale).max() <= 1e-9
    assert a.precision_certified


def _slope_primary_case(k, seed, weighted, intercept, long_share):
    """Primary groups (the most groups) with their own slope t: mostly 1-7
    rows, long_share of them 65-300 rows; t constant inside every 97th group."""
    rng = np.random.default_rng(seed)
    sizes = np.where(rng.random(k) < long_share, rng.integers(65, 300, k), rng.integers(1, 8, k))
    g1 = np.repeat(np.arange(k), sizes).astype(np.int32)
    n = g1.size
    g2 = rng.integers(0, max(20, k // 20), n).astype(np.int32)
    g3 = rng.integers(0, 10, n).astype(np.int32)
    t = rng.uniform(0.0, 5.0, n)
    t[g1 % 97 == 5] = 2.0
    X = rng.standard_normal((n, 3))
    y = X @ np.array([0.5, -1.0, 0.2]) + 0.3 * t * (g1 % 5) + rng.standard_normal(n)
    w = rng.uniform(0.3, 3.0, n) if weighted else None
    return dict(y=y, X=X, fes=[g1, g2, g3], slopes=[(0, t, intercept)], weights=w)


@pytest.mark.parametrize("intercept", [True, False])
@pytest.mark.parametrize("weighted", [False, True])
def test_slopes_schur_slope_primary_exact(absorber, pkg, weighted, intercept):
    """worker##c.t (2x2 primary blocks) and worker#c.t (slope only) eliminated
    exactly: the oracle's projection, with one-row groups and groups of
    constant t on the pseudo-inverse and long groups on the fix-up path."""
    c = _slope_primary_case(500, 41, weighted, intercept, 0.02)
    G = [int(f.max()) + 1 for f in c["fes"]]
    assert G[0] > G[1] and np.bincount(c["fes"][0]).max() > 64
    r = _oracle_check(absorber, pkg, c["y"], c["X"], c["fes"], G, c["slopes"], c["weights"])
    assert r.converged and r.primary_dim == 0


@pytest.mark.parametrize("intercept", [True, False])
@pytest.mark.parametrize("weighted", [False, True])
def test_slopes_schur_slope_primary_agrees(absorber, pkg, weighted, intercept):
    """A slope primary eliminated exactly vs block Jacobi over every
    dimension on a 12k-group panel: same projection, fewer iterations."""
    c = _slope_primary_case(12_000, 42, weighted, intercept, 0.01)
    a = _absorb(absorber, pkg, c, tol=1e-11)
    b = _absorb(absorber, pkg, c, tol=1e-11, pass_kernel=1)
    assert a.converged and b.converged and a.primary_dim == 0
    Va = np.column_stack([a.y_tilde, a.X_tilde])
    Vb = np.column_stack([b.y_tilde, b.X_tilde])
    scale = np.linalg.norm(np.column_stack([c["y"], c["X"]]), axis=0)
    assert (np.linalg.norm(Va - Vb, axis=0) / scale).max() <= 1e-9
    assert a.iterations < b.iterations
    assert a.precision_certified


def test_slopes_many_columns(absorber, pkg, panels):
    """40 columns (two column words per lane) through both forms."""
    p, sl = panels.akm_firm_tenure_slopes(20_000, n_firms=300, seed=31)
    rng = np.random.default_rng(5)
    X = np.column_stack([p.X, rng.standard_normal((p.n, 37))])
    c = dict(y=p.y, X=X, fes=p.fes, slopes=sl, weights=None)
    a = _absorb(absorber, pkg, c, tol=1e-11)
    b = _absorb(absorber, pkg, c, tol=1e-11, pass_kernel=1)
    Va = np.column_stack([a.y_tilde, a.X_tilde])
    Vb = np.column_stack([b.y_tilde, b.X_tilde])
    scale = np.linalg.norm(np.column_stack([p.y, X]), axis=0)
    assert Va.shape[1] == 40
    assert (np.linalg.norm(Va - Vb, axis=0) / scale).max() <= 1e-9


def _oracle_check(absorber, pkg, y, X, fes, G, slopes, w, tol=REL_TOL * 1e-1, **kw):
    from oracle.slope_oracle import slope_projection
    r = absorber.absorb(y, X, [np.asarray(f, dtype=np.int32) for f in fes], G, w,
                        _opts(pkg, 1e-12, **kw), slopes=slopes)
    V0 = np.column_stack([y, X])
    V = np.column_stack([r.y_tilde, r.X_tilde])
    o = slope_projection(V0, fes, slopes, w)
    scale = np.maximum(np.linalg.norm(V0, axis=0), 1e-300)
    assert (np.linalg.norm(V - o, axis=0) / scale).max() <= tol
    return r


@pytest.mark.parametrize("form", [0, 1])
def test_slopes_edge_cases(absorber, pkg, form):
    """Empty groups (num_groups above the ids present), zero weights, a slope
    that is zero everywhere, a group whose slope values are constant."""
    rng = np.random.default_rng(8)
    n = 900
    f1 = rng.integers(0, 150, n).astype(np.int32)
    f2 = rng.integers(0, 20, n).astype(np.int32)
    X = rng.standard_normal((n, 2))
    y = rng.standard_normal(n)
    z = rng.uniform(-2, 2, n)
    z[f2 == 3] = 1.5                   # constant slope values in one group
    w = rng.uniform(0.5, 2.0, n)
    w[::17] = 0.0                      # zero weights
    zero = np.zeros(n)
    r = _oracle_check(absorber, pkg, y, X, [f1, f2, f2], [160, 25, 25],
                      [(1, z, True), (2, zero, False)], w, pass_kernel=form)
    assert r.fe_levels == [160, 25, 25]


def test_slopes_tiny(absorber, pkg):
    y = np.array([1.0, 2.0, 4.0, 3.0, 5.0])
    X = np.array([[0.5], [1.0], [0.0], [2.0], [1.5]])
    f = np.array([0, 0, 1, 1, 1], dtype=np.int32)
    z = np.array([1.0, 2.0, 1.0, 2.0, 4.0])
    _oracle_check(absorber, pkg, y, X, [f], [2], [(0, z, True)], None)

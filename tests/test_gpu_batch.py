"""An uneven batch of independent panels through one absorber context.

The shape of the reference's batch workload -- independent panels of uneven
size, 2 or 3 FE dimensions, analytic weights lognormal(0, 0.5), worker-clustered
SEs, every solve checked against the FP64 oracle -- scaled to sizes (2k-80k
rows) at which the reference's CPU core checks each solve in seconds:

* the reference's own fit (src/hdfe_regressor_v11.cpp, HdfeRegressorV11::fit)
  dispatching its absorptions to this library through the reference-side
  binding, against the same fit on its CPU core in strict-residual mode:
  coefficients and SEs at 1e-8 relative;
* this library's partial_out + run_ols (cluster) against the reference's
  partial_out (CPU, strict-residual) + run_ols at the same n_effective:
  within transform at 1e-8 of the column norm, coefficients and SEs at 1e-8;
* the batch solved twice through one reused context, and once with a fresh
  context per panel: bitwise equal (workspace reuse across uneven sizes leaks
  no state).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8  # within transform (column norm) and coefficients
SE_TOL = 1e-8   # SEs of the reference's fit, GPU solve vs strict CPU solve


def _batch(panels, count=12, seed=5):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(2_000), np.log(80_000), count)).astype(int)
    dims = rng.integers(2, 4, count)
    out = []
    for i, (n, d) in enumerate(zip(sizes, dims)):
        p = panels.akm_two_way(int(n), n_firms=max(40, int(n) // 80), seed=300 + i,
                               three_way=bool(d == 3))
        p.weights = rng.lognormal(0.0, 0.5, p.n)
        out.append(p)
    return out


@pytest.fixture(scope="module")
def batch(panels):
    return _batch(panels)


def test_batch_reference_fit_on_b200(oracle_mod, batch):
    if not oracle_mod.REF_B200_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_b200.so not built (needs the reference sources)")
    so = oracle_mod.REF_B200_SO
    for p in batch:
        fg = oracle_mod.ref_fit(p.y, p.X, p.fes, p.weights, p.cluster, tol=1e-10,
                                gpu_backend="cuda", lib_path=so)
        fc = oracle_mod.ref_fit(p.y, p.X, p.fes, p.weights, p.cluster, tol=1e-14,
                                tolerance_mode="strict-residual", gpu_backend="cpu", lib_path=so)
        assert fg["gpu_status_code"] == 1, p.n
        assert fg["nobs"] == fc["nobs"] and fg["converged"]
        assert np.allclose(fg["coef"], fc["coef"], rtol=REL_TOL, atol=1e-12), p.n
        assert np.allclose(fg["se"], fc["se"], rtol=SE_TOL, atol=1e-12), p.n


def test_batch_partial_out_and_cluster_ols(pkg, oracle_mod, batch):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    for p in batch:
        ours = pkg.partial_out(p.y, p.X, p.fes, p.weights, tol=1e-10)
        ref = oracle_mod.ref_partial_out(p.y, p.X, p.fes, p.weights, tol=1e-14,
                                         tolerance_mode="strict-residual", gpu_backend="cpu")
        assert ours.converged
        assert np.array_equal(ours.sample_index, ref["sample_index"]), p.n
        keep = ours.sample_index
        V = np.column_stack([ours.y_tilde, ours.X_tilde])
        Vo = np.column_stack([p.y, p.X])[keep]
        err = np.linalg.norm(V - ref["V"], axis=0) / np.linalg.norm(Vo, axis=0)
        assert err.max() <= REL_TOL, (p.n, err)
        w, cl = p.weights[keep], p.cluster[keep]
        n_eff = keep.size - sum(int(np.unique(f[keep]).size) for f in p.fes[1:])
        o = pkg.run_ols(ours.y_tilde, ours.X_tilde, w, cl, se_type="cluster",
                        n_effective=float(n_eff))
        r = oracle_mod.ref_run_ols(ref["V"][:, 0], ref["V"][:, 1:], w, cl, se_type="cluster",
                                   n_effective=float(n_eff))
        assert np.allclose(o.coefficients, r["coef"], rtol=REL_TOL, atol=1e-12), p.n
        assert np.allclose(o.std_errors, r["se"], rtol=REL_TOL, atol=1e-12), p.n
        assert o.num_clusters == r["num_clusters"]


def test_batch_context_reuse_is_bitwise_stable(pkg, batch):
    opts = pkg.make_options(tol=1e-8)
    ctx = pkg.Absorber(0)
    try:
        first = [ctx.absorb(p.y, p.X, p.fes, p.levels, p.weights, opts) for p in batch]
        second = [ctx.absorb(p.y, p.X, p.fes, p.levels, p.weights, opts) for p in batch[::-1]]
    finally:
        ctx.close()
    for p, a, b in zip(batch, first, second[::-1]):
        fresh = pkg.Absorber(0)
        try:
            c = fresh.absorb(p.y, p.X, p.fes, p.levels, p.weights, opts)
        finally:
            fresh.close()
        for r in (b, c):
            assert np.array_equal(a.y_tilde, r.y_tilde) and np.array_equal(a.X_tilde, r.X_tilde)
            assert a.iterations == r.iterations


def test_graph_replay_matches_plain_launches(pkg, batch, monkeypatch):
    """The PCG's check blocks replayed as CUDA graphs give bitwise the same
    within transform, iteration count and kernel count as plain launches
    (B200FE_GRAPHS=0 at context creation), across panels of different size
    sharing one context (the executable updated in place)."""
    opts = pkg.make_options(tol=1e-8)
    runs = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("B200FE_GRAPHS", flag)
        ctx = pkg.Absorber(0)
        try:
            runs[flag] = [ctx.absorb(p.y, p.X, p.fes, p.levels, p.weights, opts) for p in batch]
        finally:
            ctx.close()
    for a, b in zip(runs["1"], runs["0"]):
        assert np.array_equal(a.y_tilde, b.y_tilde) and np.array_equal(a.X_tilde, b.X_tilde)
        assert a.iterations == b.iterations and a.kernel_launches == b.kernel_launches


def test_concurrent_batch_equals_sequential_calls(pkg, batch):
    """absorb_many (three host threads, each with its own context and CUDA
    stream) gives every panel bitwise the answer of a sequential absorb_device
    call, and the per-panel clustered OLS equal the sequential ones."""
    import torch
    dev = torch.device("cuda", 0)
    opts = pkg.make_options(tol=1e-8)
    jobs = []
    for p in batch:
        v = torch.empty((p.k + 1, p.n), dtype=torch.float64, device=dev)
        v[0].copy_(torch.from_numpy(p.y))
        v[1:].copy_(torch.from_numpy(np.ascontiguousarray(p.X.T)))
        jobs.append((v, [torch.from_numpy(np.ascontiguousarray(f)).to(dev) for f in p.fes], p.levels,
                     torch.from_numpy(p.weights).to(dev),
                     torch.from_numpy(p.fes[0].astype(np.int32)).to(dev)))
    ols = {"se_type": "cluster"}
    conc = pkg.absorb_many(jobs, workers=3, options=opts, ols=ols)
    ab = pkg.Absorber(0)
    try:
        for (v, g, G, w, cl), (out_c, r_c, o_c) in zip(jobs, conc):
            out_s, r_s = ab.absorb_device(v, g, G, w, opts)
            torch.cuda.synchronize()
            assert torch.equal(out_c, out_s) and r_c.iterations == r_s.iterations
            o_s = pkg.run_ols(out_s[0], out_s[1:], w, cl, se_type="cluster")
            assert np.array_equal(o_c.coefficients, o_s.coefficients)
            assert np.array_equal(o_c.std_errors, o_s.std_errors)
    finally:
        ab.close()

"""The learned warm start on the GPU, through the C ABI.

* the tensor-core forward pass and the device gradient of the loss against the
  FP64 CPU restatement (oracle/mlp_oracle.py), with the same BF16 roundings;
* the device Adam step against the oracle's;
* the training samples of a panel: one per level of the non-primary dims and
  column, finite, with targets built from the converged solution;
* a network trained from scratch on small seeded panels, installed in an
  absorber: on held-out panels the warm-started solves take fewer iterations
  than the cold ones (the gain), every solve converges (tol 1e-10), and the
  warm within transform equals the cold one to 1e-8 of the column norm and the
  oracle's tight projection to 1e-8 (the plain solver decides the answer).
"""

import numpy as np
import pytest

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8


@pytest.fixture(scope="module")
def learned(pkg):
    return pkg.learned


def _params(seed, noise=0.05):
    rng = np.random.default_rng(seed)
    p = mo.init_params(seed).astype(np.float64)
    p += noise * rng.standard_normal(p.size)
    return p.astype(np.float32)


def test_forward_matches_oracle(absorber, learned):
    import torch
    rng = np.random.default_rng(11)
    p = _params(1)
    X = rng.standard_normal((5000, mo.N_IN)).astype(np.float32)
    y = learned.forward(absorber, torch.from_numpy(p).cuda(), torch.from_numpy(X).cuda()).cpu().numpy()
    ref, _ = mo.forward(p, X)
    scale = np.abs(ref).max()
    # FP32 accumulation vs FP64 may round an activation to the neighbouring BF16 value
    assert np.abs(y - ref).max() <= 2e-2 * scale, np.abs(y - ref).max() / scale
    assert np.median(np.abs(y - ref)) <= 1e-3 * scale


def test_gradient_matches_oracle(absorber, learned):
    import torch
    rng = np.random.default_rng(12)
    p = _params(2)
    n = 3000
    X = rng.standard_normal((n, mo.N_IN)).astype(np.float32)
    T = np.column_stack([rng.standard_normal((n, 2)), rng.uniform(0.2, 1.0, (n, 2))]).astype(np.float32)
    g, loss = learned.grad(absorber, torch.from_numpy(p).cuda(), torch.from_numpy(X).cuda(),
                           torch.from_numpy(T).cuda())
    g = g.cpu().numpy()
    lref, gref = mo.loss_and_grad(p, X, T)
    assert abs(loss - lref) <= 1e-4 * abs(lref)
    assert np.linalg.norm(g - gref) <= 5e-3 * np.linalg.norm(gref)
    # per layer, too (the small output layer must not hide in the norm)
    o = 0
    for name, shape in mo.SHAPES:
        k = int(np.prod(shape))
        gl, rl = g[o:o + k], gref[o:o + k]
        assert np.linalg.norm(gl - rl) <= 1e-2 * max(np.linalg.norm(rl), 1e-12), name
        o += k


def test_adam_step_matches_oracle(absorber, learned):
    import torch
    rng = np.random.default_rng(13)
    p = _params(3)
    g = rng.standard_normal(p.size)
    m = (0.01 * rng.standard_normal(p.size)).astype(np.float32)
    v = (0.01 * rng.random(p.size)).astype(np.float32)
    dp, dm, dv = (torch.from_numpy(a.copy()).cuda() for a in (p, m, v))
    dg = torch.from_numpy(g).cuda()
    rc = absorber.lib.b200fe_mlp_adam(absorber.handle, dp.data_ptr(), dm.data_ptr(), dv.data_ptr(),
                                      dg.data_ptr(), 3, 1e-3)
    assert rc == 0
    pr, mr, vr = mo.adam_step(p.astype(np.float64), g, m.astype(np.float64), v.astype(np.float64), 3, 1e-3)
    assert np.allclose(dp.cpu().numpy(), pr, rtol=1e-6, atol=1e-7)
    assert np.allclose(dm.cpu().numpy(), mr, rtol=1e-5, atol=1e-9)


def _device(p):
    import torch
    v = torch.empty((p.k + 1, p.n), dtype=torch.float64, device="cuda")
    v[0].copy_(torch.from_numpy(p.y))
    v[1:].copy_(torch.from_numpy(np.ascontiguousarray(p.X.T)))
    return v, [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in p.fes]


def test_samples_cover_every_level_and_column(absorber, learned, panels):
    p = panels.warmstart_panel(dict(panels.warmstart_panel_spec(0, n_min=60_000, n_max=60_001), dims=3))
    v, gids = _device(p)
    f, t, r = learned.collect_samples(absorber, v, gids, p.levels)
    non_primary = sum(p.levels) - max(p.levels)
    assert r.converged and f.shape[0] == non_primary * v.shape[0]
    assert bool(f.isfinite().all()) and bool(t.isfinite().all())
    assert float(t[:, 2].min()) >= 0.0


def test_warm_start_gain_on_held_out_panels(absorber, learned, panels, pkg, oracle_mod):
    import torch
    specs = [panels.warmstart_panel_spec(i, seed=21, n_min=100_000, n_max=400_000) for i in range(14)]
    feats, targs = [], []
    for s in specs[:10]:
        p = panels.warmstart_panel(s)
        v, gids = _device(p)
        f, t, _ = learned.collect_samples(absorber, v, gids, p.levels)
        feats.append(f.clone())
        targs.append(t.clone())
    X, T = torch.cat(feats), torch.cat(targs)
    params = learned.train(absorber, X, T, epochs=3, batch=4096, lr=2e-3, seed=0)
    # tol 1e-10, so that two solves of one projection (cold and warm) and the
    # oracle's tight projection agree to 1e-8 of the column norm; at tol 1e-8
    # each is within tolerance of the exact answer but two of them can differ
    # by twice that
    opts = pkg.make_options(tol=1e-10)
    cold_its, warm_its = [], []
    for k, s in enumerate(specs[10:]):
        p = panels.warmstart_panel(s)
        v, gids = _device(p)
        learned.set_warm_start(absorber, None)
        cold, rc = absorber.absorb_device(v, gids, p.levels, None, opts)
        cold = cold.clone()
        learned.set_warm_start(absorber, params, learned.MODE_START)
        warm, rw = absorber.absorb_device(v, gids, p.levels, None, opts)
        learned.set_warm_start(absorber, None)
        assert rc.converged and rw.converged and rw.warm_columns > 0
        scale = torch.linalg.vector_norm(v, dim=1)
        scale[scale == 0] = 1.0
        d = (torch.linalg.vector_norm(warm - cold, dim=1) / scale).max().item()
        assert d <= REL_TOL, d
        cold_its.append(rc.iterations)
        warm_its.append(rw.iterations)
        if k == 0:  # the warm answer against the oracle's tight projection
            ref, _, ok = oracle_mod.project(p.y, p.X, p.fes, p.levels, tol=1e-13)
            V = warm.cpu().numpy().T
            Vo = np.column_stack([p.y, p.X])
            err = (np.linalg.norm(V - ref, axis=0) / np.linalg.norm(Vo, axis=0)).max()
            assert ok and err <= REL_TOL, err
    print(f"held-out iterations cold {cold_its} warm {warm_its}")
    assert np.mean(warm_its) < np.mean(cold_its), (cold_its, warm_its)

"""The bulk-copy FP64 data passes (stream_kernels.cuh) against the
lane-per-column passes (B200FE_STREAM=0 at context creation) and the oracle.

The cases cover what changes the staged spans: data whose base is 8 bytes off
a 16-byte boundary with an odd number of observations (every column starts at
another offset), an output of the same offset (bulk stores of the interior,
plain stores at the ends), an output of another offset (the final pass falls
back, the RHS pass still streams), the in-place call, weights, no small dim,
two large dims, sixteen columns, a structure whose last tile holds more
empty segments than a stage (the passes fall back for the whole structure),
and 1.5M observations (about 32 tiles per CTA: every stage reused, the
producer's tile records reloaded; compared with the lane pass only).
Bar: the two passes agree to 1e-9 of the column norm and both meet the
oracle's tight projection to 1e-8.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AGREE_TOL = 1e-9
REL_TOL = 1e-8


def _panel(panels, case):
    three = case != "two_way"
    if case == "many_tiles":
        p = panels.akm_two_way(1_500_001, n_firms=20_000, seed=89, three_way=True)
    else:
        p = panels.akm_two_way(24_001, n_firms=400, seed=83, three_way=three)
    p = panels.subset(p, panels.drop_singletons(p.fes))
    rng = np.random.default_rng(5)
    cols = {"two_way": 16, "weighted": 5, "four_dims": 3}.get(case, 13)
    V = np.column_stack([p.y, p.X, rng.standard_normal((p.n, max(0, cols - 1 - p.X.shape[1])))])[:, :cols]
    fes, G = list(p.fes), list(p.levels)
    w = rng.lognormal(0.0, 0.5, size=p.n) if case == "weighted" else None
    if case == "four_dims":
        fx = ((np.asarray(fes[1]) * 7 + np.asarray(fes[2])) % 997).astype(np.int32)
        uniq, fx = np.unique(fx, return_inverse=True)
        fes, G = fes + [fx.astype(np.int32)], G + [len(uniq)]
    if case == "empty_tail":
        G[0] += 1000  # a thousand workers without observations
    return np.ascontiguousarray(V), fes, G, w


def _solve(pkg, monkeypatch, flag, V, fes, G, w, v_off, out_mode):
    import torch
    monkeypatch.setenv("B200FE_STREAM", flag)
    ab = pkg.Absorber(0)
    try:
        n, cols = V.shape
        dev = torch.device("cuda", 0)
        flat = torch.empty(cols * n + 2, dtype=torch.float64, device=dev)
        v = flat[v_off:v_off + cols * n].view(cols, n)
        v.copy_(torch.from_numpy(np.ascontiguousarray(V.T)))
        if out_mode == "inplace":
            out = v
        else:
            o_off = v_off if out_mode == "same" else 1 - v_off
            oflat = torch.empty(cols * n + 2, dtype=torch.float64, device=dev)
            out = oflat[o_off:o_off + cols * n].view(cols, n)
        gids = [torch.from_numpy(np.ascontiguousarray(f, dtype=np.int32)).to(dev) for f in fes]
        wt = None if w is None else torch.from_numpy(w).to(dev)
        out, r = ab.absorb_device(v, gids, G, wt, pkg.make_options(tol=1e-10), out=out)
        torch.cuda.synchronize()
        assert r.converged and r.precision_certified
        return out.cpu().numpy().T.copy(), r
    finally:
        ab.close()


@pytest.mark.parametrize("case,v_off,out_mode", [
    ("three_way", 1, "same"),
    ("three_way", 1, "other"),
    ("three_way", 0, "inplace"),
    ("weighted", 1, "same"),
    ("two_way", 1, "same"),
    ("four_dims", 0, "same"),
    ("empty_tail", 1, "same"),
    ("many_tiles", 1, "same"),
])
def test_stream_pass_matches_lane_pass_and_oracle(pkg, oracle_mod, panels, monkeypatch, case, v_off, out_mode):
    V, fes, G, w = _panel(panels, case)
    if V.shape[0] % 2 == 0:  # odd n: the columns start at alternating offsets
        V, fes = V[:-1], [f[:-1] for f in fes]
        w = None if w is None else w[:-1]
    out_s, r_s = _solve(pkg, monkeypatch, "1", V, fes, G, w, v_off, out_mode)
    out_l, r_l = _solve(pkg, monkeypatch, "0", V, fes, G, w, v_off, out_mode)
    scale = np.linalg.norm(V, axis=0)
    scale[scale == 0] = 1.0
    assert (np.linalg.norm(out_s - out_l, axis=0) / scale).max() <= AGREE_TOL
    if case == "many_tiles":  # about 32 tiles per CTA: the stage ring wraps, tile records reload
        return
    ref, _, ok = oracle_mod.project(V[:, 0], V[:, 1:], fes, G, w, tol=1e-13)
    assert ok
    assert (np.linalg.norm(out_s - ref, axis=0) / scale).max() <= REL_TOL
    assert abs(r_s.abs_residual_rel - r_l.abs_residual_rel) <= 1e-3 * max(r_l.abs_residual_rel, 1e-14) + 1e-14

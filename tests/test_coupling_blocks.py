"""The year-coupling blocks of the Schur system, restated on the CPU.

The structure build (setup_kernels.cuh) computes, from runs (maximal stretches of
one worker at one firm, in worker order) and the worker segments,

    C_fy[f][h]  = sum_{runs m of f} ( y_m[h] - c_m Y_s(m)[h] / W_s(m) )
    C_yy[h][h'] = W_h [h = h'] - sum_s Y_s[h] Y_s[h'] / W_s

with y_m, Y_s the year weights of run m and segment s and c_m, W_s their total
weights.  These tests check that algebra against the dense blocks
D_f' W (I - P_w) D_y and D_y' W (I - P_w) D_y, and that the way the device sums
C_fy (coupling_fy_range_kernel + coupling_fy_join_kernel: fixed ranges of R runs
in firm order across firm boundaries; the piece of a firm that began before a
range in slot 0, the piece of a firm that begins in it and ends after it in slot
1; split firms joined in range order; zero rows for firm ids without runs) gives
every firm's row.  The GPU tests compare the kernels themselves with the tile
pass and the oracle (test_gpu_parity.py).
"""

import numpy as np
import pytest


def _panel(seed, n=3000, workers=300, firms=40, years=12, weighted=False, gapped=True):
    rng = np.random.default_rng(seed)
    w_id = np.sort(rng.integers(0, workers, n))
    # workers stay at a firm for a few consecutive years, then may move
    f_id = np.empty(n, np.int64)
    y_id = np.empty(n, np.int64)
    for w in np.unique(w_id):
        idx = np.flatnonzero(w_id == w)
        start = rng.integers(0, years)
        f = rng.zipf(1.5) % firms
        for j, i in enumerate(idx):
            if rng.random() < 0.2:
                f = rng.zipf(1.5) % firms
            f_id[i] = f
            y_id[i] = (start + j + (rng.random() < 0.1)) % years
    G_f = firms
    if gapped:  # even ids and the last three carry no observations
        f_id = 2 * f_id + 1
        G_f = 2 * firms + 3
    wts = rng.lognormal(0.0, 0.5, n) if weighted else np.ones(n)
    return w_id, f_id, y_id, wts, workers, G_f, years


def _dense_blocks(w_id, f_id, y_id, wts, Gp, Gf, Gy):
    n = len(w_id)
    Dp = np.zeros((n, Gp)); Dp[np.arange(n), w_id] = 1
    Df = np.zeros((n, Gf)); Df[np.arange(n), f_id] = 1
    Dy = np.zeros((n, Gy)); Dy[np.arange(n), y_id] = 1
    Wp = Dp.T @ (wts[:, None] * Dp)
    inv = np.zeros(Gp)
    d = np.diag(Wp)
    inv[d > 0] = 1.0 / d[d > 0]
    # (I - P_w) D_y with P_w = D_p (D_p' W D_p)^-1 D_p' W
    MDy = Dy - Dp @ (inv[:, None] * (Dp.T @ (wts[:, None] * Dy)))
    return Df.T @ (wts[:, None] * MDy), Dy.T @ (wts[:, None] * MDy)


def _runs(w_id, f_id, y_id, wts, Gy):
    """Runs in worker order: (firm, segment, y_m, c_m), and segment Y_s, W_s."""
    o = np.argsort(w_id, kind="stable")
    w, f, y, c = w_id[o], f_id[o], y_id[o], wts[o]
    start = np.r_[True, (w[1:] != w[:-1]) | (f[1:] != f[:-1])]
    rid = np.cumsum(start) - 1
    nr = rid[-1] + 1
    run_f = f[start]
    run_s = w[start]
    ym = np.zeros((nr, Gy))
    np.add.at(ym, (rid, y), c)
    cm = np.bincount(rid, weights=c, minlength=nr)
    Gp = w.max() + 1
    Ys = np.zeros((Gp, Gy))
    np.add.at(Ys, (w, y), c)
    Ws = np.bincount(w, weights=c, minlength=Gp)
    return run_f, run_s, ym, cm, Ys, Ws


def _run_rows(run_s, ym, cm, Ys, Ws):
    inv = np.where(Ws > 0, 1.0 / np.where(Ws > 0, Ws, 1.0), 0.0)
    return ym - (cm * inv[run_s])[:, None] * Ys[run_s]


@pytest.mark.parametrize("weighted", [False, True])
def test_run_formulas_equal_dense_blocks(weighted):
    w_id, f_id, y_id, wts, Gp, Gf, Gy = _panel(11, weighted=weighted)
    Cfy_d, Cyy_d = _dense_blocks(w_id, f_id, y_id, wts, Gp, Gf, Gy)
    run_f, run_s, ym, cm, Ys, Ws = _runs(w_id, f_id, y_id, wts, Gy)
    rows = _run_rows(run_s, ym, cm, Ys, Ws)
    Cfy = np.zeros((Gf, Gy))
    np.add.at(Cfy, run_f, rows)
    inv = np.where(Ws > 0, 1.0 / np.where(Ws > 0, Ws, 1.0), 0.0)
    Cyy = np.diag(Ys.sum(axis=0)) - (Ys * inv[:, None]).T @ Ys
    scale = np.abs(Cyy_d).max()
    assert np.abs(Cfy - Cfy_d).max() <= 1e-12 * scale
    assert np.abs(Cyy - Cyy_d).max() <= 1e-12 * scale


def _ranges_sum(sorted_f, rows, G, R):
    """The device's range partition of C_fy, step for step."""
    nr = len(sorted_f)
    SG = rows.shape[1]
    grp_off = np.searchsorted(sorted_f, np.arange(G + 1), side="left")
    nranges = -(-nr // R)
    out = np.full((G, SG), np.nan)
    part = np.full((nranges, 2, SG), np.nan)
    for rg in range(nranges):
        rb, re = rg * R, min(rg * R + R, nr)
        cur = sorted_f[rb]
        prev = sorted_f[rb - 1] if rb > 0 else -1
        if cur != prev:
            out[prev + 1:cur] = 0.0

        def flush(f, acc):
            fb, fe = grp_off[f], grp_off[f + 1]
            if fb >= rb and fe <= re:
                out[f] = acc
            elif fb < rb:
                part[rg, 0] = acc
            else:
                part[rg, 1] = acc

        acc = np.zeros(SG)
        for j in range(rb, re):
            g = sorted_f[j]
            if g != cur:
                flush(cur, acc)
                out[cur + 1:g] = 0.0
                acc = np.zeros(SG)
                cur = g
            acc = acc + rows[j]
        flush(cur, acc)
        if re == nr:
            out[cur + 1:G] = 0.0
    for r in range(nranges):  # the join
        rb, re = r * R, min(r * R + R, nr)
        f = sorted_f[re - 1]
        fb, fe = grp_off[f], grp_off[f + 1]
        if fb < rb or fe <= re:
            continue
        r1 = (fe - 1) // R
        v = part[r, 1].copy()
        for q in range(r + 1, r1 + 1):
            v = v + part[q, 0]
        out[f] = v
    return out


@pytest.mark.parametrize("R", [1, 5, 64, 100000])
@pytest.mark.parametrize("weighted", [False, True])
def test_range_partition_gives_every_firm_row(R, weighted):
    w_id, f_id, y_id, wts, Gp, Gf, Gy = _panel(23, weighted=weighted)
    run_f, run_s, ym, cm, Ys, Ws = _runs(w_id, f_id, y_id, wts, Gy)
    rows = _run_rows(run_s, ym, cm, Ys, Ws)
    o = np.argsort(run_f, kind="stable")  # firm order, worker order within a firm
    out = _ranges_sum(run_f[o], rows[o], Gf, R)
    ref = np.zeros((Gf, Gy))
    np.add.at(ref, run_f, rows)
    assert not np.isnan(out).any()  # every row written, empty ids included
    assert np.all(out[0::2][: Gf // 2] == 0.0)  # even ids carry no observations
    assert np.abs(out - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_range_partition_one_firm_over_every_range():
    rng = np.random.default_rng(5)
    nr, SG = 1000, 7
    rows = rng.standard_normal((nr, SG))
    sorted_f = np.full(nr, 3)  # one firm owns every run; ids 0-2 and 4-5 are empty
    out = _ranges_sum(sorted_f, rows, 6, 64)
    assert np.all(out[[0, 1, 2, 4, 5]] == 0.0)
    assert np.abs(out[3] - rows.sum(axis=0)).max() <= 1e-11

"""Seeded synthetic AKM worker-firm-year panels (numpy, vectorised).

The reference benchmarks its absorber on proprietary matched employer-employee
panels (README.md:27-45); these generators stand in for them with the same
shapes and value distributions:

* workers observed for T_i = min(1 + Poisson(9), T_max) consecutive years of a
  T_max-year panel, starting at a uniform year that keeps the spell inside it;
* the first firm and every move destination drawn with Zipf(s) probabilities
  over ``n_firms`` firms (rank -> firm id through a seeded permutation, so the
  big firms are scattered over the id range); each worker-year after the first
  moves with probability ``move_prob``;
* worker FE ~ N(0, 1), firm FE ~ N(0, 0.5^2), year FE ~ N(0, 0.1^2), noise N(0, 1).

Workers are drawn until the panel holds exactly ``n_obs`` rows (the last
worker's spell is truncated), so the stated N is exact.  Rows come out in panel
order (worker-major, years ascending), as a matched panel is usually stored.
Group ids are dense 0..G-1 over the levels present.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Panel:
    y: np.ndarray                 # float64 [n]
    X: np.ndarray                 # float64 [n, k], Fortran (column-major) order
    fes: list                     # list of int32 [n] dense group ids
    fe_names: list
    levels: list                  # number of levels per FE dimension
    weights: np.ndarray | None = None
    cluster: np.ndarray | None = None   # worker ids (int32), for clustered SEs
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.y.shape[0])

    @property
    def k(self) -> int:
        return int(self.X.shape[1])


def _zipf_sampler(rng: np.random.Generator, n_firms: int, s: float):
    ranks = np.arange(1, n_firms + 1, dtype=np.float64)
    p = ranks ** (-s)
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    rank_to_id = rng.permutation(n_firms).astype(np.int64)

    def draw(m: int) -> np.ndarray:
        u = rng.random(m)
        r = np.searchsorted(cdf, u, side="right")
        np.minimum(r, n_firms - 1, out=r)
        return rank_to_id[r]

    return draw


def _dense(ids: np.ndarray, n_levels: int) -> tuple[np.ndarray, int]:
    present = np.bincount(ids, minlength=n_levels) > 0
    remap = np.cumsum(present, dtype=np.int64) - 1
    return remap[ids].astype(np.int32), int(present.sum())


def akm_spells(n_obs: int, n_firms: int, n_years: int, *, seed: int,
               move_prob: float = 0.1, zipf: float = 1.1,
               mean_extra_years: float = 9.0):
    """Worker/firm/year ids and within-spell tenure for an AKM panel."""
    rng = np.random.default_rng(seed)
    est = int(n_obs / max(1.0, min(1.0 + mean_extra_years, n_years)) * 1.2) + 16
    T = np.minimum(1 + rng.poisson(mean_extra_years, size=est), n_years)
    while T.sum() < n_obs:
        T = np.concatenate([T, np.minimum(1 + rng.poisson(mean_extra_years, size=est), n_years)])
    cum = np.cumsum(T)
    W = int(np.searchsorted(cum, n_obs, side="left")) + 1
    T = T[:W].copy()
    T[-1] -= int(cum[W - 1] - n_obs)
    starts_w = rng.integers(0, n_years - T + 1)
    offsets = np.zeros(W + 1, dtype=np.int64)
    np.cumsum(T, out=offsets[1:])
    worker = np.repeat(np.arange(W, dtype=np.int64), T)
    pos = np.arange(n_obs, dtype=np.int64) - offsets[worker]
    year = starts_w[worker] + pos

    first = pos == 0
    spell_start = first | (rng.random(n_obs) < move_prob)
    draw = _zipf_sampler(rng, n_firms, zipf)
    cand = np.zeros(n_obs, dtype=np.int64)
    cand[spell_start] = draw(int(spell_start.sum()))
    idx = np.where(spell_start, np.arange(n_obs, dtype=np.int64), 0)
    np.maximum.accumulate(idx, out=idx)
    firm = cand[idx]
    tenure = np.arange(n_obs, dtype=np.int64) - idx
    return rng, worker, firm, year, tenure, pos, W


def akm_two_way(n_obs: int = 1_000_000, *, n_firms: int = 10_000, n_years: int = 10,
                seed: int = 0, move_prob: float = 0.1, zipf: float = 1.1,
                three_way: bool = False) -> Panel:
    """Plain two-way AKM design: y, x1, x2 with worker/firm (and year) FEs.

    x1, x2 = 0.3 * worker FE + sqrt(0.91) * N(0, 1);
    y = 0.5 x1 - 0.3 x2 + worker FE + firm FE + year FE + N(0, 1).
    """
    rng, worker, firm, year, _ten, _pos, W = akm_spells(
        n_obs, n_firms, n_years, seed=seed, move_prob=move_prob, zipf=zipf)
    a = rng.standard_normal(W)
    psi = 0.5 * rng.standard_normal(n_firms)
    gam = 0.1 * rng.standard_normal(n_years)
    aw = a[worker]
    X = np.empty((n_obs, 2), dtype=np.float64, order="F")
    X[:, 0] = 0.3 * aw + np.sqrt(0.91) * rng.standard_normal(n_obs)
    X[:, 1] = 0.3 * aw + np.sqrt(0.91) * rng.standard_normal(n_obs)
    y = 0.5 * X[:, 0] - 0.3 * X[:, 1] + aw + psi[firm] + gam[year] + rng.standard_normal(n_obs)
    w_id, gw = _dense(worker, W)
    f_id, gf = _dense(firm, n_firms)
    t_id, gt = _dense(year, n_years)
    fes, names, levels = [w_id, f_id], ["worker", "firm"], [gw, gf]
    if three_way:
        fes.append(t_id)
        names.append("year")
        levels.append(gt)
    return Panel(y=y, X=X, fes=fes, fe_names=names, levels=levels, cluster=w_id.copy(),
                 meta={"n_workers": W, "seed": seed, "design": "akm_two_way"})


def akm_firm_tenure_slopes(n_obs: int = 1_000_000, *, n_firms: int = 10_000,
                           n_years: int = 10, seed: int = 0, move_prob: float = 0.1,
                           zipf: float = 1.1) -> tuple[Panel, list]:
    """AKM panel with firm-specific tenure slopes (``firm##c.tenure``).

    The heterogeneous firm-seniority design of the reference's hardest
    benchmark spec, on synthetic spells: worker, firm and year FEs, plus a
    slope on tenure (years in the current spell) per firm with the firm
    intercept.  x1, x2 as in ``akm_two_way``;
    y = 0.5 x1 - 0.3 x2 + worker FE + firm FE + firm slope * tenure + year FE + N(0, 1),
    firm slopes ~ N(0.05, 0.02^2).  Returns the panel (fes: worker, firm, year)
    and the slope list [(1, tenure, True)] in the reference's
    HeterogeneousSlopeTerm form (fe_index, values, include_intercept).
    """
    rng, worker, firm, year, ten, _pos, W = akm_spells(
        n_obs, n_firms, n_years, seed=seed, move_prob=move_prob, zipf=zipf)
    a = rng.standard_normal(W)
    psi = 0.5 * rng.standard_normal(n_firms)
    slope = 0.05 + 0.02 * rng.standard_normal(n_firms)
    gam = 0.1 * rng.standard_normal(n_years)
    aw = a[worker]
    tenure = ten.astype(np.float64)
    X = np.empty((n_obs, 2), dtype=np.float64, order="F")
    X[:, 0] = 0.3 * aw + np.sqrt(0.91) * rng.standard_normal(n_obs)
    X[:, 1] = 0.3 * aw + np.sqrt(0.91) * rng.standard_normal(n_obs)
    y = (0.5 * X[:, 0] - 0.3 * X[:, 1] + aw + psi[firm] + slope[firm] * tenure + gam[year]
         + rng.standard_normal(n_obs))
    w_id, gw = _dense(worker, W)
    f_id, gf = _dense(firm, n_firms)
    t_id, gt = _dense(year, n_years)
    panel = Panel(y=y, X=X, fes=[w_id, f_id, t_id], fe_names=["worker", "firm", "year"],
                  levels=[gw, gf, gt], cluster=w_id.copy(),
                  meta={"n_workers": W, "seed": seed, "design": "akm_firm_tenure_slopes"})
    return panel, [(1, tenure, True)]


def group_individual_panel(n_groups: int = 10_000_000, *, n_individuals: int = 2_500_000,
                           n_years: int = 36, n_classes: int = 600, seed: int = 0,
                           zipf: float = 0.8, k: int = 12):
    """Group-level data with individual FEs (patents x inventors style).

    Every group (a row) holds 1-4 distinct individuals drawn with Zipf(s)
    popularity; the rows carry a year and a class FE and k regressors
    (N(0, 1)); y = 0.1 sum(X) + mean of the members' FEs + year + class FE +
    N(0, 1).  Returns (y, X, fes [year, class], edge_group, edge_individual),
    edges group-major with no repeated (group, individual) pair.
    """
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, 5, n_groups)
    eg = np.repeat(np.arange(n_groups, dtype=np.int64), sizes)
    draw = _zipf_sampler(rng, n_individuals, zipf)
    ei = draw(eg.size)
    key = np.unique(eg * n_individuals + ei)  # drop repeats inside a group
    eg, ei = key // n_individuals, key % n_individuals
    alpha = rng.standard_normal(n_individuals)
    cnt = np.bincount(eg, minlength=n_groups)
    if np.any(cnt == 0):
        raise RuntimeError("a group lost all its individuals")
    mean_alpha = np.bincount(eg, weights=alpha[ei], minlength=n_groups) / cnt
    year = rng.integers(0, n_years, n_groups).astype(np.int32)
    cls = rng.integers(0, n_classes, n_groups).astype(np.int32)
    X = np.asfortranarray(rng.standard_normal((n_groups, k)))
    y = (0.1 * X.sum(axis=1) + mean_alpha + 0.1 * rng.standard_normal(n_years)[year]
         + 0.3 * rng.standard_normal(n_classes)[cls] + rng.standard_normal(n_groups))
    return y, X, [year, cls], eg, ei


def akm_batched(n_obs: int = 50_000_000, *, n_firms: int = 800_000, n_years: int = 36,
                seed: int = 0, move_prob: float = 0.1, zipf: float = 1.1,
                n_noise: int = 7) -> Panel:
    """Three-way AKM panel with the outcome plus 12 regressors.

    Columns of X: tenure, tenure^2, age, age^2, age^3, then n_noise N(0, 1)
    controls.  Age is 20..45 at the first observed year plus years since, so it
    lies (up to rounding) in the span of the worker and year FEs.
    """
    rng, worker, firm, year, tenure, pos, W = akm_spells(
        n_obs, n_firms, n_years, seed=seed, move_prob=move_prob, zipf=zipf)
    a = rng.standard_normal(W)
    psi = 0.5 * rng.standard_normal(n_firms)
    gam = 0.1 * rng.standard_normal(n_years)
    age0 = rng.integers(20, 46, size=W).astype(np.float64)
    k = 5 + n_noise
    X = np.empty((n_obs, k), dtype=np.float64, order="F")
    ten = tenure.astype(np.float64)
    X[:, 0] = ten
    np.multiply(ten, ten, out=X[:, 1])
    age = age0[worker] + pos
    X[:, 2] = age
    np.multiply(age, age, out=X[:, 3])
    np.multiply(X[:, 3], age, out=X[:, 4])
    for j in range(n_noise):
        X[:, 5 + j] = rng.standard_normal(n_obs)
    y = a[worker] + psi[firm] + gam[year] + rng.standard_normal(n_obs)
    y += 0.02 * X[:, 0] - 0.0005 * X[:, 1] + 0.01 * X[:, 2]
    for j in range(n_noise):
        y += 0.1 * X[:, 5 + j]
    w_id, gw = _dense(worker, W)
    f_id, gf = _dense(firm, n_firms)
    t_id, gt = _dense(year, n_years)
    return Panel(y=y, X=X, fes=[w_id, f_id, t_id], fe_names=["worker", "firm", "year"],
                 levels=[gw, gf, gt], cluster=w_id.copy(),
                 meta={"n_workers": W, "seed": seed, "design": "akm_batched"})


def drop_singletons(fes: list, max_rounds: int = 1000) -> np.ndarray:
    """Boolean mask of rows kept after iteratively dropping singleton groups.

    Same rule as the reference's pre-absorption singleton drop
    (src/hdfe_regressor_v11.cpp:4056): repeat until no FE dimension has a
    level observed exactly once.
    """
    n = fes[0].shape[0]
    keep = np.ones(n, dtype=bool)
    for _ in range(max_rounds):
        changed = False
        for fe in fes:
            idx = fe[keep]
            cnt = np.bincount(idx)
            single = cnt[idx] == 1
            if single.any():
                kidx = np.flatnonzero(keep)
                keep[kidx[single]] = False
                changed = True
        if not changed:
            break
    return keep


def subset(p: Panel, keep: np.ndarray) -> Panel:
    """Rows ``keep`` of a panel with FE ids re-densified."""
    fes, levels = [], []
    for fe, g in zip(p.fes, p.levels):
        f, gg = _dense(fe[keep].astype(np.int64), g)
        fes.append(f)
        levels.append(gg)
    cl = None
    if p.cluster is not None:
        cl, _ = _dense(p.cluster[keep].astype(np.int64), int(p.cluster.max()) + 1)
    return Panel(y=np.ascontiguousarray(p.y[keep]), X=np.asfortranarray(p.X[keep]),
                 fes=fes, fe_names=list(p.fe_names), levels=levels,
                 weights=None if p.weights is None else p.weights[keep], cluster=cl,
                 meta=dict(p.meta, singletons_dropped=int((~keep).sum())))


def warmstart_panel_spec(i: int, *, seed: int = 4, n_min: int = 100_000,
                         n_max: int = 20_000_000) -> dict:
    """The i-th panel of the learned warm start's workload: N log-uniform in
    [n_min, n_max], 2-4 FE dims (worker, firm, year, firm x year), move
    probability U(0.02, 0.3), firm-size Zipf exponent U(0.8, 1.5), about 62
    observations per firm (the 50M panel's ratio), 36 years."""
    rng = np.random.default_rng([seed, i])
    n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
    return {"n": n, "dims": int(rng.integers(2, 5)), "move_prob": float(rng.uniform(0.02, 0.3)),
            "zipf": float(rng.uniform(0.8, 1.5)), "n_firms": max(200, n // 62), "seed": 10_000 + i}


def warmstart_panel(spec: dict) -> Panel:
    """The panel of ``warmstart_panel_spec`` with singletons dropped; its FE
    list holds the spec's first ``dims`` of (worker, firm, year, firm x year)."""
    p = akm_batched(spec["n"], n_firms=spec["n_firms"], n_years=36, seed=spec["seed"],
                    move_prob=spec["move_prob"], zipf=spec["zipf"])
    fes, names, levels = list(p.fes), list(p.fe_names), list(p.levels)
    if spec["dims"] >= 4:
        fy, g = _dense(p.fes[1].astype(np.int64) * p.levels[2] + p.fes[2], p.levels[1] * p.levels[2])
        fes.append(fy)
        names.append("firm_x_year")
        levels.append(g)
    k = spec["dims"]
    p = Panel(y=p.y, X=p.X, fes=fes[:k], fe_names=names[:k], levels=levels[:k], cluster=p.cluster,
              meta=dict(p.meta, spec=spec))
    return subset(p, drop_singletons(p.fes))

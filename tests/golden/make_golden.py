"""Generate the golden fixtures of tests/golden/ from the reference's own CPU core.

Run in a container where oracle/_ref/libxhdfe_ref.so was built from the
reference sources (oracle/Makefile, target ``ref``):

    python tests/golden/make_golden.py

For each case it stores, in <case>.npz:
  * sha256 digests of the generated inputs (the generators are re-run by the
    tests, which check the digests first);
  * the reference's near-exact within transform (absorb_fixed_effects_v6,
    strict-residual mode, tol 1e-14) on a fixed subset of rows, plus the
    per-column norms of the full transform;
  * the reference's result at tol 1e-8 (reghdfe-comparable): iterations,
    converged, abs_residual_rel;
  * the reference's HdfeRegressorV11::fit coefficients and standard errors.

Slope cases (``python tests/golden/make_golden.py slopes``, slopes_<case>.npz)
hold the reference's absorb_fixed_effects_v6 with heterogeneous slopes at
tol 1e-13 (reghdfe-comparable; strict-residual is refused for slopes): the within transform on all rows (on a row subset
beyond 5000 rows) and its column norms, with the input digests.

Group/individual cases (``python tests/golden/make_golden.py gi``, gi_<case>.npz)
hold the reference's absorb_fixed_effects_group_individual at tol 1e-13 on
structures built from seeded group x individual edge lists.

KSS cases (kss_<case>.npz) hold the inputs of an AKM leave-out decomposition
and the reference's hdfe::akm::akm_kss_decompose results on them:
  * kss_felsdvsimul: the reference's own example data (data/felsdvsimul.dta,
    read from the reference tree; y, worker i, firm j), exact and JLA
    (150 draws, seed 42) leverages; the reference documents these numbers
    (docs/akm-kss.md:19-27) and the fixture records the values its CPU core
    produces here;
  * kss_akm20k: a seeded two-way AKM panel of this repository's generator,
    JLA leverages (200 draws) on the reference's matrix-free PCG path.
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402
import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def case_packed120():
    i = np.arange(120)
    f1 = (i % 20).astype(np.int32)
    f2 = ((i * 7 + i // 20) % 20).astype(np.int32)
    y = 0.7 * np.sin(i / 3) + 0.2 * (f1 - 9.5) + 0.1 * (f2 - 9.5)
    X = np.cos(i / 5)[:, None]
    return dict(y=y, X=X, fes=[f1, f2], weights=None, cluster=None)


def case_soa40():
    i = np.arange(40)
    f1 = (i // 2).astype(np.int32)
    f2 = ((i + 1) // 2).astype(np.int32)
    y = np.sin(i / 3) + 0.2 * f1 - 0.1 * f2
    X = np.cos(i / 5)[:, None]
    return dict(y=y, X=X, fes=[f1, f2], weights=np.ones(40), cluster=None)


def case_validate50k():
    rng = np.random.default_rng(20260605)
    n = 50000
    fe1 = (np.arange(n) % 1000).astype(np.int32)
    fe2 = (np.arange(n) % 97).astype(np.int32)
    x1 = rng.normal(size=n)
    x2 = rng.normal(size=n)
    X = np.column_stack([x1, x2])
    y = 1.25 * x1 - 0.70 * x2 + 0.01 * fe1 - 0.02 * fe2 + rng.normal(scale=0.01, size=n)
    return dict(y=y, X=X, fes=[fe1, fe2], weights=None, cluster=None)


def _akm(n, three_way, seed, weighted=False):
    panels = ge.load_module("panels")
    p = panels.akm_two_way(n, n_firms=2000, n_years=10, seed=seed, three_way=three_way)
    p = panels.subset(p, panels.drop_singletons(p.fes))
    w = None
    if weighted:
        w = np.random.default_rng(seed + 1000).lognormal(0.0, 0.5, size=p.n)
    return dict(y=p.y, X=np.asarray(p.X), fes=p.fes, weights=w, cluster=p.cluster)


CASES = {
    "packed120": case_packed120,
    "soa40": case_soa40,
    "validate50k": case_validate50k,
    "akm2_20k": lambda: _akm(20_000, False, 101),
    "akm3_20k": lambda: _akm(20_000, True, 102),
    "akm3w_20k": lambda: _akm(20_000, True, 103, weighted=True),
}


def subset_rows(n: int) -> np.ndarray:
    step = max(1, n // 400)
    rows = np.unique(np.concatenate([np.arange(0, n, step), np.arange(max(0, n - 5), n)]))
    return rows.astype(np.int64)


def make(name: str) -> dict:
    c = CASES[name]()
    y, X, fes, w, cl = c["y"], np.asarray(c["X"]), c["fes"], c["weights"], c["cluster"]
    n = y.shape[0]
    exact = oracle.ref_absorb(y, X, fes, w, tol=1e-14, tolerance_mode="strict-residual",
                              method="gauss-seidel", threads=1, max_iter=1_000_000)
    comp = oracle.ref_absorb(y, X, fes, w, tol=1e-8, tolerance_mode="reghdfe-comparable",
                             method="auto", threads=1)
    fit = oracle.ref_fit(y, X, fes, w, cl, tol=1e-12, tolerance_mode="strict-residual",
                         threads=1, fit_intercept=False, drop_singletons=False)
    rows = subset_rows(n)
    levels = [int(np.asarray(f).max()) + 1 for f in fes]
    meta = {
        "case": name, "n": n, "k": int(X.shape[1]), "levels": levels,
        "weighted": w is not None, "clustered": cl is not None,
        "exact_iterations": exact["iterations"], "exact_converged": exact["converged"],
        "exact_abs_residual_rel": exact["abs_residual_rel"],
        "comparable_iterations": comp["iterations"], "comparable_converged": comp["converged"],
        "comparable_abs_residual_rel": comp["abs_residual_rel"],
        "comparable_precision_certified": comp["precision_certified"],
        "fit_iterations": fit["iterations"], "fit_nobs": fit["nobs"],
        "input_digest": digest(y, X, *[np.asarray(f, dtype=np.int32) for f in fes],
                               *( [w] if w is not None else [])),
    }
    np.savez_compressed(
        OUT / f"{name}.npz", rows=rows, exact_rows=exact["V"][rows],
        exact_colnorm=np.linalg.norm(exact["V"], axis=0),
        comparable_rows=comp["V"][rows], coef=fit["coef"], se=fit["se"],
        meta=np.array(json.dumps(meta)))
    return meta


REF_DATA = Path(os.environ.get("XHDFE_REFERENCE", "/root/reference")) / "data" / "felsdvsimul.dta"
KSS_KEYS = ("plugin", "agsu", "kss")


def _kss_vec(r) -> np.ndarray:
    return np.array([r[k][c] for k in KSS_KEYS for c in ("var_alpha", "var_psi", "cov_alpha_psi")])


def kss_inputs(name: str):
    if name == "felsdvsimul":
        import pandas as pd
        d = pd.read_stata(REF_DATA)
        return (d["y"].to_numpy(np.float64), d["i"].to_numpy(np.int32), d["j"].to_numpy(np.int32))
    if name == "akm20k":
        p = ge.load_module("panels").akm_two_way(20_000, n_firms=300, n_years=10, seed=11,
                                                  move_prob=0.15)
        return p.y, p.fes[0].astype(np.int32), p.fes[1].astype(np.int32)
    raise KeyError(name)


def make_kss(name: str) -> dict:
    y, w, f = kss_inputs(name)
    runs = {}
    if name == "felsdvsimul":
        runs["exact"] = oracle.ref_akm_kss(y, w, f, leverages="exact", threads=1)
        runs["jla"] = oracle.ref_akm_kss(y, w, f, leverages="jla", jla_draws=150, seed=42, threads=1)
        runs["jla_pcg"] = oracle.ref_akm_kss(y, w, f, leverages="jla", jla_draws=150, seed=42,
                                             direct_max_firms=0, threads=1)
    else:
        runs["jla_pcg"] = oracle.ref_akm_kss(y, w, f, leverages="jla", jla_draws=200, seed=20260705,
                                             direct_max_firms=0, threads=1)
    meta = {k: {"n_obs": r["n_obs"], "n_workers": r["n_workers"], "n_firms": r["n_firms"],
                "n_matches": r["n_matches"], "solver_direct": r["solver_direct"],
                "solver_iterations": r["solver_iterations"]} for k, r in runs.items()}
    np.savez_compressed(OUT / f"kss_{name}.npz", y=y, worker=w, firm=f,
                        **{f"{k}_components": _kss_vec(r) for k, r in runs.items()},
                        **{f"{k}_pii": np.array([r["mean_pii"], r["max_pii"], r["sigma2_ho"]])
                           for k, r in runs.items()},
                        meta=np.array(json.dumps(meta)))
    return meta


KSS_CASES = ("felsdvsimul", "akm20k")


# ---------------------------------------------------------------------------
# Heterogeneous slopes (slopes_<case>.npz): absorb_fixed_effects_v6 with
# HeterogeneousSlopeTerm slopes, (fe_index, values, include_intercept).
# ---------------------------------------------------------------------------
def slope_stata600():
    """The design of the reference's tests/stata/part1/heterogeneous-slopes.do:
    600 rows, firm##c.z and year."""
    i = np.arange(1, 601, dtype=np.float64)
    firm = ((i - 1) % 60).astype(np.int32)
    year = (((i - 1) // 60) % 10).astype(np.int32)
    z = np.mod(i * 17, 23) / 10
    x1, x2 = np.sin(i / 7), np.cos(i / 11)
    y = (1 + .7 * x1 - .3 * x2 + (firm + 1) / 20 + (year + 1) / 9 + .02 * (firm + 1) * z
         + np.sin(i / 13) / 10)
    return dict(y=y, X=np.c_[x1, x2], fes=[firm, year], slopes=[(0, z, True)], weights=None)


def slope_mixed3k(weighted: bool):
    """Seeded 3k rows: a slope without intercept on a dim that also enters as a
    plain FE, and a second slope with intercept on another dim."""
    rng = np.random.default_rng(20260711)
    n = 3000
    g1 = rng.integers(0, 300, n).astype(np.int32)
    g2 = rng.integers(0, 40, n).astype(np.int32)
    z1 = rng.uniform(0, 5, n)
    z2 = rng.standard_normal(n)
    X = rng.standard_normal((n, 3))
    y = X @ np.array([1.0, -2.0, 0.5]) + 0.3 * z1 + rng.standard_normal(n)
    w = rng.uniform(0.5, 2.0, n) if weighted else None
    return dict(y=y, X=X, fes=[g1, g2, g2], slopes=[(0, z1, True), (2, z2, False)], weights=w)


def slope_degenerate2k():
    """Groups whose slope block is singular: z constant within every fifth firm
    (det 0: the intercept alone), z = 0 on a slope-only dim's group."""
    rng = np.random.default_rng(20260712)
    n = 2000
    firm = rng.integers(0, 100, n).astype(np.int32)
    year = rng.integers(0, 12, n).astype(np.int32)
    z = rng.uniform(-1, 1, n)
    z[firm % 5 == 0] = 2.5
    z2 = rng.standard_normal(n)
    z2[year == 3] = 0.0
    X = rng.standard_normal((n, 2))
    y = X @ np.array([0.4, 0.2]) + z + rng.standard_normal(n)
    return dict(y=y, X=X, fes=[firm, year, year], slopes=[(0, z, True), (2, z2, False)],
                weights=None)


def slope_akm20k():
    p, sl = ge.load_module("panels").akm_firm_tenure_slopes(20_000, n_firms=600, seed=20260713)
    return dict(y=p.y, X=p.X, fes=p.fes, slopes=sl, weights=None)


SLOPE_CASES = {
    "stata600": slope_stata600,
    "mixed3k": lambda: slope_mixed3k(False),
    "mixed3kw": lambda: slope_mixed3k(True),
    "degenerate2k": slope_degenerate2k,
    "akm20k": slope_akm20k,
}


def slope_digest(c) -> str:
    arrs = [c["y"], np.asarray(c["X"], dtype=np.float64),
            *[np.asarray(f, dtype=np.int32) for f in c["fes"]],
            *[np.asarray(z, dtype=np.float64) for _, z, _ in c["slopes"]]]
    if c["weights"] is not None:
        arrs.append(c["weights"])
    return digest(*arrs)


def make_slopes(name: str) -> dict:
    c = SLOPE_CASES[name]()
    ref = oracle.ref_absorb_slopes(c["y"], c["X"], c["fes"], c["slopes"], c["weights"],
                                   tol=1e-13, tolerance_mode="reghdfe-comparable", threads=1,
                                   max_iter=1_000_000)
    n = c["y"].shape[0]
    rows = subset_rows(n) if n > 5000 else np.arange(n, dtype=np.int64)
    meta = {"case": name, "n": n, "iterations": ref["iterations"],
            "converged": ref["converged"], "abs_residual_rel": ref["abs_residual_rel"],
            "slopes": [[d, bool(i)] for d, _, i in c["slopes"]],
            "input_digest": slope_digest(c)}
    np.savez_compressed(OUT / f"slopes_{name}.npz", rows=rows, ref_rows=ref["V"][rows],
                        ref_colnorm=np.linalg.norm(ref["V"], axis=0), meta=np.array(json.dumps(meta)))
    return meta


# ---------------------------------------------------------------------------
# Group/individual FEs (gi_<case>.npz): absorb_fixed_effects_group_individual
# on structures built from seeded edge lists (patent x inventor style: groups
# of 1-4 individuals), standard FEs on the group rows.
# ---------------------------------------------------------------------------
def gi_edges(n_groups, n_individuals, seed, max_size=4):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, max_size + 1, n_groups)
    eg = np.repeat(np.arange(n_groups), sizes)
    # popular individuals: Zipf-like draws, no repeat inside a group
    p = 1.0 / np.arange(1, n_individuals + 1) ** 0.8
    p /= p.sum()
    ei = np.concatenate([rng.choice(n_individuals, s, replace=False, p=p) for s in sizes])
    return rng, eg, ei


def gi_case(n_groups, n_individuals, seed, aggregation, n_fes, weighted):
    rng, eg, ei = gi_edges(n_groups, n_individuals, seed)
    gi, _, _ = ge.load_package().build_group_individual(eg * 7 + 3, ei + 1000, aggregation)
    n = gi.num_groups
    fes = []
    if n_fes >= 1:
        fes.append(rng.integers(0, 15, n).astype(np.int32))
    if n_fes >= 2:
        fes.append(rng.integers(0, max(2, n // 20), n).astype(np.int32))
    X = rng.standard_normal((n, 3))
    y = X @ np.array([0.7, -0.2, 0.1]) + rng.standard_normal(n)
    w = rng.uniform(0.5, 2.0, n) if weighted else None
    return dict(y=y, X=X, fes=fes, gi=gi, weights=w, edges=(eg, ei), aggregation=aggregation)


GI_CASES = {
    "mean1500": lambda: gi_case(1500, 400, 20260721, "mean", 1, False),
    "sum1500w": lambda: gi_case(1500, 400, 20260722, "sum", 1, True),
    "nofe1200": lambda: gi_case(1200, 300, 20260723, "mean", 0, False),
    "mean20k": lambda: gi_case(20_000, 5_000, 20260724, "mean", 2, False),
}


def gi_digest(c) -> str:
    gi = c["gi"]
    arrs = [c["y"], np.asarray(c["X"], dtype=np.float64),
            *[np.asarray(f, dtype=np.int32) for f in c["fes"]],
            np.asarray(gi.group_ptr, dtype=np.int32), np.asarray(gi.group_individual, dtype=np.int32),
            np.asarray(gi.individual_ptr, dtype=np.int32),
            np.asarray(gi.individual_group, dtype=np.int32), np.asarray(gi.group_scale)]
    if c["weights"] is not None:
        arrs.append(c["weights"])
    return digest(*arrs)


def make_gi(name: str) -> dict:
    c = GI_CASES[name]()
    ref = oracle.ref_absorb_gi(c["y"], c["X"], c["fes"], c["gi"], c["weights"], tol=1e-13,
                               threads=1, max_iter=1_000_000)
    n = c["y"].shape[0]
    rows = subset_rows(n) if n > 5000 else np.arange(n, dtype=np.int64)
    meta = {"case": name, "n": n, "num_individuals": int(c["gi"].num_individuals),
            "num_edges": int(len(c["gi"].group_individual)), "iterations": ref["iterations"],
            "converged": ref["converged"], "abs_residual_rel": ref["abs_residual_rel"],
            "input_digest": gi_digest(c)}
    np.savez_compressed(OUT / f"gi_{name}.npz", rows=rows, ref_rows=ref["V"][rows],
                        ref_colnorm=np.linalg.norm(ref["V"], axis=0), meta=np.array(json.dumps(meta)))
    return meta


if __name__ == "__main__":
    if sys.argv[1:2] == ["gi"]:
        for nm in sys.argv[2:] or list(GI_CASES):
            print(nm, json.dumps(make_gi(nm)))
        sys.exit(0)
    if sys.argv[1:2] == ["slopes"]:
        for nm in sys.argv[2:] or list(SLOPE_CASES):
            print(nm, json.dumps(make_slopes(nm)))
        sys.exit(0)
    if sys.argv[1:2] == ["kss"]:
        for nm in sys.argv[2:] or KSS_CASES:
            print(nm, json.dumps(make_kss(nm)))
        sys.exit(0)
    names = sys.argv[1:] or list(CASES)
    for nm in names:
        m = make(nm)
        print(json.dumps({k: m[k] for k in ("case", "n", "exact_iterations",
                                            "exact_abs_residual_rel",
                                            "comparable_iterations")}))

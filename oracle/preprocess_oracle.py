"""ORACLE -- test infrastructure only: numpy restatement of the reference's
host preprocessing, the checker of the device versions.

build_indexer restates src/fe_absorption.cpp:845-940: with R = max - min + 1,
if R <= 50,000,000 and R <= 2n the ids are raw - min (num_groups = R), compacted
in raw order when fewer than 90% of the range is present (num_groups = distinct
values); otherwise the rank of the raw value among the distinct values.

singleton_keep restates compute_keep_mask_drop_singletons
(src/hdfe_regressor_v11.cpp:4056-4290): rounds dropping every kept row that is
alone in its group of some dimension, until a round drops nothing (at most
max_iter rounds, 100 in the reference).

component_stats restates compute_first_pair_component_stats
(src/hdfe_regressor_v11.cpp:7192-7270): connected components of the bipartite
graph of the two dims' groups, components with observations, the largest one's
observation count and share, and its weight share.

Only tests/ import this module, and only as the checker.
"""

from __future__ import annotations

import numpy as np


def build_indexer(raw):
    raw = np.asarray(raw, dtype=np.int64)
    n = raw.size
    lo, hi = int(raw.min()), int(raw.max())
    rng = hi - lo + 1
    if 0 < rng <= 50_000_000 and rng <= 2 * n:
        mapped = raw - lo
        seen = np.zeros(rng, dtype=bool)
        seen[mapped] = True
        unique = int(seen.sum())
        if unique * 10 < rng * 9:
            remap = np.cumsum(seen) - 1
            return remap[mapped].astype(np.int32), unique, unique
        return mapped.astype(np.int32), rng, unique
    vals, inv = np.unique(raw, return_inverse=True)
    return inv.astype(np.int32), vals.size, vals.size


def singleton_keep(ids, max_iter=100):
    ids = [np.asarray(g, dtype=np.int64) for g in ids]
    n = ids[0].size
    keep = np.ones(n, dtype=bool)
    rounds = 0
    for rounds in range(1, max_iter + 1):
        single = np.zeros(n, dtype=bool)
        for g in ids:
            cnt = np.bincount(g[keep], minlength=int(g.max()) + 1)
            single |= keep & (cnt[g] == 1)
        if not single.any():
            return keep, rounds - 1
        keep &= ~single
    return keep, rounds


def component_stats(fe1, fe2, weights=None):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    g1, G1, _ = build_indexer(fe1)
    g2, G2, _ = build_indexer(fe2)
    n = g1.size
    adj = coo_matrix((np.ones(n), (g1, G1 + g2)), shape=(G1 + G2, G1 + G2))
    _, lab = connected_components(adj, directed=False)
    comp = lab[g1]
    counts = np.bincount(comp)
    big = int(counts.max())
    out = {"num_components": int((counts > 0).sum()), "largest_component_n_obs": big,
           "largest_component_obs_share": big / n}
    if weights is None:
        out["largest_component_weight_share"] = big / n
    else:
        ws = np.bincount(comp, weights=np.asarray(weights, dtype=np.float64))
        out["largest_component_weight_share"] = float(ws.max() / ws.sum())
    return out

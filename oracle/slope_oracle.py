"""ORACLE -- test infrastructure only.

Exact weighted projection for absorption with heterogeneous slopes, a numpy
restatement of what the reference's slope absorbers converge to
(absorb_fixed_effects_v6 with HeterogeneousSlopeTerm slopes,
src/fe_absorption.cpp:8300-8330 and the per-group slope projection of
compute_slope_coefficients_kernel, src/fe_absorption_cuda.cu:586-650):

* dimension d spans, per group g, 1_g for a plain FE; z 1_g for a slope
  without intercept; 1_g and z 1_g for a slope with intercept;
* a group keeps its intercept alone when its 2x2 block [W Z; Z ZZ] has
  det <= 1e-12 max(1, W ZZ), and drops its slope column when
  ZZ <= 1e-12 max(1, ZZ) without intercept (the reference's rule);
* group/individual designs (absorb_fixed_effects_group_individual,
  src/fe_absorption.cpp:9741; GroupIndividualStructure,
  include/fe_absorption.hpp:13-21): rows are groups and the basis column of
  individual i is group_scale[g] at every group g that holds i;
* the within transform is v - D a with a the minimum-norm weighted
  least-squares solution (dense, so for small cases only).

Only tests/ import this module.
"""

from __future__ import annotations

import numpy as np

DET_TOL = 1e-12


def slope_basis(fes, slopes, weights, n):
    """Dense basis D [n, m] of every FE block, after the reference's rule."""
    w = np.ones(n) if weights is None else np.asarray(weights, dtype=np.float64)
    kind = {d: (np.asarray(z, dtype=np.float64), bool(icpt)) for d, z, icpt in slopes}
    cols = []
    for d, f in enumerate(fes):
        f = np.asarray(f, dtype=np.int64)
        G = int(f.max()) + 1 if f.size else 0
        if d not in kind:
            for g in range(G):
                c = (f == g).astype(np.float64)
                if c.any():
                    cols.append(c)
            continue
        z, icpt = kind[d]
        W = np.bincount(f, weights=w, minlength=G)
        Z = np.bincount(f, weights=w * z, minlength=G)
        ZZ = np.bincount(f, weights=w * z * z, minlength=G)
        for g in range(G):
            m = f == g
            if not m.any():
                continue
            if icpt:
                cols.append(m.astype(np.float64))
                det = W[g] * ZZ[g] - Z[g] * Z[g]
                if W[g] > 0 and det > DET_TOL * max(1.0, W[g] * ZZ[g]):
                    cols.append(np.where(m, z, 0.0))
            else:
                if ZZ[g] > DET_TOL * max(1.0, ZZ[g]):
                    cols.append(np.where(m, z, 0.0))
    return np.stack(cols, axis=1) if cols else np.zeros((n, 0))


def slope_projection(V, fes, slopes, weights=None):
    """Within transform of every column of V [n, C] (exact, min-norm LS)."""
    V = np.asarray(V, dtype=np.float64)
    n = V.shape[0]
    D = slope_basis(fes, slopes, weights, n)
    sw = np.ones(n) if weights is None else np.sqrt(np.asarray(weights, dtype=np.float64))
    A = D * sw[:, None]
    B = V * sw[:, None]
    a, *_ = np.linalg.lstsq(A, B, rcond=None)
    return V - D @ a


def gi_projection(V, fes, gi, weights=None):
    """Within transform on the standard FEs plus the individual FEs of a
    group/individual structure (exact, min-norm LS)."""
    V = np.asarray(V, dtype=np.float64)
    n = V.shape[0]
    Ds = slope_basis(fes, [], weights, n)
    Di = np.zeros((n, int(gi.num_individuals)))
    gp = np.asarray(gi.group_ptr)
    for g in range(n):
        for e in range(gp[g], gp[g + 1]):
            Di[g, gi.group_individual[e]] = gi.group_scale[g]
    D = np.hstack([Ds, Di[:, np.any(Di != 0, axis=0)]])
    sw = np.ones(n) if weights is None else np.sqrt(np.asarray(weights, dtype=np.float64))
    a, *_ = np.linalg.lstsq(D * sw[:, None], V * sw[:, None], rcond=None)
    return V - D @ a

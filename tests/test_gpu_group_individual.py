"""Group/individual FEs on the B200 (b200fe_absorb_group_individual).

Parity: the within transform against the reference's
absorb_fixed_effects_group_individual (golden vectors, tol 1e-13) and the
oracle's exact projection at REL_TOL of each column's norm; determinism;
invariance to the order of the group rows; structure validation; and the
reference's own absorb_fixed_effects_group_individual running on this library
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


def _absorb(absorber, pkg, c, tol=1e-10):
    G = [int(np.max(f)) + 1 for f in c["fes"]]
    return absorber.absorb_group_individual(c["y"], c["X"], c["fes"], G, c["gi"], c["weights"],
                                            pkg.make_options(tol=tol))


@pytest.mark.parametrize("name", sorted(make_golden.GI_CASES))
def test_gi_matches_reference_golden(absorber, pkg, name):
    d = np.load(GOLDEN / f"gi_{name}.npz")
    meta = json.loads(str(d["meta"]))
    c = make_golden.GI_CASES[name]()
    assert make_golden.gi_digest(c) == meta["input_digest"]
    r = _absorb(absorber, pkg, c)
    assert r.converged and r.precision_certified
    V = np.column_stack([r.y_tilde, r.X_tilde])
    err = np.abs(V[d["rows"]] - d["ref_rows"]).max(axis=0) / d["ref_colnorm"]
    assert err.max() <= REL_TOL
    assert r.fe_levels[-1] == c["gi"].num_individuals


@pytest.mark.parametrize("name", ["mean1500", "sum1500w", "nofe1200"])
def test_gi_matches_exact_projection(absorber, pkg, name):
    from oracle.slope_oracle import gi_projection
    c = make_golden.GI_CASES[name]()
    r = _absorb(absorber, pkg, c, tol=1e-12)
    V = np.column_stack([r.y_tilde, r.X_tilde])
    V0 = np.column_stack([c["y"], c["X"]])
    o = gi_projection(V0, c["fes"], c["gi"], c["weights"])
    assert (np.linalg.norm(V - o, axis=0) / np.linalg.norm(V0, axis=0)).max() <= REL_TOL * 1e-1


def test_gi_deterministic_and_row_order_invariant(absorber, pkg):
    c = make_golden.GI_CASES["mean20k"]()
    a = _absorb(absorber, pkg, c)
    b = _absorb(absorber, pkg, c)
    assert np.array_equal(a.y_tilde, b.y_tilde) and np.array_equal(a.X_tilde, b.X_tilde)
    # relabel the groups in a random order: same structure, rows permuted
    rng = np.random.default_rng(2)
    eg, ei = c["edges"]
    relabel = rng.permutation(c["gi"].num_groups)
    gi2, _, _ = pkg.build_group_individual(relabel[eg], ei, c["aggregation"])
    inv = np.argsort(relabel)  # new row r holds old group inv[r]
    c2 = dict(y=c["y"][inv], X=c["X"][inv], fes=[f[inv] for f in c["fes"]], gi=gi2, weights=None)
    r2 = _absorb(absorber, pkg, c2)
    V1 = np.column_stack([a.y_tilde, a.X_tilde])[inv]
    V2 = np.column_stack([r2.y_tilde, r2.X_tilde])
    assert (np.linalg.norm(V1 - V2, axis=0) / np.linalg.norm(V1, axis=0)).max() <= 1e-8


def test_gi_structure_validation(absorber, pkg):
    c = make_golden.GI_CASES["nofe1200"]()
    gi = c["gi"]
    bad = pkg.GroupIndividualStructure(gi.num_groups, gi.num_individuals, gi.group_ptr.copy(),
                                       gi.group_individual.copy(), gi.individual_ptr.copy(),
                                       gi.individual_group.copy(), gi.group_scale.copy())
    bad.group_individual[3] = gi.num_individuals  # out of range
    with pytest.raises(pkg.AbsorberError):
        absorber.absorb_group_individual(c["y"], c["X"], [], [], bad, None, pkg.make_options())
    bad2 = pkg.GroupIndividualStructure(gi.num_groups, gi.num_individuals, gi.group_ptr.copy(),
                                        gi.group_individual, gi.individual_ptr, gi.individual_group,
                                        gi.group_scale)
    bad2.group_ptr[-1] += 1  # does not end at the edge count
    with pytest.raises(pkg.AbsorberError):
        absorber.absorb_group_individual(c["y"], c["X"], [], [], bad2, None, pkg.make_options())


def test_reference_gi_dispatches_to_b200(oracle_mod):
    if not oracle_mod.REF_B200_SO.exists():
        pytest.skip("oracle/_ref/libxhdfe_ref_b200.so not built (needs the reference sources)")
    c = make_golden.GI_CASES["sum1500w"]()
    g = oracle_mod.ref_absorb_gi(c["y"], c["X"], c["fes"], c["gi"], c["weights"], tol=1e-10,
                                 gpu_backend="cuda", lib_path=oracle_mod.REF_B200_SO)
    assert g["gpu_status_code"] == 1 and g["converged"]
    d = np.load(GOLDEN / "gi_sum1500w.npz")
    err = np.abs(g["V"][d["rows"]] - d["ref_rows"]).max(axis=0) / d["ref_colnorm"]
    assert err.max() <= REL_TOL


def test_gi_edge_cases(absorber, pkg):
    """An individual in no group, single-individual groups, zero weights,
    sum aggregation without standard FEs."""
    from oracle.slope_oracle import gi_projection
    rng = np.random.default_rng(4)
    ng = 400
    sizes = rng.integers(1, 4, ng)
    eg = np.repeat(np.arange(ng), sizes)
    ei = np.concatenate([rng.choice(60, s, replace=False) for s in sizes])
    gi, _, _ = pkg.build_group_individual(eg, ei, "sum")
    # append an individual that no group holds
    gi = pkg.GroupIndividualStructure(gi.num_groups, gi.num_individuals + 1, gi.group_ptr,
                                      gi.group_individual,
                                      np.append(gi.individual_ptr, gi.individual_ptr[-1]),
                                      gi.individual_group, gi.group_scale)
    n = gi.num_groups
    X = rng.standard_normal((n, 2))
    y = rng.standard_normal(n)
    w = rng.uniform(0.5, 2.0, n)
    w[::13] = 0.0
    r = absorber.absorb_group_individual(y, X, [], [], gi, w, pkg.make_options(tol=1e-12))
    V0 = np.column_stack([y, X])
    o = gi_projection(V0, [], gi, w)
    V = np.column_stack([r.y_tilde, r.X_tilde])
    assert r.converged
    assert (np.linalg.norm(V - o, axis=0) / np.linalg.norm(V0, axis=0)).max() <= 1e-9

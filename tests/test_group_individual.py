"""Group/individual FEs on the CPU: the package's structure builder (the
reference's rules, src/hdfe_regressor_v11.cpp:5780-5920), the oracle's exact
projection (oracle/slope_oracle.py: gi_projection) pinned against the golden
vectors of the reference's absorb_fixed_effects_group_individual
(tests/golden/gi_*.npz), and the fixture generators.
"""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_golden  # noqa: E402

ORACLE_TOL = 1e-10


def load(name):
    d = np.load(GOLDEN / f"gi_{name}.npz")
    return d, json.loads(str(d["meta"]))


@pytest.mark.parametrize("name", sorted(make_golden.GI_CASES))
def test_generator_reproduces_gi_inputs(name):
    _, meta = load(name)
    assert make_golden.gi_digest(make_golden.GI_CASES[name]()) == meta["input_digest"]


@pytest.mark.parametrize("name", sorted(make_golden.GI_CASES))
def test_gi_oracle_matches_reference(name):
    from oracle.slope_oracle import gi_projection
    d, meta = load(name)
    if meta["n"] > 5000:
        pytest.skip("dense oracle: small cases only")
    c = make_golden.GI_CASES[name]()
    o = gi_projection(np.column_stack([c["y"], c["X"]]), c["fes"], c["gi"], c["weights"])
    err = np.abs(o[d["rows"]] - d["ref_rows"]).max(axis=0) / d["ref_colnorm"]
    assert err.max() <= ORACLE_TOL


def test_builder_structure(pkg):
    gi, gv, iv = pkg.build_group_individual(np.array([30, 30, 50, 50, 50, 90]),
                                            np.array([1, 2, 1, 7, 2, 7]), "mean")
    assert list(gv) == [30, 50, 90] and list(iv) == [1, 2, 7]
    assert list(gi.group_ptr) == [0, 2, 5, 6]
    assert list(gi.group_individual) == [0, 1, 0, 1, 2, 2]
    assert list(gi.individual_ptr) == [0, 2, 4, 6]
    assert list(gi.individual_group) == [0, 1, 0, 1, 1, 2]
    assert np.allclose(gi.group_scale, [0.5, 1 / 3, 1.0])
    gs, _, _ = pkg.build_group_individual(np.array([1, 1, 2]), np.array([4, 5, 4]), "sum")
    assert np.all(gs.group_scale == 1.0)
    with pytest.raises(ValueError, match="uniquely identify"):
        pkg.build_group_individual(np.array([1, 1]), np.array([4, 4]))


def test_builder_csr_consistent():
    c = make_golden.GI_CASES["mean20k"]()
    gi = c["gi"]
    eg, ei = [], []
    for g in range(gi.num_groups):
        for e in range(gi.group_ptr[g], gi.group_ptr[g + 1]):
            eg.append(g)
            ei.append(gi.group_individual[e])
    a = sorted(zip(eg, ei))
    b = sorted((int(gi.individual_group[e]), i) for i in range(gi.num_individuals)
               for e in range(gi.individual_ptr[i], gi.individual_ptr[i + 1]))
    assert a == b

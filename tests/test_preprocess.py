"""CPU checks of the preprocessing oracle (oracle/preprocess_oracle.py): the
restatement of the reference's build_indexer on hand-computed cases of its
three branches, and its singleton cascade against the package's host mask
(both reach the unique fixed point of the rule); partial_out's argument checks,
which run before any device work."""

import numpy as np
import pytest


def test_build_indexer_branches():
    from oracle.preprocess_oracle import build_indexer
    # dense range, >= 90% present: ids = raw - min, num_groups = range (a gap kept)
    raw = np.array([5, 7, 6, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 5])
    ids, G, present = build_indexer(raw)
    assert G == 20 and present == 20 and ids.tolist() == (raw - 5).tolist()
    raw = np.concatenate([np.arange(100, 110), np.arange(111, 200)])  # one gap in 100
    ids, G, present = build_indexer(raw)
    assert G == 100 and present == 99 and ids[10] == 11
    # dense range, < 90% present: compacted in raw order
    raw = np.array([-3, 10, 4, 10, -3, 7])
    ids, G, present = build_indexer(raw)
    assert (G, present) == (4, 4) and ids.tolist() == [0, 3, 1, 3, 0, 2]
    # sparse range: ranks of the distinct values
    raw = np.array([2_000_000_000, -7, 15, -7, 2_000_000_000])
    ids, G, present = build_indexer(raw)
    assert (G, present) == (3, 3) and ids.tolist() == [2, 0, 1, 0, 2]


def test_singleton_oracle_matches_host_mask(pkg, panels):
    from oracle.preprocess_oracle import singleton_keep
    p = panels.akm_two_way(30_000, n_firms=2_000, seed=91, three_way=True)
    keep, rounds = singleton_keep(p.fes)
    assert rounds >= 1 and not keep.all()
    assert np.array_equal(keep, pkg.drop_singletons_mask(p.fes))


def test_component_oracle_matches_reference(oracle_mod, panels):
    from oracle.preprocess_oracle import component_stats
    if not oracle_mod.ref_available():
        import pytest
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    p = panels.akm_two_way(20_000, n_firms=2_000, seed=7, move_prob=0.02)
    w = np.random.default_rng(2).lognormal(0.0, 0.5, size=p.n)
    for ww in (None, w):
        ref = oracle_mod.ref_components(p.fes[0], p.fes[1], ww)
        ours = component_stats(p.fes[0], p.fes[1], ww)
        assert ref["num_components"] == ours["num_components"] > 1
        assert ref["largest_component_n_obs"] == ours["largest_component_n_obs"]
        assert abs(ref["largest_component_weight_share"] - ours["largest_component_weight_share"]) <= 1e-12


def test_partial_out_argument_checks(pkg):
    """partial_out rejects what HdfeRegressorV11::partial_out rejects before any
    device work: an empty outcome, non-finite data, X of another length,
    negative or non-finite weights."""
    f = [np.array([0, 0, 1, 1], dtype=np.int32)]
    y = np.array([1.0, 2.0, 3.0, 4.0])
    with pytest.raises(ValueError):
        pkg.partial_out(np.zeros(0), None, f)
    with pytest.raises(ValueError):
        pkg.partial_out(np.array([1.0, np.nan, 3.0, 4.0]), None, f)
    with pytest.raises(ValueError):
        pkg.partial_out(y, np.array([[1.0], [np.inf], [0.0], [2.0]]), f)
    with pytest.raises(ValueError):
        pkg.partial_out(y, np.ones((3, 1)), f)
    with pytest.raises(ValueError):
        pkg.partial_out(y, None, f, weights=np.array([1.0, -1.0, 1.0, 1.0]))
    with pytest.raises(ValueError):
        pkg.partial_out(y, None, f, weights=np.ones(3))

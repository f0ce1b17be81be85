"""Preprocessing on the device against the oracle restatement of the
reference's host code (bit-exact ids and counts) and against the reference
itself: the rows its own partial_out keeps after the singleton cascade."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["dense_full", "dense_sparse", "sparse", "negative", "zipf_5m"])
def test_dense_ids_match_build_indexer(pkg, case):
    from oracle.preprocess_oracle import build_indexer
    rng = np.random.default_rng(17)
    if case == "dense_full":
        raw = rng.integers(1000, 2000, size=50_000)
    elif case == "dense_sparse":
        raw = rng.choice(np.arange(0, 100_000, 3), size=60_000)
    elif case == "sparse":
        raw = rng.integers(-2**31, 2**31 - 1, size=40_000)
    elif case == "negative":
        raw = rng.integers(-500, 500, size=30_000)
    else:
        p = 1.0 / np.arange(1, 800_001) ** 1.1
        raw = rng.choice(800_000, size=5_000_000, p=p / p.sum()) * 7 + 11
    raw = raw.astype(np.int32)
    ids, G, present = pkg.dense_ids_device(raw)
    ref_ids, ref_G, ref_present = build_indexer(raw)
    assert (G, present) == (ref_G, ref_present)
    assert np.array_equal(ids.cpu().numpy(), ref_ids)


def test_singletons_match_oracle_and_reference(pkg, panels, oracle_mod):
    import torch
    from oracle.preprocess_oracle import singleton_keep
    p = panels.akm_two_way(60_000, n_firms=3_000, seed=93, three_way=True)
    ids = [torch.from_numpy(np.ascontiguousarray(f, dtype=np.int32)).cuda() for f in p.fes]
    keep, dropped, rounds = pkg.drop_singletons_device(ids, p.levels)
    ref_keep, ref_rounds = singleton_keep(p.fes)
    assert np.array_equal(keep.cpu().numpy(), ref_keep)
    assert dropped == int((~ref_keep).sum()) and rounds == ref_rounds
    if oracle_mod.ref_available():
        r = oracle_mod.ref_partial_out(p.y, p.X, p.fes, tol=1e-8)
        assert np.array_equal(np.flatnonzero(keep.cpu().numpy()), np.sort(r["sample_index"]))


def test_partial_out_uses_device_preprocessing(pkg, panels, oracle_mod):
    p = panels.akm_two_way(40_000, n_firms=1_500, seed=95, three_way=True)
    raw = [np.asarray(f) * 13 + 1000 for f in p.fes]  # raw, non-dense ids
    res = pkg.partial_out(p.y, p.X, raw, tol=1e-10)
    keep = pkg.drop_singletons_mask(p.fes)
    assert np.array_equal(res.sample_index, np.flatnonzero(keep))
    ref, _, ok = oracle_mod.project(p.y[keep], p.X[keep], [np.asarray(f)[keep] for f in p.fes],
                                    [int(g) for g in p.levels], tol=1e-13)
    V = np.column_stack([p.y[keep], p.X[keep]])
    out = np.column_stack([res.y_tilde, res.X_tilde])
    err = np.linalg.norm(out - ref, axis=0) / np.linalg.norm(V, axis=0)
    assert err.max() <= 1e-8


@pytest.mark.parametrize("case", ["akm_low_mobility", "akm_50k_weighted", "raw_sparse_ids"])
def test_first_pair_components_match_reference(pkg, panels, oracle_mod, case):
    from oracle.preprocess_oracle import component_stats
    rng = np.random.default_rng(23)
    p = panels.akm_two_way(50_000, n_firms=4_000, seed=97, move_prob=0.02)
    f1, f2 = np.asarray(p.fes[0]), np.asarray(p.fes[1])
    w = rng.lognormal(0.0, 0.5, size=p.n) if case == "akm_50k_weighted" else None
    if case == "raw_sparse_ids":
        f1 = (f1.astype(np.int64) * 40_503 - 1_000_000_000).astype(np.int32)
        f2 = (f2.astype(np.int64) * 7 + 3).astype(np.int32)
    ours = pkg.first_pair_component_stats(f1, f2, w)
    want = (oracle_mod.ref_components(f1, f2, w) if oracle_mod.ref_available()
            else component_stats(f1, f2, w))
    assert ours.num_components == want["num_components"] > 1
    assert ours.largest_component_n_obs == want["largest_component_n_obs"]
    assert ours.largest_component_obs_share == pytest.approx(want["largest_component_obs_share"], abs=1e-15)
    assert ours.largest_component_weight_share == pytest.approx(
        want["largest_component_weight_share"], abs=1e-12)

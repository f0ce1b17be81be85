"""CPU checks of the JLA leverages' checker.

The numpy restatement of the reference's JLA draw loop (oracle/kss_oracle.py:
jla_leverages; src/akm_kss.cpp:2753-3160 and :3275-3289) run on the working
rows of the reference's own decomposition reproduces that decomposition's
per-row leverages (AkmKssResult::pii) with the same seed and draw count: the
SplitMix64 streams, the scatters and the accumulation order are the
reference's, so the two agree to rounding (1e-10 here).  Also the restated
streams against SplitMix64 values computed independently in Python ints.
"""

import numpy as np
import pytest


def _ref_or_skip(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")


def _splitmix64_int(x):
    m = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & m
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    return x ^ (x >> 31)


def test_streams_match_python_int_splitmix64():
    from oracle import kss_oracle as ko
    m = (1 << 64) - 1
    for seed, tag in ((20260705, 0), (7, 5), (2**63 + 11, 3)):
        s = _splitmix64_int(seed ^ ((0xA24BAED4963EE407 * (tag + 1)) & m))
        want = [_splitmix64_int(s ^ ((0x9FB21C651E98DF25 * (u + 1)) & m)) for u in range(5)]
        got = ko.stream_seed(seed, tag, np.arange(5))
        assert [int(v) for v in got] == want


@pytest.mark.parametrize("seed,draws,n,firms", [(123, 20, 20_000, 200), (20260705, 7, 30_000, 300)])
def test_restated_jla_reproduces_reference_leverages(oracle_mod, panels, seed, draws, n, firms):
    _ref_or_skip(oracle_mod)
    from oracle import kss_oracle as ko
    p = panels.akm_two_way(n, n_firms=firms, seed=seed % 1000)
    r = oracle_mod.ref_akm_kss_rows(p.y, p.fes[0], p.fes[1], leverages="jla", jla_draws=draws, seed=seed)
    st = ko.match_system_from_rows(r["row_worker"], r["row_firm"], r["row_weight"])
    o = ko.jla_leverages(st, seed, draws)
    assert np.abs(o["pii"] - r["pii"]).max() <= 1e-10

"""The device JLA leverages (b200fe_kss_jla) against the reference's own
decomposition and the numpy restatement of its draw loop.

Workload: seeded AKM panels; the reference's akm_kss_decompose (CPU core,
JLA with the given seed and draws) returns its working rows (matches) in its
order with their leverages; the match system of those rows in that order
goes to the device, whose streams are then the reference's.  Bar: pii within
1e-9 of the reference's, and pii, mii, corr, bfe, bpe, bcov within 1e-9 of
the restatement (solved exactly), relative to each output's largest entry,
for draw blocks of 1, 8 and 21 (lane pitches 4, 32, 64) and a single draw.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _case(oracle_mod, panels, seed, draws, n, firms):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    from oracle import kss_oracle as ko
    p = panels.akm_two_way(n, n_firms=firms, seed=seed % 1000)
    r = oracle_mod.ref_akm_kss_rows(p.y, p.fes[0], p.fes[1], leverages="jla", jla_draws=draws, seed=seed)
    st = ko.match_system_from_rows(r["row_worker"], r["row_firm"], r["row_weight"])
    return r, st, ko


def _device(pkg, st, seed, draws, block):
    system = pkg.kss_system(st["m_w"], st["m_f"], st["m_c"], st["N"], st["J"])
    solver = pkg.KssSolver(system)
    try:
        return solver.jla(st["m_w"], st["m_f"], st["m_c"].astype(np.int64), float(st["m_c"].sum()),
                          row_sw=np.sqrt(st["m_c"]), seed=seed, draws=draws, block=block, tol=1e-12,
                          max_iter=5000)
    finally:
        solver.close()


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("block", [8, 1, 21])
def test_device_jla_matches_reference_and_restatement(pkg, oracle_mod, panels, block):
    seed, draws = 123, 20
    r, st, ko = _case(oracle_mod, panels, seed, draws, 20_000, 200)
    d = _device(pkg, st, seed, draws, block)
    assert d["failed_lanes"] == 0 and d["iterations"] > 0
    assert _rel(d["pii"], r["pii"]) <= TOL
    o = ko.jla_leverages(st, seed, draws)
    for k in ("pii", "mii", "corr", "bfe", "bpe", "bcov"):
        assert _rel(d[k], o[k]) <= TOL, k


def test_device_jla_single_draw_and_other_seed(pkg, oracle_mod, panels):
    seed = 20260705
    r, st, ko = _case(oracle_mod, panels, seed, 1, 30_000, 300)
    d = _device(pkg, st, seed, 1, 8)
    assert d["failed_lanes"] == 0
    o = ko.jla_leverages(st, seed, 1)
    for k in ("pii", "mii", "bfe", "bpe", "bcov"):
        assert _rel(d[k], o[k]) <= TOL, k
    assert _rel(d["pii"], r["pii"]) <= TOL

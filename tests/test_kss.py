"""CPU checks of the AKM/KSS solver's checker and host logic.

* the numpy restatement of the reference's grounded Jacobi-PCG
  (oracle/kss_oracle.py) against a dense direct solve of the grounded system;
* the package's host-side structure builder (kss_system) against the
  oracle's restatement of TwoWaySolver::build;
* the golden fixture of the reference's own worked example
  (tests/golden/kss_felsdvsimul.npz) against the numbers the reference
  documents for it (docs/akm-kss.md:19-27), and, where the reference's CPU core
  is built, that core reproducing both KSS fixtures.
"""

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def match_set(N, J, seed, zipf=1.3, max_firms=3):
    """Workers with 1..max_firms distinct firms (Zipf firm sizes), weights 1..8."""
    rng = np.random.default_rng(seed)
    p = 1.0 / np.arange(1, J + 1) ** zipf
    p /= p.sum()
    rows = []
    for w in range(N):
        k = int(rng.integers(1, max_firms + 1))
        fs = np.unique(rng.choice(J, size=k, p=p))
        for f in fs:
            rows.append((w, int(f), int(rng.integers(1, 9))))
    rows = np.array(rows)
    # every firm appears at least once (a connected set has no empty firm)
    missing = np.setdiff1d(np.arange(J), rows[:, 1])
    extra = np.array([(int(rng.integers(0, N)), int(f), 1) for f in missing]).reshape(-1, 3)
    rows = np.concatenate([rows, extra]) if extra.size else rows
    rows = rows[np.lexsort((rows[:, 1], rows[:, 0]))]
    keep = np.ones(len(rows), bool)
    keep[1:] = (rows[1:, 0] != rows[:-1, 0]) | (rows[1:, 1] != rows[:-1, 1])
    rows = rows[keep]
    # largest connected component of the worker-firm graph, ids made dense
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    g = coo_matrix((np.ones(len(rows)), (rows[:, 0], N + rows[:, 1])), shape=(N + J, N + J))
    _, lab = connected_components(g, directed=False)
    rows = rows[lab[rows[:, 0]] == np.bincount(lab[rows[:, 0]]).argmax()]
    rows[:, 0] = np.unique(rows[:, 0], return_inverse=True)[1]
    rows[:, 1] = np.unique(rows[:, 1], return_inverse=True)[1]
    return rows


def dims(rows):
    return int(rows[:, 0].max()) + 1, int(rows[:, 1].max()) + 1


def test_oracle_pcg_matches_direct_solve(oracle_mod):
    from oracle import kss_oracle as ko
    rows = match_set(400, 40, seed=1)
    N, J = dims(rows)
    st = ko.kss_structure(rows[:, 0], rows[:, 1], rows[:, 2], N, J)
    b = np.random.default_rng(2).standard_normal(J)
    z, it = ko.kss_pcg(st, b, tol=1e-13, max_iter=10_000)
    zd = ko.grounded_direct(st, b)
    assert it > 0
    assert z[-1] == 0.0
    assert np.abs(z - zd).max() <= 1e-10 * np.abs(zd).max()
    # zero rhs: no iteration, zero solution; too few iterations: failure
    z0, it0 = ko.kss_pcg(st, np.zeros(J))
    assert it0 == 0 and not z0.any()
    zf, itf = ko.kss_pcg(st, b, tol=1e-13, max_iter=2)
    assert itf == -1 and not zf.any()


def test_host_structure_matches_oracle(pkg, oracle_mod):
    from oracle import kss_oracle as ko
    rows = match_set(300, 30, seed=3)
    N, J = dims(rows)
    a = pkg.kss_system(rows[:, 0], rows[:, 1], rows[:, 2], N, J)
    b = ko.kss_structure(rows[:, 0], rows[:, 1], rows[:, 2], N, J)
    for k in ("m_w", "m_f", "m_c", "w_ptr", "f_ptr", "f_matches", "Dw", "Df", "inv_diagS"):
        assert np.array_equal(a[k], b[k]), k


def test_felsdvsimul_fixture_matches_documented_values():
    g = np.load(GOLDEN / "kss_felsdvsimul.npz")
    exact = g["exact_components"]  # plugin (3), agsu (3), kss (3)
    # documented: kss var_alpha, var_psi, cov; plug-in var_psi
    assert exact[6:9] == pytest.approx([-6.2429443959, 6.2254112695, 2.6372007926], abs=5e-11)
    assert exact[1] == pytest.approx(34.398203, abs=5e-7)
    assert g["jla_components"][7] == pytest.approx(6.13308521068209, abs=5e-14)
    # the matrix-free PCG path of the reference agrees with its direct path
    assert g["jla_pcg_components"] == pytest.approx(g["jla_components"], rel=1e-10)


@pytest.mark.parametrize("case", ["felsdvsimul", "akm20k"])
def test_reference_core_reproduces_kss_fixture(oracle_mod, case):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref/libxhdfe_ref.so not built")
    g = np.load(GOLDEN / f"kss_{case}.npz")
    draws = 150 if case == "felsdvsimul" else 200
    seed = 42 if case == "felsdvsimul" else 20260705
    r = oracle_mod.ref_akm_kss(g["y"], g["worker"], g["firm"], leverages="jla", jla_draws=draws,
                               seed=seed, direct_max_firms=0, threads=1)
    got = np.array([r[k][c] for k in ("plugin", "agsu", "kss")
                    for c in ("var_alpha", "var_psi", "cov_alpha_psi")])
    assert got == pytest.approx(g["jla_pcg_components"], rel=1e-12)
    meta = json.loads(str(g["meta"]))["jla_pcg"]
    assert r["solver_iterations"] == meta["solver_iterations"]

"""The oracle pinned to the reference's golden vectors (CPU).

Golden numbers are PySCF 2.13.1 values stored in the reference's
testdata/reference/validation/{sos_mp2,kappa_mp2}/*.json (exact-JK RHF,
DF-MP2 with the named auxiliary basis).  The fixtures in tests/golden/ were
made by tests/golden/make_golden.py with the oracle's own integral engine and
RHF; these tests check the oracle against the golden values (through the
committed fixtures, and -- where the reference's basis files are mounted --
by rerunning the whole oracle pipeline for water).
"""
import os

import numpy as np
import pytest

from oracle import rimp2 as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SYSTEMS = ["h2o_ccpvdz", "ch4_ccpvdz", "h2o_augccpvdz"]
PIN = 1e-9  # Eh: oracle vs PySCF golden (measured <= 6e-13)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.mark.parametrize("name", SYSTEMS)
def test_oracle_rimp2_matches_golden(name):
    d = load(name)
    nocc, nvir = int(d["nocc"]), int(d["nvir"])
    e_os, e_ss, e_tot = orc.spin_components(d["b_ov"], d["eps"], nocc, nvir)
    assert abs(e_os - d["golden_e_os"]) < PIN
    assert abs(e_ss - d["golden_e_ss"]) < PIN
    assert abs(d["oracle_e_rhf"] - d["golden_e_rhf"]) < PIN


@pytest.mark.parametrize("name", ["h2o_ccpvdz", "ch4_ccpvdz"])
def test_oracle_kappa_matches_golden(name):
    d = load(name)
    nocc, nvir = int(d["nocc"]), int(d["nvir"])
    for k, g_os, g_ss in zip(d["kappa"], d["golden_kappa_e_os"], d["golden_kappa_e_ss"]):
        e_os, e_ss, _ = orc.spin_components(d["b_ov"], d["eps"], nocc, nvir, kappa=float(k))
        assert abs(e_os - g_os) < PIN and abs(e_ss - g_ss) < PIN


def test_df_jk_rhf_anchor():
    # DF-JK RHF within 3e-3 of the exact-JK water energy (ferric-scf/tests/dfk_occ_path.rs:216-222)
    d = load("h2o_ccpvdz")
    assert abs(d["oracle_e_dfrhf"] - (-76.0267679973766)) < 3e-3


def test_oracle_pipeline_reruns_to_golden():
    """Integrals -> RHF -> dressing -> RI-MP2 for water from the reference's basis files."""
    from oracle import basis, integrals, scf
    if not basis.available():
        pytest.skip("reference basis files not mounted")
    d = load("h2o_ccpvdz")
    atoms = [("O", (0.0, 0.0, 0.22259084021251865)), ("H", (0.0, 1.4275992699810498, -0.8903652505761991)),
             ("H", (0.0, -1.4275992699810498, -0.8903652505761991))]
    zs = [8, 1, 1]
    rs = [c for _, c in atoms]
    sh = basis.shells_for(atoms, "cc-pvdz")
    S, T = integrals.overlap_kinetic(sh)
    V = integrals.nuclear(sh, zs, rs)
    enuc = scf.nuclear_repulsion(zs, rs)
    assert abs(enuc - 9.189193229309746) < 1e-12
    e, eps, C = scf.rhf(S, T + V, 5, enuc, scf.exact_jk(integrals.eri4(sh)))
    assert abs(e - d["golden_e_rhf"]) < PIN
    b, _, _ = scf.dressed(basis.shells_for(atoms, "cc-pvdz-ri"), sh)
    e_os, e_ss, _ = orc.spin_components(scf.b_ov(b, C, 5), eps, 5, 19)
    assert abs(e_os - d["golden_e_os"]) < PIN
    assert abs(e_ss - d["golden_e_ss"]) < PIN


def test_boys_and_spherical_subspace():
    from oracle import integrals
    t = np.array([0.0, 1e-4, 0.5, 3.0, 30.0])
    f = integrals.boys(3, t)
    assert abs(f[0, 0] - 1.0) < 1e-15 and abs(f[2, 0] - 1.0 / 5.0) < 1e-15
    # F_0(t) = sqrt(pi/t) erf(sqrt(t)) / 2
    from scipy.special import erf
    assert np.allclose(f[0, 2:], 0.5 * np.sqrt(np.pi / t[2:]) * erf(np.sqrt(t[2:])), rtol=1e-14)
    # downward recursion F_n = (2t F_{n+1} + e^-t) / (2n + 1)
    assert np.allclose(f[1, 1:], (2 * t[1:] * f[2, 1:] + np.exp(-t[1:])) / 3.0, rtol=1e-13)
    for l in range(5):
        assert integrals.spherical_transform(l).shape[1] == 2 * l + 1

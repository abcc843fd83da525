"""Device kernels against the reference's golden values (GPU).

The RI-MP2 inputs of water, CH4 and water/aug-cc-pVDZ come from the committed
fixtures (tests/golden/); the golden energies are the reference's PySCF values.
The config-1 case runs a DF-JK RHF whose J and K come from the device
builders every iteration (the host SCF loop is the oracle's), then the RI-MP2
energy on the device from its orbitals.
"""
import os

import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import scf as oscf

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SYSTEMS = ["h2o_ccpvdz", "ch4_ccpvdz", "h2o_augccpvdz"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


@pytest.mark.parametrize("name", SYSTEMS)
@pytest.mark.parametrize("precision,tol", [("f64", 1e-10), ("mixed", 1e-6)])
def test_device_energy_matches_golden(fc, name, precision, tol):
    from ferric_b200 import rimp2
    d = load(name)
    nocc, nvir = int(d["nocc"]), int(d["nvir"])
    sc = rimp2.spin_components_on_device(d["b_ov"], d["eps"], nocc, nvir, precision=precision)
    # golden within tol (the oracle itself sits within 6e-13 of golden)
    assert abs(sc.e_os - d["golden_e_os"]) < tol
    assert abs(sc.e_ss - d["golden_e_ss"]) < tol
    if precision == "f64":
        assert abs(sc.e_os - d["oracle_e_os"]) < 1e-12
        assert abs(sc.e_ss - d["oracle_e_ss"]) < 1e-12


@pytest.mark.parametrize("name", ["h2o_ccpvdz", "ch4_ccpvdz"])
def test_device_kappa_matches_golden(fc, name):
    from ferric_b200 import rimp2
    d = load(name)
    nocc, nvir = int(d["nocc"]), int(d["nvir"])
    for k, g_os, g_ss in zip(d["kappa"], d["golden_kappa_e_os"], d["golden_kappa_e_ss"]):
        sc = rimp2.spin_components_on_device(d["b_ov"], d["eps"], nocc, nvir, kappa=float(k))
        assert abs(sc.e_os - g_os) < 1e-10 and abs(sc.e_ss - g_ss) < 1e-10


@pytest.mark.parametrize("precision", ["f64"])
def test_config1_dfjk_scf_then_rimp2_on_device(fc, precision):
    """Water cc-pVDZ: RHF with DF-JK (cc-pVTZ-JKFIT) on the device builders,
    then the device RI-MP2 energy (cc-pVDZ-RI) from its orbitals."""
    from ferric_b200 import rimp2
    from ferric_b200.dfjk import DfJ, DfJK, DfK
    d = load("h2o_ccpvdz")
    nocc = int(d["nocc"])
    handle = DfJK(d["b_jk"], layout="square", precision=precision)
    jb, kb = DfJ(None, shared=handle), DfK(None, shared=handle)
    n = d["s"].shape[0]

    calls = {"n": 0}

    def device_jk(D):
        # RHF density D = 2 C C^T: J from D, K(D) = 2 K(C_occ) (ferric-scf/src/rhf.rs:3164-3178)
        w, v = np.linalg.eigh(D)
        c = v[:, w > 1e-10] * np.sqrt(w[w > 1e-10] / 2.0)
        J = np.zeros((n, n))
        K = np.zeros((n, n))
        jb.build(D, J)
        kb.build_from_occ(c, K)
        calls["n"] += 1
        return J, 2.0 * K

    e, eps, C = oscf.rhf(d["s"], d["h_core"], nocc, float(d["e_nuc"]), device_jk)
    assert calls["n"] > 3
    assert abs(e - d["oracle_e_dfrhf"]) < 1e-10
    assert abs(e - d["golden_e_rhf"]) < 3e-3   # the DF-JK anchor of ferric-scf/tests/dfk_occ_path.rs:216-222
    b_ov = oscf.b_ov(d["b_ri"], C, nocc)
    sc = rimp2.spin_components_on_device(b_ov, eps, nocc, n - nocc, precision="f64")
    assert abs(sc.e_os - d["oracle_dfrhf_e_os"]) < 1e-10
    assert abs(sc.e_ss - d["oracle_dfrhf_e_ss"]) < 1e-10
    sc_m = rimp2.spin_components_on_device(b_ov, eps, nocc, n - nocc, precision="mixed")
    assert abs(sc_m.e_total - sc.e_total) < 1e-6
    handle.close()

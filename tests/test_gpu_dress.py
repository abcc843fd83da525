"""MO transform + metric dressing on the device (the step before the RI-MP2
path) against the oracle's streamed restatement, on synthetic tensors and on
water (cc-pVDZ / cc-pVDZ-RI from the oracle's own integrals), where the
dressed B_ov then reproduces the golden RI-MP2 energy."""
import os

import numpy as np
import pytest

from oracle import rimp2 as orc

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _synthetic(naux, n, nl, nr, seed=71):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((naux, n, n)) * 0.05
    t3 = (x + x.transpose(0, 2, 1)) / 2
    a = rng.standard_normal((naux, naux))
    v = a @ a.T / naux + np.eye(naux)
    m = np.linalg.inv(np.linalg.cholesky(v))   # L^-1
    cl = rng.standard_normal((n, nl)) / np.sqrt(n)
    cr = rng.standard_normal((n, nr)) / np.sqrt(n)
    return t3, m, cl, cr


@pytest.mark.parametrize("naux,n,nl,nr", [(60, 24, 5, 19), (130, 70, 9, 61), (300, 41, 3, 38), (7, 5, 1, 4)])
def test_dress_f64_and_mixed_match_oracle(fc, naux, n, nl, nr):
    from ferric_b200.dress import mo_dress
    t3, m, cl, cr = _synthetic(naux, n, nl, nr)
    ref = orc.stream_dressed_mo(t3, m, cl, cr)
    st = {}
    b64 = mo_dress(t3, m, cl, cr, precision="f64", stats=st)
    assert st["precision"] == 0
    assert np.abs(b64 - ref).max() <= 1e-12 * np.abs(ref).max()
    bm = mo_dress(t3, m, cl, cr, precision="mixed", stats=st)
    assert st["precision"] == 1
    # exact-slice dressing: each operand row is carried to 2^-23 of its maximum
    # (|dx| <= 2^-17 s, s <= max/64), so
    # |dB_Pw| <= 2^-23 (max_Q |M_PQ| sum_Q |MO_Qw| + max_Q |MO_Qw| sum_Q |M_PQ|)  (x 2 margin)
    mo = np.abs(np.einsum("ml,qmn,nr->qlr", cl, t3, cr).reshape(naux, -1))
    am = np.abs(m)
    bound = 2.0 ** -22 * (am.max(axis=1)[:, None] * mo.sum(axis=0)[None, :]
                          + am.sum(axis=1)[:, None] * mo.max(axis=0)[None, :])
    err = np.abs(bm - ref)
    assert np.all(err <= bound), float((err / bound).max())
    assert err.max() > 0   # the split path really ran


def test_dress_device_api(fc):
    import torch
    from ferric_b200.dress import mo_dress
    t3, m, cl, cr = _synthetic(90, 33, 4, 25, seed=72)
    ref = orc.stream_dressed_mo(t3, m, cl, cr)
    dev = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (t3, m, cl, cr)]
    b = mo_dress(*dev, precision="f64").cpu().numpy()
    assert np.abs(b - ref).max() <= 1e-12 * np.abs(ref).max()


def test_dress_water_reproduces_golden_energy(fc):
    """Raw (P|mn) of water in cc-pVDZ-RI, the metric's L^-1 and the exact-JK
    RHF orbitals (the oracle's own integrals and SCF, fixture made by
    golden/make_golden.py): the device-dressed B_ov gives the golden RI-MP2
    energy."""
    from ferric_b200 import rimp2
    from ferric_b200.dress import mo_dress
    d = np.load(os.path.join(HERE, "golden", "h2o_ccpvdz.npz"))
    nocc, nvir = int(d["nocc"]), int(d["nvir"])
    t3, v, c, eps = d["t3_ri"], d["v_ri"], d["c"], d["eps"]
    m = np.linalg.inv(np.linalg.cholesky(v))
    # mixed: each operand row of the dressing GEMM carries ~24 bits and
    # M = L^-1 . MO cancels heavily (the metric's conditioning), so the energy
    # is within the 1 uEh bar (measured 2.9e-7 Eh here) rather than 1e-10
    for prec, tol in (("f64", 1e-10), ("mixed", 1e-6)):
        b = mo_dress(t3, m, c[:, :nocc], c[:, nocc:], precision=prec)
        if prec == "f64":
            assert np.abs(b - d["b_ov"]).max() <= 1e-11 * np.abs(d["b_ov"]).max()
        e_os, e_ss = rimp2.rimp2_energy(b, eps[:nocc], eps[nocc:], precision="f64")
        assert abs(e_os - float(d["golden_e_os"])) < 1e-6
        assert abs(e_os - float(d["oracle_e_os"])) < tol
        assert abs(e_ss - float(d["oracle_e_ss"])) < tol

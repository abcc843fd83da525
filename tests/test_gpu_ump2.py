"""Unrestricted RI-MP2 energy components on the device against the oracle
(u_rimp2.rs:693-753 restated) and the reference's golden UMP2 energies of
OH and NH2 (cc-pVDZ / cc-pVDZ-RI, PySCF DF-UMP2; inputs from the oracle's own
integrals and UHF, fixtures made by golden/make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
# Energy bound of the split: each element of G carries 23-24 bits relative
# to its row maximum, so for small systems, where a few elements dominate E,
# E's relative error reaches ~2.6e-7 (largest of 120 seeded random systems
# of 2-4 occupied orbitals; either integer-slice format, emulated exactly);
# large systems sit near 1e-10.
MIXED_E_REL = 3e-7


def _spin(naux, nocc, nvir, seed):
    return synthetic.rimp2_inputs(naux, nocc, nvir, seed_b=seed, seed_eps=seed + 1)


@pytest.mark.parametrize("naux,noa,nva,nob,nvb", [(96, 5, 23, 4, 24), (200, 7, 65, 6, 66), (130, 1, 30, 2, 29),
                                                  (300, 9, 130, 8, 131), (64, 3, 128, 3, 128)])
def test_ump2_matches_oracle(fc, naux, noa, nva, nob, nvb):
    from ferric_b200 import rimp2
    ba, eoa, eva = _spin(naux, noa, nva, 81)
    bb, eob, evb = _spin(naux, nob, nvb, 91)
    ref = (orc.u_same_spin(ba, eoa, eva), orc.u_same_spin(bb, eob, evb),
           orc.u_opposite_spin(ba, eoa, eva, bb, eob, evb))
    e64 = rimp2.ump2_energy(ba, eoa, eva, bb, eob, evb, precision="f64")
    for x, r in zip(e64, ref):
        assert abs(x - r) <= 1e-10 + 1e-13 * abs(r)
    em = rimp2.ump2_energy(ba, eoa, eva, bb, eob, evb, precision="mixed")
    # same-spin sums (X - Y)^2, whose cancellation costs relative precision:
    # each component within the mixed bar of the total correlation energy
    scale = sum(abs(r) for r in ref)
    for x, r in zip(em, ref):
        assert abs(x - r) <= MIXED_E_REL * scale + 1e-12


def test_ump2_closed_shell_limit(fc):
    """alpha = beta: e_aa + e_bb = E_SS and e_ab = E_OS of the closed-shell kernel.
    In mixed precision e_ab comes from the opposite-spin GEMM on bf16 slices and
    E_OS from the pair kernel on int8 slices: two independent splits, equal to
    the split's precision."""
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(150, 6, 45)
    for prec in ("f64", "mixed"):
        e_os, e_ss = rimp2.rimp2_energy(b, eo, ev, precision=prec)
        e_aa, e_bb, e_ab = rimp2.ump2_energy(b, eo, ev, b, eo, ev, precision=prec)
        assert abs(e_aa + e_bb - e_ss) <= 1e-12 * abs(e_ss)
        assert abs(e_ab - e_os) <= (1e-12 if prec == "f64" else MIXED_E_REL) * abs(e_os)


@pytest.mark.parametrize("name", ["oh_ump2", "nh2_ump2"])
def test_ump2_golden(fc, name):
    from ferric_b200 import rimp2
    d = np.load(os.path.join(HERE, "golden", name + ".npz"))
    na, nb = int(d["na"]), int(d["nb"])
    ea, eb = d["eps_a"], d["eps_b"]
    args = (d["b_a"], ea[:na], ea[na:], d["b_b"], eb[:nb], eb[nb:])
    for prec, tol_oracle in (("f64", 1e-10), ("mixed", 1e-8)):
        e = rimp2.ump2_energy(*args, precision=prec)
        for x, key in zip(e, ("e_aa", "e_bb", "e_ab")):
            assert abs(x - float(d["oracle_" + key])) < tol_oracle, (prec, key)
            assert abs(x - float(d["golden_" + key])) < 1e-9 + (tol_oracle if prec == "mixed" else 0), (prec, key)


def test_ump2_device_api(fc):
    import torch
    from ferric_b200 import rimp2
    ba, eoa, eva = _spin(120, 5, 40, 101)
    bb, eob, evb = _spin(120, 4, 41, 111)
    host = rimp2.ump2_energy(ba, eoa, eva, bb, eob, evb, precision="mixed")
    dev = rimp2.ump2_energy(*(torch.from_numpy(x).cuda() for x in (ba, eoa, eva, bb, eob, evb)), precision="mixed")
    assert np.allclose(host, dev, rtol=1e-14, atol=0)

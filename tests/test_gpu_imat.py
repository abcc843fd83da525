"""RI Lagrangian Imat on the device (the first consumer of the RI-MP2 adjoint)
against the oracle's restatement of build_imat_ri, with the reference's own
known-answer bar (zvector.rs:1245-1290), and fed with the device's own
Gamma."""
import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("naux,nocc,nvir,fo", [(9, 4, 7, 2), (70, 5, 19, 1), (200, 9, 70, 0), (131, 3, 129, 2)])
def test_imat_f64_and_mixed(fc, naux, nocc, nvir, fo):
    from ferric_b200 import rimp2
    nmo = fo + nocc + nvir
    rng = np.random.default_rng(naux + nocc)
    x = rng.uniform(-1, 1, (naux, nocc * nvir))
    bf = rng.uniform(-1, 1, (naux, nmo, nmo))
    want = orc.imat_ri(x, bf, nocc, nvir, fo)
    absum = 2.0 * np.abs(orc.imat_ri(np.abs(x), np.abs(bf), nocc, nvir, fo)) / 2.0
    st = {}
    got = rimp2.rimp2_imat(x, bf, nocc, nvir, fo, precision="f64", stats=st)
    bar = (naux * max(nocc, nvir) + 2.0) * np.finfo(float).eps
    assert np.all(np.abs(got - want) <= bar * absum + 1e-300)
    assert np.all(got[:, :fo] == 0.0)
    gm = rimp2.rimp2_imat(x, bf, nocc, nvir, fo, precision="mixed")
    # exact slices: each operand row to 2^-23 of its maximum
    assert np.all(np.abs(gm - want) <= 2.0 ** -21 * absum * 4 + 1e-300)
    assert np.all(gm[:, :fo] == 0.0)


def test_imat_from_device_gamma(fc):
    """Imat of x_ov = Gamma / 4 from the device adjoint equals the oracle's
    Imat of the oracle's x_ov."""
    import torch
    from ferric_b200 import rimp2
    naux, nocc, nvir = 120, 6, 37
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    nmo = nocc + nvir
    bf = np.random.default_rng(5).standard_normal((naux, nmo, nmo)) * 0.05
    bf[:, :nocc, nocc:] = b.reshape(naux, nocc, nvir)
    _, gamma, _, _ = rimp2.rimp2_energy_grad(b, eo, ev, precision="f64")
    t2, _ = orc.t2_and_integrals(b, eo, ev)
    x_ov = orc.x_ov_from_t2(t2, b, nocc, nvir)
    want = orc.imat_ri(x_ov, bf, nocc, nvir)
    got = rimp2.rimp2_imat(torch.from_numpy(gamma / 4).cuda(), torch.from_numpy(bf).cuda(), nocc, nvir).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()

"""RiMp2Energy autograd function: gradients against central finite differences
of the oracle energy and against the oracle's Gamma = 4 x_ov and 2 diag(P)."""
import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu


def test_autograd_f64_matches_fd_and_identities(fc):
    import torch
    from ferric_b200.torch_ops import RiMp2Energy
    naux, nocc, nvir = 120, 6, 37
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    tb = torch.from_numpy(b).cuda().requires_grad_(True)
    to = torch.from_numpy(eo).cuda().requires_grad_(True)
    tv = torch.from_numpy(ev).cuda().requires_grad_(True)
    e = RiMp2Energy.apply(tb, to, tv, "f64")
    e.backward()
    gb, go, gv = tb.grad.cpu().numpy(), to.grad.cpu().numpy(), tv.grad.cpu().numpy()

    # identities: Gamma = 4 x_ov, dE/deps = 2 diag(P)
    t2, _ = orc.t2_and_integrals(b, eo, ev)
    x_ov = orc.x_ov_from_t2(t2, b, nocc, nvir)
    p_oo, p_vv = orc.mp2_density(t2, nocc, nvir)
    assert np.abs(gb - 4 * x_ov).max() < 1e-12 * np.abs(gb).max()
    assert np.abs(go - 2 * np.diag(p_oo)).max() < 1e-12 * np.abs(go).max()
    assert np.abs(gv - 2 * np.diag(p_vv)).max() < 1e-12 * np.abs(gv).max()

    # central differences of the oracle energy at h = 1e-5 on seeded entries
    eps = np.concatenate([eo, ev])
    h = 1e-5
    rows, cols = synthetic.fd_entries(naux, nocc * nvir, count=64)
    for p, ia in zip(rows, cols):
        bp = b.copy(); bp[p, ia] += h
        bm = b.copy(); bm[p, ia] -= h
        fd = (orc.spin_components(bp, eps, nocc, nvir)[2]
              - orc.spin_components(bm, eps, nocc, nvir)[2]) / (2 * h)
        assert abs(fd - gb[p, ia]) < 1e-8 * max(1.0, abs(fd)) + 1e-11


def test_no_grad_forward_is_energy_only(fc):
    import torch
    from ferric_b200.torch_ops import RiMp2Energy
    b, eo, ev = synthetic.rimp2_inputs(96, 5, 23)
    with torch.no_grad():
        e = RiMp2Energy.apply(torch.from_numpy(b).cuda(), torch.from_numpy(eo).cuda(),
                              torch.from_numpy(ev).cuda(), "f64")
    ref = orc.spin_components(b, np.concatenate([eo, ev]), 5, 23)[2]
    assert abs(e.item() - ref) < 1e-10


def test_autograd_mixed_matches_fd_of_fp64_oracle(fc):
    import torch
    from ferric_b200.torch_ops import RiMp2Energy
    naux, nocc, nvir = 150, 6, 45
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    tb = torch.from_numpy(b).cuda().requires_grad_(True)
    to = torch.from_numpy(eo).cuda().requires_grad_(True)
    tv = torch.from_numpy(ev).cuda().requires_grad_(True)
    e = RiMp2Energy.apply(tb, to, tv, "mixed")
    e.backward()
    gb = tb.grad.cpu().numpy()
    eps = np.concatenate([eo, ev])
    ref = orc.spin_components(b, eps, nocc, nvir)[2]
    assert abs(e.item() - ref) <= 5e-8 * abs(ref)
    h = 1e-5
    rows, cols = synthetic.fd_entries(naux, nocc * nvir, count=64)
    scale = np.abs(gb).max()
    for p, ia in zip(rows, cols):
        bp = b.copy(); bp[p, ia] += h
        bm = b.copy(); bm[p, ia] -= h
        fd = (orc.spin_components(bp, eps, nocc, nvir)[2] - orc.spin_components(bm, eps, nocc, nvir)[2]) / (2 * h)
        assert abs(fd - gb[p, ia]) <= 1e-5 * scale

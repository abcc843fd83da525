"""Full-size checks (config 3: naux 4800, nocc 120, nvir 1100; config 2: n 600,
naux 2400, nocc 60) through size-independent identities, where the oracle
would take hours:
  * Euler: E is homogeneous of degree 4 in B, so sum(B * Gamma) = 4 E;
  * shift invariance: D_ijab does not change when every orbital energy
    moves by the same constant, so sum_p dE/d eps_p = 0;
  * power-of-two scaling: 2 B gives exactly 16 E and 8 Gamma through the
    exact slices (the split scales are powers of two);
  * the mixed energy within its bar of the FP64 plain energy;
  * DF-JK: J, K exactly symmetric, K positive semidefinite, and
    tr(J D) = sum_P d_P^2 with d_P = <B_P, D> (dressed B, no metric).
Inputs are the bench's seeded synthetic distributions, made on the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rimp2_inputs(torch):
    naux, nocc, nvir = 4800, 120, 1100
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    b = torch.randn((naux, nocc * nvir), generator=g, device="cuda", dtype=torch.float64)
    b *= 0.02 * torch.exp(-torch.arange(naux, device="cuda", dtype=torch.float64) / 3000.0)[:, None]
    r = np.random.default_rng(30)
    eo = torch.from_numpy(np.sort(r.uniform(-20.0, -0.3, nocc))).cuda()
    ev = torch.from_numpy(np.sort(r.uniform(0.05, 6.0, nvir))).cuda()
    return b, eo, ev


def test_rimp2_config3_identities(fc):
    import torch
    from ferric_b200 import rimp2
    b, eo, ev = _rimp2_inputs(torch)
    sc, gamma, d_o, d_v = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    e = sc.e_total
    euler = float((b * gamma).sum())
    assert abs(euler - 4.0 * e) <= 2e-6 * abs(4.0 * e)
    shift = float(d_o.sum() + d_v.sum())
    assert abs(shift) <= 1e-9 * float(d_o.abs().sum() + d_v.abs().sum())
    e_only = rimp2.rimp2_energy(b, eo, ev, precision="mixed")
    assert abs(sum(e_only) - e) <= 1e-9 * abs(e)
    sc2, gamma2, _, _ = rimp2.rimp2_energy_grad(2.0 * b, eo, ev, precision="mixed")
    assert abs(sc2.e_total - 16.0 * e) <= 1e-12 * abs(16.0 * e)
    assert float((gamma2 - 8.0 * gamma).abs().max()) <= 1e-12 * float(gamma2.abs().max())
    e64 = rimp2.rimp2_energy(b, eo, ev, precision="f64")
    assert abs(sum(e64) - e) <= 5e-8 * abs(e)


def test_dfjk_config2_identities(fc):
    import torch
    from ferric_b200.dfjk import DfJK
    n, naux, nocc = 600, 2400, 60
    g = torch.Generator(device="cuda")
    g.manual_seed(2)
    idx = torch.arange(n, device="cuda", dtype=torch.float64)
    env = 0.05 * torch.exp(-(idx[:, None] - idx[None, :]).abs() / 50.0)
    bjk = torch.empty((naux, n, n), device="cuda", dtype=torch.float64)
    for q0 in range(0, naux, 256):
        x = torch.randn((min(256, naux - q0), n, n), generator=g, device="cuda", dtype=torch.float64) * env
        bjk[q0:q0 + x.shape[0]] = (x + x.transpose(1, 2)) / (2.0 ** 0.5)
    c, _ = np.linalg.qr(np.random.default_rng(20).standard_normal((n, nocc)))
    c = torch.from_numpy(np.ascontiguousarray(c)).cuda()
    d = c @ c.T
    dp = torch.einsum("qmn,mn->q", bjk, d)
    for prec in ("f64", "mixed"):
        jk = DfJK(bjk, layout="square", precision=prec)
        j = jk.j(d)
        k = jk.k_from_occ(c)
        assert torch.equal(j, j.T) and torch.equal(k, k.T)
        w = torch.linalg.eigvalsh(k)
        assert float(w.min()) >= -1e-9 * float(w.max())
        tr = float((j * d).sum())
        ref = float((dp * dp).sum())
        assert abs(tr - ref) <= (1e-12 if prec == "f64" else 1e-6) * ref
        jk.close()

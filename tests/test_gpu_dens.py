"""Unrelaxed MP2 densities P_oo / P_vv on the B200 (fc_rimp2_energy_grad_dens)
against the oracle's build_mp2_density restatement
(ferric-mp2/src/oo_rimp2.rs:1170-1300), FP64 and FC_PREC_MIXED, one column
chunk and several (pair blocks recomputed per column)."""
import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

SHAPES = [
    (96, 5, 23),     # nvir below one 128-tile, odd
    (200, 7, 65),    # one past a 32-tile edge
    (300, 9, 140),   # two 128-tiles of virtuals
    (17, 1, 1),      # one occupied, one virtual
    (160, 130, 9),   # two 128-tiles of occupied orbitals (P_oo tile pairs (0,0), (0,1), (1,1))
]


def _ref(b, eo, ev):
    nocc, nvir = len(eo), len(ev)
    t2, _ = orc.t2_and_integrals(b, eo, ev)
    p_oo, p_vv = orc.mp2_density(t2, nocc, nvir)
    return t2, p_oo, p_vv


def _mixed_bound(t2, nocc, nvir):
    """Elementwise bound of the FC_PREC_MIXED density error.  Each slab row
    (i, a) of t and of Tt = 2t - t^T is cut into three int8 slices at a
    power-of-two scale s with max|x| / s in (63.5, 127]: the residual is at
    most s / (2 * 254^2) <= max|x| / (127 * 254^2).  Tt is stored in FP32
    (2^-24 relative) and t is formed from it in FP32.  The bound sums these
    over the contraction with absolute values."""
    t = t2.reshape(nocc, nvir, nocc, nvir)
    tt = 2.0 * t - t.transpose(0, 3, 2, 1)
    at, att = np.abs(t), np.abs(tt)
    sl = 1.0 / (127.0 * 254.0 ** 2)
    rm_t = at.max(axis=(2, 3))     # [i, a]: row maxima over all columns (>= a slab's)
    rm_tt = att.max(axis=(2, 3))
    s1_t = at.sum(axis=(2, 3))     # [i, a]: row sums
    s1_tt = att.sum(axis=(2, 3))
    f32 = 4.0 * 2.0 ** -24
    # P_vv[a, b] = sum_i sum_(j c) t[i a, j c] Tt[i b, j c]
    vv = sl * (np.einsum("ia,ib->ab", rm_t, s1_tt) + np.einsum("ia,ib->ab", s1_t, rm_tt)) \
        + f32 * np.einsum("iajc,ibjc->ab", at + np.abs(t.transpose(0, 3, 2, 1)), att)
    # P_oo[i, j] = -sum_a sum_(k b) t[i a, k b] Tt[j a, k b]
    oo = sl * (np.einsum("ia,ja->ij", rm_t, s1_tt) + np.einsum("ia,ja->ij", s1_t, rm_tt)) \
        + f32 * np.einsum("iakb,jakb->ij", at + np.abs(t.transpose(0, 3, 2, 1)), att)
    # mirrored tiles carry the transposed entry's error
    return np.maximum(oo, oo.T), np.maximum(vv, vv.T)


@pytest.mark.parametrize("naux,nocc,nvir", SHAPES)
def test_densities_f64_match_oracle(fc, naux, nocc, nvir):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    _, p_oo, p_vv = _ref(b, eo, ev)
    sc, g, d_o, d_v, q_oo, q_vv = rimp2.rimp2_energy_grad_dens(b, eo, ev, precision="f64")
    assert np.abs(q_oo - p_oo).max() <= 1e-12 * np.abs(p_oo).max() + 1e-300
    assert np.abs(q_vv - p_vv).max() <= 1e-12 * np.abs(p_vv).max() + 1e-300
    assert np.array_equal(q_oo, q_oo.T) and np.array_equal(q_vv, q_vv.T)
    # dE/deps = 2 diag(P) (oo_rimp2.rs:1170-1191), from the pair kernel
    assert np.abs(2.0 * np.diag(q_oo) - d_o).max() <= 1e-12 * np.abs(d_o).max()
    assert np.abs(2.0 * np.diag(q_vv) - d_v).max() <= 1e-12 * np.abs(d_v).max()
    # energy and Gamma as the gradient call's
    sc2, g2, _, _ = rimp2.rimp2_energy_grad(b, eo, ev, precision="f64")
    assert abs(sc.e_total - sc2.e_total) <= 1e-13 * abs(sc2.e_total)
    assert np.abs(g - g2).max() <= 1e-13 * np.abs(g2).max()


@pytest.mark.parametrize("naux,nocc,nvir", SHAPES)
def test_densities_mixed_match_oracle(fc, naux, nocc, nvir):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    t2, p_oo, p_vv = _ref(b, eo, ev)
    bo, bv = _mixed_bound(t2, nocc, nvir)
    sc, g, d_o, d_v, q_oo, q_vv = rimp2.rimp2_energy_grad_dens(b, eo, ev, precision="mixed")
    assert np.all(np.abs(q_oo - p_oo) <= bo + 1e-300)
    assert np.all(np.abs(q_vv - p_vv) <= bv + 1e-300)
    assert np.array_equal(q_oo, q_oo.T) and np.array_equal(q_vv, q_vv.T)
    # the mixed gradient's outputs are unchanged by the density schedule
    sc2, g2, d_o2, d_v2 = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert abs(sc.e_total - sc2.e_total) <= 1e-14 * abs(sc2.e_total)
    assert np.array_equal(g, g2)
    assert np.abs(d_o - d_o2).max() <= 1e-14 * np.abs(d_o2).max()
    assert np.abs(d_v - d_v2).max() <= 1e-14 * np.abs(d_v2).max()


def _fx_budget(nocc, nvir, chunk):
    tp = (nvir + 15) // 16 * 16
    return (chunk + 1) ** 2 * (tp * tp * 11 + 1024 * tp) - 1


def _f64_budget(nvir, chunk):
    return 2 * (chunk + 1) ** 2 * nvir * nvir * 8 - 1


@pytest.mark.parametrize("prec,store", [("f64", "1"), ("mixed", "1"), ("mixed", "0")])
def test_densities_chunked(fc, monkeypatch, prec, store):
    """Occupied chunks of 2 (the last shorter): every column chunk's slab
    takes blocks from chunk pairs on both sides of the diagonal.  FP64 and
    the recomputing mixed form run the off-diagonal chunk pairs once per
    column (25 pair launches); the mixed store form runs each chunk pair once
    (15) and keeps the blocks above the diagonal in FP32 until their column.
    Energy, dE/deps and the densities are those of one chunk (FP64 to
    summation order; mixed within the slicing bound, the slab rows being
    split at their own maxima)."""
    from ferric_b200 import rimp2
    monkeypatch.setenv("FERRIC_CUDA_DENS_STORE", store)
    naux, nocc, nvir = 160, 9, 40
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    t2, p_oo, p_vv = _ref(b, eo, ev)
    one = rimp2.rimp2_energy_grad_dens(b, eo, ev, precision=prec)
    budget = _f64_budget(nvir, 2) if prec == "f64" else _fx_budget(nocc, nvir, 2)
    monkeypatch.setenv("FERRIC_CUDA_CHUNK_BYTES", str(budget))
    st = {}
    many = rimp2.rimp2_energy_grad_dens(b, eo, ev, precision=prec, stats=st)
    # 5 column chunks: 5 x 5 blocks, or the 15 chunk pairs once
    assert st["main_launches"] == (15 if prec == "mixed" and store == "1" else 25)
    assert abs(one[0].e_total - many[0].e_total) <= 1e-13 * abs(one[0].e_total)
    assert np.abs(one[2] - many[2]).max() <= 1e-13 * np.abs(one[2]).max()
    assert np.abs(one[3] - many[3]).max() <= 1e-13 * np.abs(one[3]).max()
    if prec == "f64":
        assert np.abs(many[4] - p_oo).max() <= 1e-12 * np.abs(p_oo).max()
        assert np.abs(many[5] - p_vv).max() <= 1e-12 * np.abs(p_vv).max()
        assert np.abs(many[1] - one[1]).max() <= 1e-13 * np.abs(one[1]).max()
    else:
        bo, bv = _mixed_bound(t2, nocc, nvir)
        assert np.all(np.abs(many[4] - p_oo) <= bo)
        assert np.all(np.abs(many[5] - p_vv) <= bv)
        # Gamma as the chunked gradient call's: the same blocks, split alike
        g = rimp2.rimp2_energy_grad(b, eo, ev, precision=prec)[1]
        assert np.abs(many[1] - g).max() <= 1e-13 * np.abs(g).max()
    # the chunked gradient call (no densities) gives the same energy
    sc, *_ = rimp2.rimp2_energy_grad(b, eo, ev, precision=prec)
    assert abs(sc.e_total - many[0].e_total) <= 1e-13 * abs(sc.e_total)


def test_densities_device_api(fc):
    """The device form on torch CUDA tensors equals the host form bit for bit."""
    import torch
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(120, 6, 50)
    for prec in ("f64", "mixed"):
        h = rimp2.rimp2_energy_grad_dens(b, eo, ev, precision=prec)
        d = rimp2.rimp2_energy_grad_dens(*(torch.from_numpy(x).cuda() for x in (b, eo, ev)), precision=prec)
        assert h[0].e_total == d[0].e_total
        for x, y in zip(h[1:], d[1:]):
            assert np.array_equal(x, y.cpu().numpy())


def test_ri_densities_shapes(fc):
    """ri_densities gives exactly from_ri_densities' arguments (after rpa):
    x_ov (naux, nov), p_oo (nocc, nocc), p_vv (nvir, nvir), e_corr
    (ferric-mp2/src/rimp2.rs:1849-1854)."""
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(64, 4, 12)
    x, p_oo, p_vv, e = rimp2.ri_densities(b, eo, ev)
    assert x.shape == (64, 48) and p_oo.shape == (4, 4) and p_vv.shape == (12, 12)
    e_os, e_ss, gamma, _, _ = orc.energy_gamma_deps(b, eo, ev)
    assert abs(e - (e_os + e_ss)) <= 1e-10
    assert np.abs(x - gamma / 4.0).max() <= 1e-12 * np.abs(gamma).max()


def test_densities_empty_and_refusals(fc):
    """No virtuals: E = 0, P_oo = 0 (nocc x nocc), P_vv empty; a non-finite
    B_ov element is refused by the mixed split (FC_ERR_RANGE), as in the
    gradient call."""
    from ferric_b200 import rimp2, _lib
    b = np.zeros((10, 0))
    sc, g, d_o, d_v, p_oo, p_vv = rimp2.rimp2_energy_grad_dens(b, np.array([-1.0, -0.5]), np.zeros(0))
    assert sc.e_total == 0.0 and p_oo.shape == (2, 2) and not p_oo.any() and p_vv.shape == (0, 0)
    b, eo, ev = synthetic.rimp2_inputs(40, 3, 9)
    b[5, 7] = np.inf
    with pytest.raises(_lib.FcError) as e:
        rimp2.rimp2_energy_grad_dens(b, eo, ev, precision="mixed")
    assert e.value.name == "FC_ERR_RANGE"

"""DF-J / DF-K parity on the B200: the FP64 plain kernels against the oracle."""
import numpy as np
import pytest

from oracle import dfjk as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

F_TOL = 1e-10  # max|dJ|, max|dK| of the FP64 plain form


@pytest.mark.parametrize("n,naux,nocc", [(30, 50, 6), (65, 130, 9), (130, 260, 17), (1, 3, 1)])
def test_dfj_dfk_f64_match_oracle(fc, n, naux, nocc):
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(n, naux, nocc)
    jk = DfJK(b, layout="square", precision="f64")
    j = jk.j(d)
    k = jk.k_from_occ(c)
    assert np.abs(j - orc.df_j_square(b, d)).max() < F_TOL
    assert np.abs(k - orc.df_k_occ(b, c)).max() < F_TOL
    assert np.array_equal(k, k.T)
    assert np.array_equal(j, j.T)
    jk.close()


def test_packed_layout_and_metric(fc):
    from ferric_b200.dfjk import DfJ
    rng = np.random.default_rng(5)
    b, c, d = synthetic.dfjk_inputs(40, 70, 5)
    a = rng.standard_normal((70, 70))
    v = a @ a.T + 70 * np.eye(70)
    l = orc.cholesky_lower(v)
    raw = np.einsum("pq,qmn->pmn", l, b)
    bp = orc.pack_lower(raw)
    builder = DfJ(bp, n=40, layout="packed_lower", metric_chol=l)
    j = np.zeros((40, 40))
    assert builder.build(d, j) == 0
    assert np.abs(j - orc.df_j_packed(bp, d, metric_chol=l)).max() < F_TOL


def test_nonsymmetric_density_j(fc):
    from ferric_b200.dfjk import DfJK
    b, c, _ = synthetic.dfjk_inputs(33, 40, 4)
    d = np.random.default_rng(9).standard_normal((33, 33))
    jk = DfJK(b)
    assert np.abs(jk.j(d) - orc.df_j_packed(orc.pack_lower(b), d)).max() < F_TOL


def test_k_from_occ_empty_channel(fc):
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(20, 30, 3)
    jk = DfJK(b)
    k = jk.k_from_occ(np.zeros((20, 0)))
    assert np.all(k == 0)


def test_k_rebuild_bit_identical(fc):
    # device K must be bit-identical on rebuild (gpu_dfk_resident.rs:30-36)
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(65, 130, 9)
    jk = DfJK(b)
    assert np.array_equal(jk.k_from_occ(c), jk.k_from_occ(c))
    assert np.array_equal(jk.j(d), jk.j(d))


def test_device_api(fc):
    import torch
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(65, 130, 9)
    jk = DfJK(torch.from_numpy(b).cuda())
    j = jk.j(torch.from_numpy(d).cuda()).cpu().numpy()
    k = jk.k_from_occ(torch.from_numpy(c).cuda()).cpu().numpy()
    assert np.abs(j - orc.df_j_square(b, d)).max() < F_TOL
    assert np.abs(k - orc.df_k_occ(b, c)).max() < F_TOL


def test_mixed_dfj_fp32_storage(fc):
    """Mixed DF-J keeps B in FP32 (the reference's f32 RI-J tier) with FP64
    accumulation: max|dJ| within FP32 rounding of the terms."""
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(130, 260, 17)
    ref = orc.df_j_square(b, d)
    jk = DfJK(b, precision="mixed")
    st = {}
    j = jk.j(d, stats=st)
    assert st["precision"] == 1
    # |dJ_k| <= 2 u32 sum_P |B_Pk| |c_P| (two passes through the rounded B)
    bound = 2 * 2.0 ** -24 * np.abs(b).reshape(260, -1).T @ np.abs(np.einsum("qmn,mn->q", b, d))
    assert np.all(np.abs(j - ref).reshape(-1) <= bound + 1e-300)
    assert np.abs(j - ref).max() > 0      # it really ran on the FP32 copy
    jk.set_precision("f64")
    j64 = jk.j(d)
    assert np.abs(j64 - ref).max() < F_TOL
    k64 = jk.k_from_occ(c)
    assert np.abs(k64 - orc.df_k_occ(b, c)).max() < F_TOL
    jk.set_precision("mixed")
    assert np.array_equal(jk.j(d), j)


@pytest.mark.parametrize("sub", [False, True])
@pytest.mark.parametrize("n,naux", [(65, 30), (190, 40)])
def test_mixed_dfj_widening_exact(fc, n, naux, sub):
    """The FP32 passes widen each stored element to FP64 exactly: J equals the
    FP64 build of the FP32-rounded tensor to FP64 rounding.  Zeros (+0 and
    -0) and negatives are planted, and with ``sub`` FP32 subnormals, which
    the copy keeps (round_f64_to_f32.cu: no flush) and the passes then widen
    through their exact variant; n = 65 gives a pair count that is not a
    multiple of 4 (padded pitch), n = 190 more than one pass-1 segment."""
    from ferric_b200.dfjk import DfJK
    b, _, d = synthetic.dfjk_inputs(n, naux, 23)
    b = b.copy()
    rng = np.random.default_rng(8)
    q = rng.integers(0, naux, 600)
    m = rng.integers(0, n, 600)
    k = rng.integers(0, n, 600)
    tiny = rng.choice([-1.0, 1.0], 200) * 10.0 ** (rng.uniform(-44, -39, 200) if sub else rng.uniform(-37, -30, 200))
    vals = np.concatenate([np.zeros(100), -np.zeros(100), tiny, -np.abs(rng.standard_normal(200))])
    b[q, m, k] = vals
    lo, hi = np.tril_indices(n, -1)
    b[:, hi, lo] = b[:, lo, hi]        # symmetric again (planted pairs may collide)
    b32 = b.astype(np.float32).astype(np.float64)
    assert np.any((b32 != 0) & (np.abs(b32) < np.finfo(np.float32).tiny)) == sub
    ref = orc.df_j_square(b32, d)
    jk = DfJK(b, precision="mixed")
    j = jk.j(d)
    assert np.abs(j - ref).max() <= 1e-12 * np.abs(ref).max()
    jk.close()


def test_set_precision_refuses_missing_copy(fc):
    import ferric_b200._lib as L
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(20, 30, 3)
    jk = DfJK(b, precision="f64")
    with pytest.raises(L.FcError):
        jk.set_precision("mixed")


@pytest.mark.parametrize("n,naux,nocc", [(30, 50, 6), (65, 130, 9), (130, 260, 17), (200, 300, 70), (1, 3, 1)])
def test_mixed_dfk_exact_slices(fc, n, naux, nocc):
    """Exact-slice DF-K (tcgen05: stage 1 on int8 slices with exact int32
    levels, stage 2 on bf16 slices with a k-panel FP64 flush): |dK| within
    the slicing error -- B, C and W rows carry about 24 significant bits and
    W is rounded to FP32 once -- and K exactly symmetric and bit-identical on
    rebuild."""
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(n, naux, nocc)
    ref = orc.df_k_occ(b, c)
    jk = DfJK(b, precision="mixed")
    st = {}
    k = jk.k_from_occ(c, stats=st)
    assert st["precision"] == 1
    assert np.array_equal(k, k.T)
    # |dK_mn| <= 2^-20 sum_Qi |W_m,Qi| |W_n,Qi| with W = B_Q C (four slice / rounding terms of 2^-23 .. 2^-24)
    w = np.abs(np.einsum("qmn,ni->mqi", b, c)).reshape(n, -1)
    bound = 2.0 ** -20 * (w @ w.T)
    err = np.abs(k - ref)
    assert np.all(err <= bound + 1e-300), float((err / (bound + 1e-300)).max())
    assert np.array_equal(jk.k_from_occ(c), k)
    jk.close()


def test_mixed_dfk_refuses_nonfinite_c(fc):
    import ferric_b200._lib as L
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(30, 50, 6)
    jk = DfJK(b, precision="mixed")
    c = c.copy()
    c[3, 2] = np.nan
    with pytest.raises(L.FcError) as ei:
        jk.k_from_occ(c)
    assert ei.value.name == "FC_ERR_RANGE"
    jk.close()


# (320, 40, 301) and (1040, 12, 1030): more than 256 vectors per aux row in
# J's first pass (FP64 odd nocc, one double per vector; mixed, four floats)
@pytest.mark.parametrize("n,naux,nocc", [(30, 50, 6), (65, 130, 9), (130, 260, 17), (200, 300, 70), (1, 3, 1),
                                         (320, 40, 301), (1040, 12, 1030)])
def test_fused_jk_from_occ(fc, n, naux, nocc):
    """fc_dfjk_build_occ: K as fc_dfk_build_occ (the same bits) and
    J = J(C C^T) with J's first pass read off K's stage-1 product W = B C:
    FP64 within 1e-10 of the oracle; mixed within the FP32-storage bound of
    J's second pass plus the slicing and FP32 rounding of W in d."""
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(n, naux, nocc)
    j_ref, k_ref = orc.df_j_square(b, d), orc.df_k_occ(b, c)
    for prec in ("f64", "mixed"):
        jk = DfJK(b, precision=prec)
        st = {}
        j, k = jk.jk_from_occ(c, stats=st)
        assert st["aux_launches"] == 1 and st["aux_ms"] > 0
        assert np.array_equal(k, jk.k_from_occ(c))
        assert np.array_equal(j, j.T)
        if prec == "f64":
            assert np.abs(j - j_ref).max() < F_TOL and np.abs(k - k_ref).max() < F_TOL
            assert np.abs(j - jk.j(d)).max() <= 1e-12 * max(1.0, np.abs(j_ref).max())
        else:
            # pass 2 on FP32-stored B, plus d's error: W = B C from slices
            # carrying ~24 bits of each row of B and of C, rounded to FP32
            dp = np.einsum("qmn,mn->q", b, d)
            cc = np.abs(c) @ np.abs(c).T
            bound = 2.0 ** -23 * np.einsum("qmn,q->mn", np.abs(b), np.abs(dp)) \
                + 2.0 ** -20 * np.einsum("qmn,q->mn", np.abs(b), np.einsum("qmn,mn->q", np.abs(b), cc))
            assert np.all(np.abs(j - j_ref) <= bound + 1e-300)
        jk.close()


def test_fused_jk_device_api_and_metric(fc):
    """The device form on torch tensors equals the host form, and a metric
    set on the handle enters J as in fc_dfj_build (c = V^-1 d)."""
    import torch
    from ferric_b200.dfjk import DfJK
    rng = np.random.default_rng(7)
    b, c, d = synthetic.dfjk_inputs(48, 90, 7)
    a = rng.standard_normal((90, 90))
    l = orc.cholesky_lower(a @ a.T + 90 * np.eye(90))
    jk = DfJK(b, precision="f64", metric_chol=l)
    jh, kh = jk.jk_from_occ(c)
    jd, kd = jk.jk_from_occ(torch.from_numpy(c).cuda())
    assert np.array_equal(jh, jd.cpu().numpy()) and np.array_equal(kh, kd.cpu().numpy())
    assert np.abs(jh - orc.df_j_square(b, d, metric_chol=l)).max() < F_TOL
    assert np.abs(jh - jk.j(d)).max() <= 1e-12 * np.abs(jh).max()
    jk.close()


def test_fused_jk_empty_channel(fc):
    from ferric_b200.dfjk import DfJK
    b, c, d = synthetic.dfjk_inputs(20, 30, 3)
    jk = DfJK(b)
    j, k = jk.jk_from_occ(np.zeros((20, 0)))
    assert not j.any() and not k.any()

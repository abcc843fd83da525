"""Oracle self-tests (CPU): the reference's structural known-answer tests,
restated against the NumPy restatement of the path."""
import numpy as np
import pytest

from oracle import dfjk, rimp2, synthetic


@pytest.fixture(scope="module")
def small():
    b, eo, ev = synthetic.rimp2_inputs(96, 5, 23)
    return b, eo, ev


def test_symmetry_loop_matches_naive_double_loop(small):
    # spin_components_symmetry_matches_naive_double_loop (ferric-mp2/src/rimp2.rs:3107)
    b, eo, ev = small
    eps = np.concatenate([eo, ev])
    fast = rimp2.spin_components(b, eps, 5, 23)
    naive = rimp2.spin_components_full_loop(b, eo, ev)
    assert np.allclose(fast, naive, rtol=0, atol=1e-15)


def test_first_occ_and_nocc_total_indexing(small):
    # eps indexed first_occ + i and nocc_total + a (rimp2.rs:1399-1441): frozen core
    b, eo, ev = small
    eps = np.concatenate([[-50.0, -40.0], eo, [0.01], ev])  # 2 frozen, 1 inactive
    # nocc_total counts every occupied; the virtual block starts after it
    eps2 = np.concatenate([[-50.0, -40.0], eo, ev])
    got = rimp2.spin_components(b, eps2, 5, 23, first_occ=2, nocc_total=7)
    ref = rimp2.spin_components(b, np.concatenate([eo, ev]), 5, 23)
    assert got == ref
    assert eps.shape[0] == 31


def test_kappa_limit_is_plain(small):
    b, eo, ev = small
    eps = np.concatenate([eo, ev])
    plain = rimp2.spin_components(b, eps, 5, 23)
    damped = rimp2.spin_components(b, eps, 5, 23, kappa=1e6)
    assert np.allclose(plain, damped, rtol=1e-14)
    weak = rimp2.spin_components(b, eps, 5, 23, kappa=0.5)
    assert abs(weak[2]) < abs(plain[2])


def test_x_ov_gemm_matches_scalar_definition(small):
    # x_ov_gemm_matches_the_scalar_definition (ferric-mp2/src/zvector.rs:1135)
    b, eo, ev = small
    nocc, nvir = len(eo), len(ev)
    t2, _ = rimp2.t2_and_integrals(b, eo, ev)
    x = rimp2.x_ov_from_t2(t2, b, nocc, nvir)
    t = t2.reshape(nocc, nvir, nocc, nvir)
    p, i, a = 3, 2, 7
    ref = 0.0
    for j in range(nocc):
        for bb in range(nvir):
            ref += (2 * t[i, a, j, bb] - t[i, bb, j, a]) * b[p, j * nvir + bb]
    assert abs(x[p, i * nvir + a] - ref) < 1e-16 + 1e-13 * abs(ref)


def test_mp2_density_matches_scalar_definition(small):
    # mp2_density_gemm_matches_the_scalar_definition (ferric-mp2/src/oo_rimp2.rs:2042)
    b, eo, ev = small
    nocc, nvir = len(eo), len(ev)
    t2, _ = rimp2.t2_and_integrals(b, eo, ev)
    p_oo, p_vv = rimp2.mp2_density(t2, nocc, nvir)
    t = t2.reshape(nocc, nvir, nocc, nvir)
    i, j = 1, 3
    ref = 0.0
    for k in range(nocc):
        for a in range(nvir):
            for c in range(nvir):
                ref -= t[i, a, k, c] * (2 * t[j, a, k, c] - t[j, c, k, a])
    assert abs(p_oo[i, j] - ref) < 1e-13 * max(1.0, abs(ref))
    a, c = 4, 9
    ref = 0.0
    for i in range(nocc):
        for j in range(nocc):
            for d in range(nvir):
                ref += t[i, a, j, d] * (2 * t[i, c, j, d] - t[i, d, j, c])
    assert abs(p_vv[a, c] - ref) < 1e-13 * max(1.0, abs(ref))


def test_recompute_route_matches_stored_amplitudes(small):
    b, eo, ev = small
    r1 = rimp2.energy_gamma_deps(b, eo, ev)
    r2 = rimp2.energy_gamma_deps_small(b, eo, ev)
    assert abs(r1[0] - r2[0]) < 1e-15 and abs(r1[1] - r2[1]) < 1e-15
    for u, v in zip(r1[2:], r2[2:]):
        assert np.abs(u - v).max() < 1e-15


def test_gamma_and_deps_match_central_differences(small):
    b, eo, ev = small
    eps = np.concatenate([eo, ev])
    _, _, gamma, d_o, d_v = rimp2.energy_gamma_deps(b, eo, ev)
    h = 1e-5
    rows, cols = synthetic.fd_entries(b.shape[0], b.shape[1], count=8)
    for p, ia in zip(rows, cols):
        bp = b.copy(); bp[p, ia] += h
        bm = b.copy(); bm[p, ia] -= h
        fd = (rimp2.spin_components(bp, eps, 5, 23)[2] - rimp2.spin_components(bm, eps, 5, 23)[2]) / (2 * h)
        assert abs(fd - gamma[p, ia]) < 1e-9 * max(1.0, abs(gamma[p, ia])) + 1e-11
    for k in (0, 3, 5 + 2, 5 + 20):
        ep = eps.copy(); ep[k] += h
        em = eps.copy(); em[k] -= h
        fd = (rimp2.spin_components(b, ep, 5, 23)[2] - rimp2.spin_components(b, em, 5, 23)[2]) / (2 * h)
        an = d_o[k] if k < 5 else d_v[k - 5]
        assert abs(fd - an) < 1e-9 * max(1.0, abs(an)) + 1e-12


def test_df_k_occ_matches_density_build():
    # df_k_build_from_occ_matches_density_build (ferric-scf/src/df_k.rs:2471)
    b, c, d = synthetic.dfjk_inputs(30, 50, 6)
    assert np.abs(dfjk.df_k_occ(b, c) - dfjk.df_k_density(b, d)).max() < 1e-14


def test_df_j_packed_matches_square_and_naive():
    # df_j_chunked_matches_naive_contraction (ferric-scf/src/df_j.rs:1836)
    b, c, d = synthetic.dfjk_inputs(24, 40, 5)
    jp = dfjk.df_j_packed(dfjk.pack_lower(b), d)
    js = dfjk.df_j_square(b, d)
    naive = np.einsum("qmn,qls,ls->mn", b, b, d)
    assert np.abs(jp - js).max() < 1e-14
    assert np.abs(js - naive).max() < 1e-14


def test_df_j_metric_solve_equals_dressed():
    rng = np.random.default_rng(5)
    b, c, d = synthetic.dfjk_inputs(20, 30, 4)
    a = rng.standard_normal((30, 30))
    v = a @ a.T + 30 * np.eye(30)
    l = dfjk.cholesky_lower(v)
    raw = np.einsum("pq,qmn->pmn", l, b)           # (P|mn) = L B
    j_raw = dfjk.df_j_packed(dfjk.pack_lower(raw), d, metric_chol=l)
    j_dressed = dfjk.df_j_square(b, d)
    assert np.abs(j_raw - j_dressed).max() < 1e-12


def test_density_weights_nonsymmetric():
    rng = np.random.default_rng(1)
    d = rng.standard_normal((7, 7))
    w = dfjk.packed_density_weights(d)
    b = rng.standard_normal((7, 7)); b = b + b.T
    assert abs(np.sum(b * d) - np.dot(dfjk.pack_lower(b[None])[0], w)) < 1e-13


def test_ump2_oracle_closed_shell_identities():
    """u_rimp2.rs's same/opposite-spin sums at alpha = beta reproduce the
    closed-shell E_SS / 2 and E_OS (rimp2.rs:1399-1544)."""
    from oracle import rimp2 as orc
    from oracle import synthetic
    b, eo, ev = synthetic.rimp2_inputs(60, 4, 11)
    e_os, e_ss, _ = orc.spin_components(b, np.concatenate([eo, ev]), 4, 11)
    assert abs(2 * orc.u_same_spin(b, eo, ev) - e_ss) < 1e-14 * abs(e_ss) + 1e-18
    assert abs(orc.u_opposite_spin(b, eo, ev, b, eo, ev) - e_os) < 1e-13 * abs(e_os)


def test_ump2_fixtures_pinned_to_golden():
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    for name in ("oh_ump2", "nh2_ump2"):
        d = np.load(os.path.join(here, "golden", name + ".npz"))
        assert abs(float(d["oracle_e_uhf"]) - float(d["golden_e_uhf"])) < 1e-9
        for k in ("e_aa", "e_bb", "e_ab"):
            assert abs(float(d["oracle_" + k]) - float(d["golden_" + k])) < 1e-9


def test_imat_gemm_matches_scalar_definition():
    """zvector.rs:1245-1290 restated: the GEMM form of Imat equals its scalar
    definition within (n_max + 2) eps of the absolute sums, frozen-core
    columns zero."""
    from oracle import rimp2 as orc
    naux, nocc, nvir, fo = 9, 4, 7, 2
    nmo = fo + nocc + nvir
    rng = np.random.default_rng(0x9E37)
    x = rng.uniform(-1, 1, (naux, nocc * nvir))
    bf = rng.uniform(-1, 1, (naux, nmo, nmo))
    got = orc.imat_ri(x, bf, nocc, nvir, fo)
    want, absum = orc.imat_scalar(x, bf, nocc, nvir, fo)
    bar = (naux * max(nocc, nvir) + 2.0) * np.finfo(float).eps
    assert np.all(np.abs(got - want) <= bar * absum)
    assert np.all(got[:, :fo] == 0.0)
    assert np.any(got != 0.0)


def test_response_restatement_matches_scalar_definition():
    """The oracle's 3c/2c response (gradient.rs:559-887) against the
    definitions written as einsums: y = V^T x, gamma_2c = -w (V^T b) y^T,
    g3c[P] = w (G_P + G_P^T), G_P[mu, nu] = sum_ia C_occ[mu, i] Y[P, ia] C_vir[nu, a]."""
    from oracle import rimp2 as orc
    rng = np.random.default_rng(3)
    naux, nocc, nvir, nbf = 11, 3, 4, 6
    x, b = rng.standard_normal((2, naux, nocc * nvir))
    v = rng.standard_normal((naux, naux))
    co, cv = rng.standard_normal((nbf, nocc)), rng.standard_normal((nbf, nvir))
    y, g2 = orc.response_2c(x, b, v, 1.5)
    assert np.allclose(y, np.einsum("qp,qk->pk", v, x), rtol=1e-13, atol=1e-13)
    assert np.allclose(g2, -1.5 * np.einsum("qp,qk,rk->pr", v, b, y), rtol=1e-12, atol=1e-12)
    g3 = orc.response_3c(y, co, cv, 2, 5, 1.5)
    gp = np.einsum("mi,pia,na->pmn", co, y[2:7].reshape(5, nocc, nvir), cv)
    assert np.allclose(g3, 1.5 * (gp + gp.transpose(0, 2, 1)), rtol=1e-12, atol=1e-12)

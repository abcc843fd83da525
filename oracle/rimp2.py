"""FP64 restatement of the reference's closed-shell RI-MP2 path (oracle only).

Layout conventions follow the reference exactly:

* ``b_ov`` is row-major ``(naux, nocc*nvir)`` with column ``i*nvir + a``
  (ferric-mp2/src/rimp2.rs:1445-1499);
* ``eps`` is the full MO-energy vector, indexed ``first_occ + i`` for an
  active occupied orbital and ``nocc_total + a`` for a virtual
  (ferric-mp2/src/rimp2.rs:1399-1441).

Energies
    ``E_OS = sum_ij sum_ab g_ab^2 / D``,
    ``E_SS = sum_ij sum_ab g_ab (g_ab - g_ba) / D``, ``g_ab = (ia|jb)``,
    ``D = e_i + e_j - e_a - e_b``, over unique pairs ``j >= i`` with weight 1
    on the diagonal and 2 off it; per-i partials summed serially in ascending
    i (rimp2.rs:1506-1544).  Optional kappa damping ``(1 - exp(kappa*D))^2``
    on both components (rimp2.rs:1425-1437).

Adjoint
    ``Gamma[P, ia] = dE/dB[P, ia] = 4 x_ov[P, ia]`` (rimp2.rs:1832-1836) with
    ``x_ov[P, ia] = sum_jb Tt_ij^ab B[P, jb]`` and ``Tt = 2t - tbar``
    (zvector.rs:651-703); ``dE/d eps_p = 2 P_pp`` (rimp2.rs:1835-1836) with
    the unrelaxed densities of oo_rimp2.rs:1170-1300.
"""
from __future__ import annotations

import numpy as np


def _pair_terms(g, e_ij, eps_vir, kappa):
    """(e_os_ij, e_ss_ij) of one pair block ``g[a, b] = (ia|jb)``.

    Restates ``pair_energy`` (ferric-mp2/src/rimp2.rs:1399-1441).
    """
    denom = e_ij - eps_vir[:, None] - eps_vir[None, :]
    if kappa is None:
        w = 1.0 / denom
    else:
        d1 = 1.0 - np.exp(kappa * denom)
        w = d1 * d1 / denom
    e_os = float(np.sum(g * g * w))
    e_ss = float(np.sum(g * (g - g.T) * w))
    return e_os, e_ss


def spin_components(b_ov, eps, nocc, nvir, first_occ=0, nocc_total=None, kappa=None):
    """Closed-shell RI-MP2 ``(e_os, e_ss, e_total)``.

    Restates ``spin_components_from_b_ov_kappa_cpu`` and
    ``spin_components_from_blocks`` (ferric-mp2/src/rimp2.rs:1445-1544):
    one wide product ``G_i = B_i^T B_{j>=i}`` per occupied ``i``, the pair
    loop over ``j >= i`` with weight 1 (i == j) or 2, and an ascending-i
    serial sum of the per-i partials.
    """
    b_ov = np.ascontiguousarray(b_ov, dtype=np.float64)
    eps = np.asarray(eps, dtype=np.float64)
    if nocc_total is None:
        nocc_total = first_occ + nocc
    eps_vir = eps[nocc_total:nocc_total + nvir]
    partials = []
    for i in range(nocc):
        b_i = b_ov[:, i * nvir:(i + 1) * nvir]
        g_i = b_i.T @ b_ov[:, i * nvir:]
        e_os_i = e_ss_i = 0.0
        for j in range(i, nocc):
            fac = 1.0 if i == j else 2.0
            jcol = (j - i) * nvir
            g = g_i[:, jcol:jcol + nvir]
            e_ij = eps[first_occ + i] + eps[first_occ + j]
            eo, es = _pair_terms(g, e_ij, eps_vir, kappa)
            e_os_i += fac * eo
            e_ss_i += fac * es
        partials.append((e_os_i, e_ss_i))
    e_os = 0.0
    e_ss = 0.0
    for eo, es in partials:
        e_os += eo
        e_ss += es
    return e_os, e_ss, e_os + e_ss


def spin_components_full_loop(b_ov, eps_occ, eps_vir, kappa=None):
    """Every ordered pair (i, j), no symmetry weights: the naive cross-check
    the reference keeps beside the fast loop
    (ferric-mp2/src/rimp2.rs:984-1018 and the test at rimp2.rs:3107)."""
    nocc, nvir = len(eps_occ), len(eps_vir)
    e_os = e_ss = 0.0
    for i in range(nocc):
        for j in range(nocc):
            g = b_ov[:, i * nvir:(i + 1) * nvir].T @ b_ov[:, j * nvir:(j + 1) * nvir]
            eo, es = _pair_terms(g, eps_occ[i] + eps_occ[j], eps_vir, kappa)
            e_os += eo
            e_ss += es
    return e_os, e_ss, e_os + e_ss


def t2_and_integrals(b_ov, eps_occ, eps_vir):
    """``(t2, eri_ov)`` flat ``nov x nov``: ``eri = B^T B`` and ``t2 = eri / D``.

    Restates ``compute_t2_and_integrals`` (ferric-mp2/src/oo_rimp2.rs:1079-1123).
    Small cases only (it stores ``nov^2`` doubles twice).
    """
    nocc, nvir = len(eps_occ), len(eps_vir)
    eri = b_ov.T @ b_ov
    e_ov = (eps_occ[:, None] - eps_vir[None, :]).reshape(-1)   # e_i - e_a at ia
    denom = e_ov[:, None] + e_ov[None, :]
    return eri / denom, eri


def mp2_density(t2, nocc, nvir):
    """Unrelaxed ``(P_oo, P_vv)`` from flat amplitudes ``t2[ia, jb]``.

    Restates ``build_mp2_density`` (ferric-mp2/src/oo_rimp2.rs:1170-1300):
    ``P_ij = -sum_kab t_ik^ab (2 t_jk^ab - t_jk^ba)``,
    ``P_ab =  sum_ijc t_ij^ac (2 t_ij^bc - t_ij^cb)``.
    """
    t = np.asarray(t2).reshape(nocc, nvir, nocc, nvir)          # t[i,a,j,b]
    tt = 2.0 * t - t.transpose(0, 3, 2, 1)                       # 2t - tbar
    p_oo = -np.einsum("iakb,jakb->ij", t, tt, optimize=True)
    p_vv = np.einsum("iajc,ibjc->ab", t, tt, optimize=True)
    return p_oo, p_vv


def x_ov_from_t2(t2, b_ov, nocc, nvir):
    """``x_ov[P, ia] = sum_jb (2t - tbar)_ij^ab B[P, jb]``.

    Restates ``build_x_ov_weighted`` / ``tt_block`` at MP2 weights (d, e) =
    (2, 1) (ferric-mp2/src/zvector.rs:651-703).
    """
    nov = nocc * nvir
    t = np.asarray(t2).reshape(nocc, nvir, nocc, nvir)
    tt = (2.0 * t - t.transpose(0, 3, 2, 1)).reshape(nov, nov)
    return b_ov @ tt.T


def energy_gamma_deps_small(b_ov, eps_occ, eps_vir):
    """E, Gamma and dE/deps through the stored-amplitude route the reference
    takes (t2 -> P, x_ov).  Small cases only.

    Returns ``(e_os, e_ss, gamma, de_docc, de_dvir)``.
    """
    nocc, nvir = len(eps_occ), len(eps_vir)
    t2, eri = t2_and_integrals(b_ov, eps_occ, eps_vir)
    tt = (2.0 * t2.reshape(nocc, nvir, nocc, nvir)
          - t2.reshape(nocc, nvir, nocc, nvir).transpose(0, 3, 2, 1)).reshape(t2.shape)
    e_os = float(np.sum(eri * t2))
    e_ss = float(np.sum(eri * (t2 - t2.reshape(nocc, nvir, nocc, nvir)
                                  .transpose(0, 3, 2, 1).reshape(t2.shape))))
    gamma = 4.0 * x_ov_from_t2(t2, b_ov, nocc, nvir)
    p_oo, p_vv = mp2_density(t2, nocc, nvir)
    del tt
    return e_os, e_ss, gamma, 2.0 * np.diag(p_oo).copy(), 2.0 * np.diag(p_vv).copy()


def energy_gamma_deps_pairs(b_ov, eps_occ, eps_vir, pairs):
    """The contributions of a set of unordered occupied pairs (i <= j) to E,
    Gamma and dE/deps: each pair stands for its orderings (i, j) and (j, i),
    computed with the per-ordered-pair terms of ``energy_gamma_deps``
    (zvector.rs:651-703, oo_rimp2.rs:1170-1191).  The sums over a partition of
    all pairs equal ``energy_gamma_deps``.  Small cases only.

    Returns ``(e_os, e_ss, gamma, de_docc, de_dvir)``.
    """
    b_ov = np.ascontiguousarray(b_ov, dtype=np.float64)
    eps_occ = np.asarray(eps_occ, dtype=np.float64)
    eps_vir = np.asarray(eps_vir, dtype=np.float64)
    naux = b_ov.shape[0]
    nocc, nvir = len(eps_occ), len(eps_vir)
    gamma = np.zeros((naux, nocc * nvir))
    de_docc = np.zeros(nocc)
    de_dvir = np.zeros(nvir)
    e_os = e_ss = 0.0
    for i0, j0 in pairs:
        for i, j in ((i0, j0), (j0, i0)) if i0 != j0 else ((i0, j0),):
            bi, bj = b_ov[:, i * nvir:(i + 1) * nvir], b_ov[:, j * nvir:(j + 1) * nvir]
            g = bi.T @ bj                                          # (ia|jb)
            denom = eps_occ[i] + eps_occ[j] - eps_vir[:, None] - eps_vir[None, :]
            t = g / denom
            tt = (2.0 * g - g.T) / denom
            e_os += float(np.sum(g * t))
            e_ss += float(np.sum(g * (g - g.T) / denom))
            c = t * tt
            de_docc[i] += -2.0 * float(np.sum(c))
            de_dvir += 2.0 * np.sum(c, axis=1)
            gamma[:, i * nvir:(i + 1) * nvir] += 4.0 * (bj @ tt.T)
    return e_os, e_ss, gamma, de_docc, de_dvir


def energy_gamma_deps(b_ov, eps_occ, eps_vir, occ=None):
    """E, Gamma = dE/dB and dE/deps without storing ``t2``.

    The amplitudes of one occupied ``i`` are recomputed from
    ``G_i = B_i^T B`` (``nvir x nov``), turned into ``Tt_i = (2 G_i - G_i^swap)/D``
    and contracted at once: ``x_i = B Tt_i^T`` -- the per-i GEMM of
    ``build_x_ov_weighted`` (zvector.rs:651-703) with ``tt_block`` built from
    the recomputed block instead of the stored ``t2``.  The densities'
    diagonals follow ``P_ii = -sum_jab t_ij^ab Tt_ij^ab`` and
    ``P_aa = sum_ijb t_ij^ab Tt_ij^ab`` (oo_rimp2.rs:1170-1191).

    ``occ`` restricts the loop to a subset of occupied ``i`` (a bounded
    sample: the energies, Gamma columns and dE/deps then hold only those
    rows' contributions).

    Returns ``(e_os, e_ss, gamma, de_docc, de_dvir)``.
    """
    b_ov = np.ascontiguousarray(b_ov, dtype=np.float64)
    eps_occ = np.asarray(eps_occ, dtype=np.float64)
    eps_vir = np.asarray(eps_vir, dtype=np.float64)
    naux = b_ov.shape[0]
    nocc, nvir = len(eps_occ), len(eps_vir)
    nov = nocc * nvir
    gamma = np.zeros((naux, nov))
    de_docc = np.zeros(nocc)
    de_dvir = np.zeros(nvir)
    e_os = e_ss = 0.0
    for i in (range(nocc) if occ is None else occ):
        g = (b_ov[:, i * nvir:(i + 1) * nvir].T @ b_ov).reshape(nvir, nocc, nvir)  # g[a,j,b]
        gs = g.transpose(2, 1, 0)                                                # g[b,j,a] at [a,j,b]
        denom = (eps_occ[i] + eps_occ[None, :, None]
                 - eps_vir[:, None, None] - eps_vir[None, None, :])
        t = g / denom
        tt = (2.0 * g - gs) / denom
        e_os += float(np.sum(g * t))
        e_ss += float(np.sum(g * (g - gs) / denom))
        c = t * tt                                 # t_ij^ab Tt_ij^ab
        de_docc[i] += -2.0 * float(np.sum(c))
        de_dvir += 2.0 * np.sum(c, axis=(1, 2))
        gamma[:, i * nvir:(i + 1) * nvir] = 4.0 * (b_ov @ tt.reshape(nvir, nov).T)
    return e_os, e_ss, gamma, de_docc, de_dvir


def stream_dressed_mo(t3, m, c_left, c_right, chunk=256):
    """B[P, l*nr + r] = sum_Q M[P, Q] (Q|lr), (Q|lr) = C_left^T (Q|mu nu) C_right,
    streamed over aux chunks with an accumulating GEMM into B
    (stream_dressed_mo_band_budgeted, ferric-mp2/src/rimp2.rs:665-737:
    occupied-side contraction first, then the right index, then
    ``b += V^-1/2[:, chunk] . mo_blk``)."""
    naux = t3.shape[0]
    nl, nr = c_left.shape[1], c_right.shape[1]
    b = np.zeros((naux, nl * nr))
    for q0 in range(0, naux, chunk):
        q1 = min(naux, q0 + chunk)
        half = np.einsum("ml,qmn->qln", c_left, t3[q0:q1], optimize=True)   # (qc, nl, nao)
        mo = np.einsum("qln,nr->qlr", half, c_right, optimize=True).reshape(q1 - q0, nl * nr)
        b += m[:, q0:q1] @ mo
    return b


def u_same_spin(b_ov, eps_occ, eps_vir):
    """Same-spin (alpha-alpha or beta-beta) RI-MP2 energy of one spin channel:
    0.25 * sum_i sum_{j>=i} fac_ij sum_ab (g_ab - g_ba)^2 / D, fac 1 on i == j
    and 2 off (same_spin_block_energy, ferric-mp2/src/u_rimp2.rs:693-724)."""
    nocc, nvir = len(eps_occ), len(eps_vir)
    e = 0.0
    for i in range(nocc):
        bi = b_ov[:, i * nvir:(i + 1) * nvir]
        for j in range(i, nocc):
            g = bi.T @ b_ov[:, j * nvir:(j + 1) * nvir]          # (ia|jb)
            k = g - g.T
            d = eps_occ[i] + eps_occ[j] - eps_vir[:, None] - eps_vir[None, :]
            e += (1.0 if i == j else 2.0) * np.sum(k * k / d)
    return 0.25 * e


def u_opposite_spin(b_a, eps_occ_a, eps_vir_a, b_b, eps_occ_b, eps_vir_b):
    """Opposite-spin (alpha-beta) RI-MP2 energy: sum_{i a J B} (ia|JB)^2 / D
    (opposite_spin_block_energy, ferric-mp2/src/u_rimp2.rs:731-753)."""
    noa, nva = len(eps_occ_a), len(eps_vir_a)
    nob, nvb = len(eps_occ_b), len(eps_vir_b)
    e = 0.0
    for i in range(noa):
        g = b_a[:, i * nva:(i + 1) * nva].T @ b_b                      # (nva, nob*nvb)
        d = (eps_occ_a[i] + np.repeat(eps_occ_b, nvb)[None, :]
             - eps_vir_a[:, None] - np.tile(eps_vir_b, nob)[None, :])
        e += np.sum(g * g / d)
    return e


def imat_ri(x_ov, b_full, nocc, nvir, first_occ=0):
    """RI Lagrangian Imat (build_imat_ri / imat_fill_rows,
    ferric-mp2/src/zvector.rs:735-832): for every MO row q,
    Imat[q, first_occ + i] = -2 sum_{P,a} x_ov[P, i*nvir + a] b_full[P, q, nocc_total + a],
    Imat[q, nocc_total + a] = -2 sum_{P,i} x_ov[P, i*nvir + a] b_full[P, q, first_occ + i];
    frozen-core columns stay zero."""
    naux, nmo = b_full.shape[0], b_full.shape[1]
    nt = first_occ + nocc
    x = x_ov.reshape(naux, nocc, nvir)
    imat = np.zeros((nmo, nmo))
    imat[:, first_occ:nt] = -2.0 * np.einsum("pqa,pia->qi", b_full[:, :, nt:nt + nvir], x, optimize=True)
    imat[:, nt:nt + nvir] = -2.0 * np.einsum("pqi,pia->qa", b_full[:, :, first_occ:nt], x, optimize=True)
    return imat


def imat_scalar(x_ov, b_full, nocc, nvir, first_occ=0):
    """The scalar definition of Imat and the sum of |terms| per element (the
    reference's known-answer test, zvector.rs:1245-1290)."""
    naux, nmo = b_full.shape[0], b_full.shape[1]
    nt = first_occ + nocc
    want = np.zeros((nmo, nmo))
    absum = np.zeros((nmo, nmo))
    for q in range(nmo):
        for i in range(nocc):
            for p in range(naux):
                for a in range(nvir):
                    t = x_ov[p, i * nvir + a] * b_full[p, q, nt + a]
                    want[q, first_occ + i] -= 2.0 * t
                    absum[q, first_occ + i] += 2.0 * abs(t)
                    t2 = x_ov[p, i * nvir + a] * b_full[p, q, first_occ + i]
                    want[q, nt + a] -= 2.0 * t2
                    absum[q, nt + a] += 2.0 * abs(t2)
    return want, absum


def response_2c(x_ov, b_ov, v_inv_sqrt, weight=2.0):
    """``(y_ov, gamma_2c)`` of one response channel: ``y_ov = V^{-1/2 T}
    x_ov`` (ferric-mp2/src/gradient.rs:656-658) and ``gamma_2c = -w C_fit
    y_ov^T`` with ``C_fit = V^{-1/2 T} b_ov`` (gradient.rs:881-887)."""
    y = v_inv_sqrt.T @ x_ov
    c_fit = v_inv_sqrt.T @ b_ov
    return y, -weight * (c_fit @ y.T)


def response_3c(y_ov, c_occ, c_vir, p0, np_, weight=2.0):
    """The 3-centre weight of aux rows ``[p0, p0 + np_)``: ``w (G_P + G_P^T)``,
    ``G_P = C_occ Y_P C_vir^T`` with ``Y_P`` row P of y_ov as (nocc, nvir)
    (ferric-mp2/src/gradient.rs:772-804)."""
    nocc, nvir = c_occ.shape[1], c_vir.shape[1]
    out = np.empty((np_, c_occ.shape[0], c_occ.shape[0]))
    for k in range(np_):
        g = c_occ @ y_ov[p0 + k].reshape(nocc, nvir) @ c_vir.T
        out[k] = weight * (g + g.T)
    return out

"""FP64 restatement of the reference's DF-J and DF-K builders (oracle only).

DF-J (ferric-scf/src/df_j.rs:1-31, 1134-1245, 1459-1572)
    ``w`` = packed density weights (diagonal ``D_mm``, off-diagonal
    ``D_mn + D_nm``, lower triangle ``(mu, nu <= mu)`` row-major);
    pass 1 ``d_P = sum_k Bp[P, k] w_k``; metric solve ``c = V^-1 d`` by the
    Cholesky factor (df_j.rs:931); pass 2 ``J_k = sum_P Bp[P, k] c_P``;
    unpack symmetric (df_j.rs:1176).  With a dressed ``B = L^-1 (P|mn)`` the
    metric is the identity and ``J = B^T (B . D)``.

DF-K (ferric-scf/src/df_k.rs:1409-1520, 1575-1660)
    occupied path ``M_Q = B_Q C_occ`` (n x nocc), ``K = sum_Q M_Q M_Q^T``;
    no occupation factor is applied (ferric-scf/src/fock.rs:29-45).  The
    density path ``K = sum_Q B_Q D B_Q^T`` (df_k.rs:1531-1562) is the
    cross-check the reference's test ``df_k_build_from_occ_matches_density_build``
    (df_k.rs:2471) uses.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg


def packed_density_weights(d):
    """``packed_density_weights`` (ferric-scf/src/df_j.rs:1134-1150)."""
    d = np.asarray(d, dtype=np.float64)
    n = d.shape[0]
    il, jl = np.tril_indices(n)
    w = d[il, jl] + d[jl, il]
    diag = il == jl
    w[diag] = d[il[diag], il[diag]]
    return w


def pack_lower(b_square):
    """(naux, n, n) symmetric -> (naux, n(n+1)/2) packed lower rows, the
    ``(mu, nu <= mu)`` order of ferric's packed tier."""
    n = b_square.shape[1]
    il, jl = np.tril_indices(n)
    return np.ascontiguousarray(b_square[:, il, jl])


def unpack_symmetric(packed, n):
    """``unpack_symmetric`` (ferric-scf/src/df_j.rs:1166-1180)."""
    j = np.zeros((n, n))
    il, jl = np.tril_indices(n)
    j[il, jl] = packed
    j[jl, il] = packed
    return j


def df_j_packed(bp, d, metric_chol=None):
    """Two-pass packed DF-J (``DfJ::build_packed``, df_j.rs:1199-1245).

    ``bp``: (naux, n(n+1)/2) packed raw ``(P|mn)`` rows.  ``metric_chol``:
    lower Cholesky factor ``L`` of ``V = L L^T`` or None for a dressed tensor.
    """
    d = np.asarray(d, dtype=np.float64)
    n = d.shape[0]
    w = packed_density_weights(d)
    d_p = bp @ w
    if metric_chol is not None:
        c_p = scipy.linalg.cho_solve((metric_chol, True), d_p)
    else:
        c_p = d_p
    acc = bp.T @ c_p
    return unpack_symmetric(acc, n)


def df_j_square(b, d, metric_chol=None):
    """Unpacked two-pass DF-J over the square tensor (df_j.rs:1511-1565)."""
    naux, n, _ = b.shape
    flat = b.reshape(naux, n * n)
    d_p = flat @ np.asarray(d, dtype=np.float64).reshape(-1)
    c_p = d_p if metric_chol is None else scipy.linalg.cho_solve((metric_chol, True), d_p)
    return (flat.T @ c_p).reshape(n, n)


def df_k_occ(b, c_occ):
    """Occupied-path DF-K (``occ_chunk_k`` / ``occ_half_panel``,
    df_k.rs:1575-1660): ``K = sum_Q (B_Q C)(B_Q C)^T``."""
    naux, n, _ = b.shape
    c_occ = np.asarray(c_occ, dtype=np.float64)
    m = (b.reshape(naux * n, n) @ c_occ).reshape(naux, n, -1)        # M_Q
    w = m.transpose(1, 0, 2).reshape(n, -1)                          # [mu, (Q,i)]
    k = w @ w.T
    return 0.5 * (k + k.T)


def df_k_density(b, d):
    """Density-path DF-K (``density_chunk_k``, df_k.rs:1531-1562):
    ``K = sum_Q B_Q D B_Q^T``."""
    k = np.zeros((b.shape[1], b.shape[1]))
    for q in range(b.shape[0]):
        k += b[q] @ d @ b[q].T
    return k


def cholesky_lower(v):
    """Lower Cholesky factor of the Coulomb metric (the factor ``DfJ`` stores,
    df_j.rs:931); FP64, once per geometry."""
    return np.linalg.cholesky(np.asarray(v, dtype=np.float64))


def cholesky_inverse_lower(v):
    """``L^-1`` with ``V = L L^T`` (``cholesky_inverse_lower``,
    ferric-core/src/linalg.rs:495; used as the metric dressing of
    ``cholesky_inverse_sqrt``, ferric-mp2/src/rimp2.rs:2478-2489)."""
    l = cholesky_lower(v)
    return scipy.linalg.solve_triangular(l, np.eye(l.shape[0]), lower=True)

"""Closed-shell RHF and the dressed 3-index tensors for the oracle's golden pin
(test infrastructure only).

RHF with exact J/K (the reference JSONs were made with PySCF ``scf.RHF``,
exact J/K, conv_tol 1e-12; see testdata/reference/validation/sos_mp2/h2o_cc-pvdz.json
provenance) or with a dressed DF tensor (``F = H + J - K/2``, ``K(D) = 2 K(C_occ)``,
ferric-scf/src/rhf.rs:3040-3090, 3164-3178).  DIIS on the commutator FDS - SDF.
Then the RI-MP2 inputs: metric V = (P|Q) = L L^T, B = L^-1 (P|mn)
(ferric-mp2/src/rimp2.rs:2478-2489, 666-756), B_ov = C_occ^T B C_vir.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg

from . import integrals


def nuclear_repulsion(charges, coords):
    e = 0.0
    for a in range(len(charges)):
        for b in range(a):
            e += charges[a] * charges[b] / np.linalg.norm(np.asarray(coords[a]) - np.asarray(coords[b]))
    return e


def rhf(S, H, nocc, e_nuc, jk, tol=1e-12, max_iter=200):
    """jk(D) -> (J, K) for a symmetric density D.  Returns (E, eps, C)."""
    s, u = np.linalg.eigh(S)
    X = u / np.sqrt(s)                       # canonical orthogonaliser
    e, c = np.linalg.eigh(X.T @ H @ X)
    C = X @ c
    focks, errs = [], []
    e_old = 0.0
    for it in range(max_iter):
        Co = C[:, :nocc]
        D = 2.0 * Co @ Co.T
        J, K = jk(D)
        F = H + J - 0.5 * K
        E = 0.5 * np.sum(D * (H + F)) + e_nuc
        err = F @ D @ S - S @ D @ F
        focks.append(F)
        errs.append(X.T @ err @ X)
        if len(focks) > 8:
            focks.pop(0)
            errs.pop(0)
        if np.abs(errs[-1]).max() < tol * 100 and abs(E - e_old) < tol:
            break
        e_old = E
        m = len(focks)
        Bm = -np.ones((m + 1, m + 1))
        Bm[m, m] = 0.0
        for a in range(m):
            for b in range(m):
                Bm[a, b] = np.sum(errs[a] * errs[b])
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        coef = np.linalg.lstsq(Bm, rhs, rcond=None)[0][:m]
        Fd = sum(cf * f for cf, f in zip(coef, focks))
        eps, c = np.linalg.eigh(X.T @ Fd @ X)
        C = X @ c
    # final canonical orbitals of the converged Fock matrix
    eps, c = np.linalg.eigh(X.T @ F @ X)
    C = X @ c
    return E, eps, C


def exact_jk(eri):
    def jk(D):
        return np.einsum("mnls,ls->mn", eri, D, optimize=True), np.einsum("mlns,ls->mn", eri, D, optimize=True)
    return jk


def df_jk(b):
    """J, K from a dressed tensor b (naux, n, n): J = B^T (B.D), K = sum_Q B_Q D B_Q."""
    def jk(D):
        d = np.einsum("qmn,mn->q", b, D)
        J = np.einsum("qmn,q->mn", b, d)
        K = np.einsum("qml,ls,qns->mn", b, D, b, optimize=True)
        return J, K
    return jk


def dressed(aux, shells):
    """B = L^-1 (P|mn) with V = (P|Q) = L L^T."""
    v = integrals.eri2(aux)
    l = np.linalg.cholesky(v)
    t3 = integrals.eri3(aux, shells)
    b = scipy.linalg.solve_triangular(l, t3.reshape(t3.shape[0], -1), lower=True)
    return b.reshape(t3.shape), v, t3


def b_ov(b, C, nocc):
    co, cv = C[:, :nocc], C[:, nocc:]
    return np.einsum("qmn,mi,na->qia", b, co, cv, optimize=True).reshape(b.shape[0], -1)


def uhf(S, H, na, nb, e_nuc, eri, tol=1e-11, max_iter=300, guess=None):
    """Unrestricted HF with exact J/K and DIIS on both spins' commutators
    (F_s = H + J(D_a + D_b) - K(D_s)); returns (E, (eps_a, eps_b), (C_a, C_b)).
    The reference's UMP2 goldens were made with PySCF scf.UHF at conv_tol
    1e-11 (testdata/reference/validation/u_rimp2/*.json provenance)."""
    s, u = np.linalg.eigh(S)
    X = u / np.sqrt(s)
    if guess is None:
        e, c = np.linalg.eigh(X.T @ H @ X)
        Ca = Cb = X @ c
    else:
        Ca, Cb = guess
    jk = exact_jk(eri)
    focks, errs = [], []
    e_old = 0.0
    for it in range(max_iter):
        Da = Ca[:, :na] @ Ca[:, :na].T
        Db = Cb[:, :nb] @ Cb[:, :nb].T
        Ja, Ka = jk(Da)
        Jb, Kb = jk(Db)
        Fa = H + Ja + Jb - Ka
        Fb = H + Ja + Jb - Kb
        E = 0.5 * (np.sum(Da * (H + Fa)) + np.sum(Db * (H + Fb))) + e_nuc
        ea = X.T @ (Fa @ Da @ S - S @ Da @ Fa) @ X
        eb = X.T @ (Fb @ Db @ S - S @ Db @ Fb) @ X
        focks.append((Fa, Fb))
        errs.append(np.concatenate([ea.ravel(), eb.ravel()]))
        if len(focks) > 10:
            focks.pop(0)
            errs.pop(0)
        if np.abs(errs[-1]).max() < tol * 100 and abs(E - e_old) < tol:
            break
        e_old = E
        m = len(focks)
        Bm = -np.ones((m + 1, m + 1))
        Bm[m, m] = 0.0
        for a in range(m):
            for b in range(m):
                Bm[a, b] = errs[a] @ errs[b]
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        coef = np.linalg.lstsq(Bm, rhs, rcond=None)[0][:m]
        Fda = sum(cf * f[0] for cf, f in zip(coef, focks))
        Fdb = sum(cf * f[1] for cf, f in zip(coef, focks))
        Ca = X @ np.linalg.eigh(X.T @ Fda @ X)[1]
        Cb = X @ np.linalg.eigh(X.T @ Fdb @ X)[1]
    epa, ca = np.linalg.eigh(X.T @ Fa @ X)
    epb, cb = np.linalg.eigh(X.T @ Fb @ X)
    return E, (epa, epb), (X @ ca, X @ cb)

"""Gaussian integrals for the oracle's golden pin (test infrastructure only).

A McMurchie-Davidson engine in NumPy (Helgaker, Jorgensen, Olsen, "Molecular
Electronic-Structure Theory", ch. 9: Hermite expansion coefficients E_t^{ij},
Hermite Coulomb integrals R_tuv^n from the Boys function).  It replaces, for
the oracle only, the libint2 2.13.1 integrals ferric takes through its C++ shim
(ferric-integrals/shim/shim.h:167-194); nothing here is derived from libint2.

Spherical shells.  The reference's bases use pure (spherical) functions for
l >= 2 (BSE ``gto_spherical``).  Their span is the set of harmonic homogeneous
polynomials of degree l times the radial Gaussian, i.e. the null space of the
Laplacian on the Cartesian monomials of degree l; this module takes a basis of
that null space.  SCF and MP2 energies are invariant to the choice of basis
inside each shell's span, so no solid-harmonic convention is needed.

Boys function F_n(T) from the regularised lower incomplete gamma function
(scipy.special.gammainc), with its Taylor series for small T.
"""
from __future__ import annotations

import itertools
import math

import numpy as np
from scipy.special import gamma as gamma_fn
from scipy.special import gammainc


# ----------------------------------------------------------------- Boys --

def boys(nmax, t):
    """F_n(t) for n = 0..nmax, array of shape (nmax + 1,) + t.shape."""
    t = np.asarray(t, dtype=np.float64)
    out = np.empty((nmax + 1,) + t.shape)
    small = t < 1e-2
    tl = np.where(small, 1.0, t)
    for n in range(nmax + 1):
        a = n + 0.5
        big = gamma_fn(a) * gammainc(a, tl) / (2.0 * tl ** a)
        # series: sum_k (-t)^k / (k! (2n + 2k + 1))
        ser = np.zeros_like(t)
        term = np.ones_like(t)
        for k in range(30):
            ser += term / (2 * n + 2 * k + 1)
            term = term * (-t) / (k + 1)
        out[n] = np.where(small, ser, big)
    return out


# ---------------------------------------------------------------- shells --

def cart_components(l):
    """Cartesian exponents (x, y, z) of degree l in a fixed order."""
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def spherical_transform(l):
    """(ncart, 2l+1) basis of the harmonic subspace of degree-l monomials."""
    comps = cart_components(l)
    if l < 2:
        return np.eye(len(comps))
    lower = {c: k for k, c in enumerate(cart_components(l - 2))}
    lap = np.zeros((len(lower), len(comps)))
    for j, (a, b, c) in enumerate(comps):
        for (e, f) in ((0, a), (1, b), (2, c)):
            if f >= 2:
                m = [a, b, c]
                m[e] -= 2
                lap[lower[tuple(m)], j] += f * (f - 1)
    _, s, vt = np.linalg.svd(lap)
    null = vt[len(lower):].T
    assert null.shape[1] == 2 * l + 1
    return null


def _dfact(n):
    return 1.0 if n <= 0 else float(np.prod(np.arange(n, 0, -2)))


class Shell:
    """A (generally) contracted shell: centre, l, exponents, coefficient
    columns (one per contracted function), spherical or Cartesian."""

    def __init__(self, center, l, exps, coefs, spherical):
        self.center = np.asarray(center, dtype=np.float64)
        self.l = int(l)
        self.exps = np.asarray(exps, dtype=np.float64)
        c = np.asarray(coefs, dtype=np.float64).reshape(len(self.exps), -1)
        # primitive normalisation of the x^l component, then contracted norm
        norm = (2 * self.exps / np.pi) ** 0.75 * (4 * self.exps) ** (self.l / 2) / math.sqrt(_dfact(2 * self.l - 1))
        c = c * norm[:, None]
        ee = self.exps[:, None] + self.exps[None, :]
        s = (np.pi / ee) ** 1.5 * _dfact(2 * self.l - 1) / (2 * ee) ** self.l
        for k in range(c.shape[1]):
            c[:, k] /= math.sqrt(c[:, k] @ s @ c[:, k])
        self.coefs = c
        self.spherical = bool(spherical) and self.l >= 2
        self.ncart = (self.l + 1) * (self.l + 2) // 2
        self.nfunc_shell = 2 * self.l + 1 if self.spherical else self.ncart
        self.ncontr = c.shape[1]

    def cart_to_func(self):
        return spherical_transform(self.l) if self.spherical else np.eye(self.ncart)


def dummy_shell(center):
    """Unit s function with exponent 0 (for 3- and 2-centre integrals)."""
    sh = Shell.__new__(Shell)
    sh.center = np.asarray(center, dtype=np.float64)
    sh.l = 0
    sh.exps = np.zeros(1)
    sh.coefs = np.ones((1, 1))
    sh.spherical = False
    sh.ncart = 1
    sh.nfunc_shell = 1
    sh.ncontr = 1
    return sh


# ------------------------------------------------------- Hermite algebra --

def hermite_e(la, lb, a, b, xa, xb):
    """E[i, j, t, Ka, Kb] of one Cartesian direction, i <= la, j <= lb."""
    p = a[:, None] + b[None, :]
    mu = a[:, None] * b[None, :] / np.where(p > 0, p, 1.0)
    px = (a[:, None] * xa + b[None, :] * xb) / np.where(p > 0, p, 1.0)
    xpa, xpb = px - xa, px - xb
    inv2p = 0.5 / np.where(p > 0, p, 1.0)
    lt = la + lb + 2
    e = np.zeros((la + 1, lb + 1, lt + 1) + p.shape)
    e[0, 0, 0] = np.exp(-mu * (xa - xb) ** 2)
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            if i > 0:
                src, x = e[i - 1, j], xpa
            else:
                src, x = e[i, j - 1], xpb
            for t in range(i + j + 1):
                v = x * src[t] + (t + 1) * src[t + 1]
                if t > 0:
                    v = v + inv2p * src[t - 1]
                e[i, j, t] = v
    return e


def pair_data(sa, sb, lb_extra=0):
    """Hermite coefficients of a shell pair over all primitive pairs.

    Returns dict with p (P,), centre P (P,3), E (Ca, Cb, L+1, L+1, L+1, P)."""
    a, b = sa.exps, sb.exps
    lb = sb.l + lb_extra
    ex = [hermite_e(sa.l, lb, a, b, sa.center[d], sb.center[d]) for d in range(3)]
    ca = cart_components(sa.l)
    cb = cart_components(lb)
    L = sa.l + lb
    npair = len(a) * len(b)
    e3 = np.zeros((len(ca), len(cb), L + 1, L + 1, L + 1, npair))
    for ia, (ax, ay, az) in enumerate(ca):
        for ib, (bx, by, bz) in enumerate(cb):
            exx = ex[0][ax, bx, :ax + bx + 1].reshape(ax + bx + 1, -1)
            eyy = ex[1][ay, by, :ay + by + 1].reshape(ay + by + 1, -1)
            ezz = ex[2][az, bz, :az + bz + 1].reshape(az + bz + 1, -1)
            e3[ia, ib, :ax + bx + 1, :ay + by + 1, :az + bz + 1] = (
                exx[:, None, None, :] * eyy[None, :, None, :] * ezz[None, None, :, :])
    p = (a[:, None] + b[None, :]).reshape(-1)
    pc = ((a[:, None, None] * sa.center + b[None, :, None] * sb.center)
          / (a[:, None, None] + b[None, :, None])).reshape(-1, 3)
    coef = (sa.coefs[:, None, :, None] * sb.coefs[None, :, None, :]).reshape(npair, sa.ncontr * sb.ncontr)
    return dict(p=p, P=pc, E=e3, L=L, coef=coef, ex=ex)


def hermite_r(L, alpha, rpq):
    """R^0_{tuv}(alpha, R_PQ) for t+u+v <= L; shape (L+1, L+1, L+1) + alpha.shape."""
    x, y, z = rpq[..., 0], rpq[..., 1], rpq[..., 2]
    r2 = x * x + y * y + z * z
    f = boys(L, alpha * r2)
    shape = alpha.shape
    # r[n][t][u][v]
    r = np.zeros((L + 1, L + 1, L + 1, L + 1) + shape)
    for n in range(L + 1):
        r[n, 0, 0, 0] = (-2.0 * alpha) ** n * f[n]
    for n in range(L - 1, -1, -1):
        for tot in range(1, L - n + 1):
            for t in range(tot + 1):
                for u in range(tot - t + 1):
                    v = tot - t - u
                    if t > 0:
                        val = x * r[n + 1, t - 1, u, v]
                        if t > 1:
                            val = val + (t - 1) * r[n + 1, t - 2, u, v]
                    elif u > 0:
                        val = y * r[n + 1, t, u - 1, v]
                        if u > 1:
                            val = val + (u - 1) * r[n + 1, t, u - 2, v]
                    else:
                        val = z * r[n + 1, t, u, v - 1]
                        if v > 1:
                            val = val + (v - 1) * r[n + 1, t, u, v - 2]
                    r[n, t, u, v] = val
    return r[0]


# ------------------------------------------------------------ integrals --

def _herm_index(L):
    idx = [(t, u, v) for t in range(L + 1) for u in range(L + 1) for v in range(L + 1) if t + u + v <= L]
    return np.array(idx, dtype=np.int64).reshape(-1, 3)


def eri_pairs(d1, d2):
    """(ab|cd) over contracted functions, Cartesian components:
    shape (Ca, na, Cb, nb, Cc, nc, Cd, nd) flattened as (Ca*Cb*nab, Cc*Cd*ncd)."""
    L1, L2 = d1["L"], d2["L"]
    p, q = d1["p"], d2["p"]
    pp, qq = p[:, None], q[None, :]
    alpha = pp * qq / (pp + qq)
    rpq = d1["P"][:, None, :] - d2["P"][None, :, :]
    R = hermite_r(L1 + L2, alpha, rpq)                               # (L,L,L,P1,P2)
    pref = 2.0 * np.pi ** 2.5 / (pp * qq * np.sqrt(pp + qq))
    h1, h2 = _herm_index(L1), _herm_index(L2)
    sign = (-1.0) ** h2.sum(axis=1)
    tt = h1[:, None, :] + h2[None, :, :]
    Rg = R[tt[..., 0], tt[..., 1], tt[..., 2]] * (sign[None, :, None, None] * pref[None, None])
    E1 = d1["E"][:, :, h1[:, 0], h1[:, 1], h1[:, 2]]                  # (Ca,Cb,H1,P1)
    E2 = d2["E"][:, :, h2[:, 0], h2[:, 1], h2[:, 2]]                  # (Cc,Cd,H2,P2)
    ca, cb = E1.shape[:2]
    cc, cd = E2.shape[:2]
    E1 = E1.reshape(ca * cb, len(h1), -1)
    E2 = E2.reshape(cc * cd, len(h2), -1)
    T1 = np.einsum("ahp,hkpq->akpq", E1, Rg, optimize=True)
    T2 = np.einsum("akpq,ckq,qm->apcm", T1, E2, d2["coef"], optimize=True)
    out = np.einsum("apcm,pn->ancm", T2, d1["coef"], optimize=True)  # (Ca*Cb, n12, Cc*Cd, n34)
    return out


def _shell_funcs(shells):
    """Per shell: (offset, ncontr, nfunc, transform)."""
    info, off = [], 0
    for sh in shells:
        tr = sh.cart_to_func()
        info.append((off, sh.ncontr, tr.shape[1], tr))
        off += sh.ncontr * tr.shape[1]
    return info, off


def _to_funcs(block, sa, sb, ta, tb):
    """(Ca*Cb, na*nb) pair block -> (na, fa, nb, fb) function block."""
    ca, cb = sa.ncart, sb.ncart
    b = block.reshape(ca, cb, sa.ncontr, sb.ncontr)
    return np.einsum("xyij,xf,yg->ifjg", b, ta, tb)


def overlap_kinetic(shells):
    info, n = _shell_funcs(shells)
    S = np.zeros((n, n))
    T = np.zeros((n, n))
    for (ia, sa), (ib, sb) in itertools.product(enumerate(shells), repeat=2):
        d = pair_data(sa, sb, lb_extra=2)
        ex = d["ex"]
        p = (sa.exps[:, None] + sb.exps[None, :])
        sq = np.sqrt(np.pi / p)
        b = sb.exps[None, :]
        s_blk = np.zeros((sa.ncart, sb.ncart) + p.shape)
        t_blk = np.zeros_like(s_blk)
        for x, (a1, a2, a3) in enumerate(cart_components(sa.l)):
            for y, (b1, b2, b3) in enumerate(cart_components(sb.l)):
                s1d = [lambda i, j, dd=dd: ex[dd][i, j, 0] * sq if j >= 0 else 0.0 for dd in range(3)]
                sx, sy, sz = s1d[0](a1, b1), s1d[1](a2, b2), s1d[2](a3, b3)
                s_blk[x, y] = sx * sy * sz

                def kin(dd, i, j):
                    v = -2.0 * b * b * s1d[dd](i, j + 2) + b * (2 * j + 1) * s1d[dd](i, j)
                    if j >= 2:
                        v = v - 0.5 * j * (j - 1) * s1d[dd](i, j - 2)
                    return v
                t_blk[x, y] = kin(0, a1, b1) * sy * sz + sx * kin(1, a2, b2) * sz + sx * sy * kin(2, a3, b3)
        cs = sa.coefs[:, None, :, None] * sb.coefs[None, :, None, :]
        for blk, M in ((s_blk, S), (t_blk, T)):
            c = np.einsum("xypq,pqij->xyij", blk, cs).reshape(sa.ncart * sb.ncart, -1)
            f = _to_funcs(c, sa, sb, info[ia][3], info[ib][3])
            oa, ob = info[ia][0], info[ib][0]
            M[oa:oa + f.shape[0] * f.shape[1], ob:ob + f.shape[2] * f.shape[3]] = f.reshape(
                f.shape[0] * f.shape[1], -1)
    return S, T


def nuclear(shells, charges, coords):
    info, n = _shell_funcs(shells)
    V = np.zeros((n, n))
    for (ia, sa), (ib, sb) in itertools.product(enumerate(shells), repeat=2):
        d = pair_data(sa, sb)
        L = d["L"]
        h = _herm_index(L)
        E = d["E"][:, :, h[:, 0], h[:, 1], h[:, 2]]                  # (Ca,Cb,H,P)
        acc = np.zeros(E.shape[:2] + (E.shape[3],))
        for z, c in zip(charges, coords):
            R = hermite_r(L, d["p"], d["P"] - np.asarray(c)[None, :])  # (L,L,L,P)
            Rg = R[h[:, 0], h[:, 1], h[:, 2]]
            acc += -z * np.einsum("xyhp,hp->xyp", E, Rg)
        acc *= (2.0 * np.pi / d["p"])[None, None]
        c = (acc.reshape(sa.ncart * sb.ncart, -1) @ d["coef"])
        f = _to_funcs(c, sa, sb, info[ia][3], info[ib][3])
        oa, ob = info[ia][0], info[ib][0]
        V[oa:oa + f.shape[0] * f.shape[1], ob:ob + f.shape[2] * f.shape[3]] = f.reshape(f.shape[0] * f.shape[1], -1)
    return V


def eri4(shells):
    """Full (mn|ls) tensor (exact-JK pin only; small bases)."""
    info, n = _shell_funcs(shells)
    ns = len(shells)
    pdata = {}
    for a in range(ns):
        for b in range(a + 1):
            pdata[(a, b)] = pair_data(shells[a], shells[b])
    out = np.zeros((n, n, n, n))
    pairs = sorted(pdata)
    for k1, (a, b) in enumerate(pairs):
        for (c, d) in pairs[:k1 + 1]:
            blk = eri_pairs(pdata[(a, b)], pdata[(c, d)])
            sa, sb, sc, sd = shells[a], shells[b], shells[c], shells[d]
            blk = blk.reshape(sa.ncart, sb.ncart, sa.ncontr, sb.ncontr, sc.ncart, sd.ncart, sc.ncontr, sd.ncontr)
            f = np.einsum("wxijyzkl,wA,xB,yC,zD->iAjBkClD", blk, info[a][3], info[b][3], info[c][3], info[d][3],
                          optimize=True)
            na = f.shape[0] * f.shape[1]
            nb = f.shape[2] * f.shape[3]
            nc = f.shape[4] * f.shape[5]
            nd = f.shape[6] * f.shape[7]
            f = f.reshape(na, nb, nc, nd)
            oa, ob, oc, od = info[a][0], info[b][0], info[c][0], info[d][0]
            for (x0, y0, z0, w0, g) in (
                    (oa, ob, oc, od, f), (ob, oa, oc, od, f.transpose(1, 0, 2, 3)),
                    (oa, ob, od, oc, f.transpose(0, 1, 3, 2)), (ob, oa, od, oc, f.transpose(1, 0, 3, 2)),
                    (oc, od, oa, ob, f.transpose(2, 3, 0, 1)), (od, oc, oa, ob, f.transpose(3, 2, 0, 1)),
                    (oc, od, ob, oa, f.transpose(2, 3, 1, 0)), (od, oc, ob, oa, f.transpose(3, 2, 1, 0))):
                out[x0:x0 + g.shape[0], y0:y0 + g.shape[1], z0:z0 + g.shape[2], w0:w0 + g.shape[3]] = g
    return out


def eri3(aux, shells):
    """(P|mn), shape (naux, n, n)."""
    ainfo, naux = _shell_funcs(aux)
    info, n = _shell_funcs(shells)
    out = np.zeros((naux, n, n))
    pd = {}
    for a in range(len(shells)):
        for b in range(a + 1):
            pd[(a, b)] = pair_data(shells[a], shells[b])
    for k, sp in enumerate(aux):
        dp = pair_data(sp, dummy_shell(sp.center))
        for (a, b), d2 in pd.items():
            blk = eri_pairs(dp, d2)
            sa, sb = shells[a], shells[b]
            blk = blk.reshape(sp.ncart, sp.ncontr, sa.ncart, sb.ncart, sa.ncontr, sb.ncontr)
            f = np.einsum("pkxyij,pP,xA,yB->kPiAjB", blk, ainfo[k][3], info[a][3], info[b][3], optimize=True)
            f = f.reshape(f.shape[0] * f.shape[1], f.shape[2] * f.shape[3], f.shape[4] * f.shape[5])
            o, oa, ob = ainfo[k][0], info[a][0], info[b][0]
            out[o:o + f.shape[0], oa:oa + f.shape[1], ob:ob + f.shape[2]] = f
            out[o:o + f.shape[0], ob:ob + f.shape[2], oa:oa + f.shape[1]] = f.transpose(0, 2, 1)
    return out


def eri2(aux):
    """(P|Q) Coulomb metric."""
    ainfo, naux = _shell_funcs(aux)
    out = np.zeros((naux, naux))
    dd = [pair_data(s, dummy_shell(s.center)) for s in aux]
    for a in range(len(aux)):
        for b in range(a + 1):
            blk = eri_pairs(dd[a], dd[b]).reshape(aux[a].ncart, aux[a].ncontr, aux[b].ncart, aux[b].ncontr)
            f = np.einsum("xiyj,xA,yB->iAjB", blk, ainfo[a][3], ainfo[b][3])
            f = f.reshape(f.shape[0] * f.shape[1], -1)
            oa, ob = ainfo[a][0], ainfo[b][0]
            out[oa:oa + f.shape[0], ob:ob + f.shape[1]] = f
            out[ob:ob + f.shape[1], oa:oa + f.shape[0]] = f.T
    return out

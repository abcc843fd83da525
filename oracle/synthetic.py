"""Seeded synthetic inputs of the benchmark shapes (oracle side, NumPy).

Distributions (one seed per tensor, NumPy ``default_rng``):

* DF-JK: ``B_Q,mn = 0.05 N(0,1) exp(-|m-n|/50)``, symmetrised per Q as
  ``(X + X^T)/sqrt(2)``; ``C_occ`` = Q factor of the QR of a Gaussian
  ``n x nocc``; ``D = C_occ C_occ^T``.  Full size: n 600, naux 2400, nocc 60.
* RI-MP2: ``B_Q,ia = 0.02 N(0,1) exp(-Q/3000)``; ``eps_occ ~ U[-20, -0.3]``,
  ``eps_vir ~ U[0.05, 6]``, both sorted ascending.  Full size: naux 4800,
  nocc 120, nvir 1100.

Scaled-down cases keep the distributions; the Q decay length scales with
naux (``3000 * naux / 4800``) so a small case has the same spectrum shape.
"""
from __future__ import annotations

import numpy as np


def dfjk_inputs(n=600, naux=2400, nocc=60, seed_b=2, seed_c=20):
    rng = np.random.default_rng(seed_b)
    idx = np.arange(n)
    env = 0.05 * np.exp(-np.abs(idx[:, None] - idx[None, :]) / 50.0)
    b = np.empty((naux, n, n))
    for q in range(naux):
        x = rng.standard_normal((n, n)) * env
        b[q] = (x + x.T) / np.sqrt(2.0)
    rc = np.random.default_rng(seed_c)
    c_occ, _ = np.linalg.qr(rc.standard_normal((n, nocc)))
    c_occ = np.ascontiguousarray(c_occ)
    d = c_occ @ c_occ.T
    return b, c_occ, d


def rimp2_inputs(naux=4800, nocc=120, nvir=1100, seed_b=3, seed_eps=30, decay=None):
    if decay is None:
        decay = 3000.0 * naux / 4800.0
    rng = np.random.default_rng(seed_b)
    b = 0.02 * rng.standard_normal((naux, nocc * nvir))
    b *= np.exp(-np.arange(naux) / decay)[:, None]
    r2 = np.random.default_rng(seed_eps)
    eps_occ = np.sort(r2.uniform(-20.0, -0.3, nocc))
    eps_vir = np.sort(r2.uniform(0.05, 6.0, nvir))
    return b, eps_occ, eps_vir


def fd_entries(naux, nov, count=64, seed=31):
    """The 64 seeded (P, ia) entries of the finite-difference check."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, naux, count), rng.integers(0, nov, count)

"""Generate the RI-MP2 inputs of the batched benchmark's alkanes C_nH_2n+2, n = 1..8.

All-trans linear alkanes with C-C 1.54 A, C-H 1.09 A and tetrahedral angles
(the batched RI-MP2 benchmark's molecules), cc-pVDZ orbital basis,
cc-pVDZ-RI auxiliary basis.  The oracle's own integral engine and RHF
(oracle/integrals.py, oracle/scf.py) make, per molecule:

* the dressed 3-index tensor B = L^-1 (P|mu nu), V = (P|Q) = L L^T
  (ferric-mp2/src/rimp2.rs:2478-2489, 666-756);
* a closed-shell RHF whose J and K are fitted with the same dressed tensor
  (F = H + J - K/2, ferric-scf/src/rhf.rs:3040-3090), converged to 1e-10;
* B_ov = C_occ^T B C_vir and the orbital energies, and the oracle's FP64
  RI-MP2 energy of them (rimp2.rs:1399-1544).

The SCF fits J and K in the RI basis rather than a JK-fitting set so the
oracle's integral work stays within minutes; the inputs are those of a
converged RHF either way.

    FERRIC_REFERENCE_ROOT=<reference checkout> python tests/golden/make_alkanes.py [nmax] [--procs P]

Writes tests/golden/alkanes_c1_c3.npz (n = 1..3, committed, read by the GPU
tests) and tests/golden/_cache/alkanes_c1_c8.npz (all eight, ~80 MB, kept out
of git; the benchmark's batched leg reads it when present).  Needs the
reference checkout only for the basis JSONs.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np
import scipy.linalg

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import basis, integrals, scf  # noqa: E402
from oracle import rimp2 as orc  # noqa: E402

R_CC, R_CH = 1.54, 1.09               # Angstrom
TETRA = np.arccos(-1.0 / 3.0)          # 109.4712 degrees


def alkane_geometry(n):
    """[(symbol, (x, y, z) Angstrom)] of all-trans C_nH_2n+2.

    Carbons zig-zag in the xy plane (C-C-C = tetrahedral).  Each carbon's two
    in-plane bond directions point at its backbone neighbours; where a
    neighbour is missing (chain ends) a hydrogen takes its place, so the end
    hydrogens lie in the plane, anti to the next C-C bond.  The other two
    hydrogens of every carbon sit above and below the plane, symmetric about
    the bisector of the in-plane bonds, at tetrahedral angles.
    """
    s, c = R_CC * np.sin(TETRA / 2), R_CC * np.cos(TETRA / 2)

    def cpos(k):                      # backbone site k (virtual beyond the chain)
        return np.array([k * s, (k % 2) * c, 0.0])

    atoms = [("C", cpos(k)) for k in range(n)]
    z = np.array([0.0, 0.0, 1.0])
    for k in range(n):
        ck = cpos(k)
        dirs = []
        for nb in (k - 1, k + 1):
            u = cpos(nb) - ck
            u /= np.linalg.norm(u)
            dirs.append(u)
            if not 0 <= nb < n:
                atoms.append(("H", ck + R_CH * u))
        bis = -(dirs[0] + dirs[1])
        bis /= np.linalg.norm(bis)
        half = TETRA / 2
        for sgn in (1.0, -1.0):
            atoms.append(("H", ck + R_CH * (np.cos(half) * bis + sgn * np.sin(half) * z)))
    return [(sym, tuple(float(x) for x in p)) for sym, p in atoms]


def _eri3_part(args):
    aux, shells = args
    return integrals.eri3(aux, shells)


def build(n, procs):
    t0 = time.time()
    atoms_a = alkane_geometry(n)
    atoms = [(sym, tuple(basis.BOHR_PER_ANGSTROM * x for x in p)) for sym, p in atoms_a]
    zs = [basis.SYMBOLS[s] for s, _ in atoms]
    rs = [p for _, p in atoms]
    sh = basis.shells_for(atoms, "cc-pvdz")
    aux = basis.shells_for(atoms, "cc-pvdz-ri")
    S, T = integrals.overlap_kinetic(sh)
    V = integrals.nuclear(sh, zs, rs)
    enuc = scf.nuclear_repulsion(zs, rs)
    # contiguous runs of aux shells, many more than processes (uneven cost
    # per shell); results come back in order, so they stack in basis order
    nchunk = min(len(aux), 6 * procs)
    bounds = np.linspace(0, len(aux), nchunk + 1).astype(int)
    parts = [aux[bounds[k]:bounds[k + 1]] for k in range(nchunk) if bounds[k + 1] > bounds[k]]
    with mp.get_context("spawn").Pool(procs) as pool:
        t3 = np.concatenate(pool.map(_eri3_part, [(p, sh) for p in parts], chunksize=1), axis=0)
    naux, nb = t3.shape[0], S.shape[0]
    vm = integrals.eri2(aux)
    l = np.linalg.cholesky(vm)
    b = scipy.linalg.solve_triangular(l, t3.reshape(naux, -1), lower=True).reshape(naux, nb, nb)
    nocc = (sum(zs)) // 2
    e_rhf, eps, C = scf.rhf(S, T + V, nocc, enuc, scf.df_jk(b), tol=1e-10)
    bov = scf.b_ov(b, C, nocc)
    nvir = nb - nocc
    e_os, e_ss, _ = orc.spin_components(bov, eps, nocc, nvir)
    print(f"C{n}H{2 * n + 2}: nbf {nb} naux {naux} nocc {nocc} nvir {nvir} E_rhf {e_rhf:.10f} "
          f"E_os {e_os:.12f} E_ss {e_ss:.12f} ({time.time() - t0:.0f} s)", flush=True)
    return dict(b_ov=bov, eps_occ=eps[:nocc].copy(), eps_vir=eps[nocc:].copy(), e_rhf=e_rhf, e_os=e_os,
                e_ss=e_ss, geometry=np.array([p for _, p in atoms_a]), symbols=np.array([s for s, _ in atoms_a]))


def main():
    nmax = int(next((a for a in sys.argv[1:] if a.isdigit()), 8))
    procs = int(sys.argv[sys.argv.index("--procs") + 1]) if "--procs" in sys.argv else os.cpu_count()
    if not basis.available():
        sys.exit("set FERRIC_REFERENCE_ROOT to the reference checkout (basis JSONs)")
    out = {}
    for n in range(1, nmax + 1):
        r = build(n, procs)
        for k, v in r.items():
            out[f"c{n}_{k}"] = v
        if n == 3:
            np.savez_compressed(os.path.join(HERE, "alkanes_c1_c3.npz"), **out)
    os.makedirs(os.path.join(HERE, "_cache"), exist_ok=True)
    np.savez(os.path.join(HERE, "_cache", f"alkanes_c1_c{nmax}.npz"), **out)


if __name__ == "__main__":
    main()

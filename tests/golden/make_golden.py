"""Generate the golden fixtures of the RI-MP2 / DF-JK parity tests.

Runs the oracle's own integral engine and RHF (oracle/integrals.py, oracle/scf.py)
on the reference's validation molecules and writes, per system, the RI-MP2
inputs (dressed B_ov, orbital energies) and the reference's golden energies
(PySCF 2.13.1 numbers from the reference's testdata/reference/validation JSONs)
into ``<name>.npz``.  The device tests read only these fixtures.

    FERRIC_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py [name ...]

Reads the basis JSONs and golden JSONs from the reference checkout named by
``FERRIC_REFERENCE_ROOT``.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import basis, integrals, scf  # noqa: E402
from oracle import rimp2 as orc  # noqa: E402


def validation_dir():
    root = basis.reference_root()
    if root is None:
        sys.exit("set FERRIC_REFERENCE_ROOT to the reference checkout")
    return os.path.join(root, "testdata", "reference", "validation")

SYSTEMS = {
    # name: (golden json, basis, aux basis, kappa json or None, JK-fit basis for the DF-JK SCF or None)
    "h2o_ccpvdz": ("sos_mp2/h2o_cc-pvdz.json", "cc-pvdz", "cc-pvdz-ri", "kappa_mp2/h2o_cc-pvdz.json", "cc-pvtz-jkfit"),
    "ch4_ccpvdz": ("sos_mp2/ch4_cc-pvdz.json", "cc-pvdz", "cc-pvdz-ri", "kappa_mp2/ch4_cc-pvdz.json", None),
    "h2o_augccpvdz": ("sos_mp2/h2o_aug_aug-cc-pvdz.json", "aug-cc-pvdz", "aug-cc-pvdz-rifit", None, None),
}


def build(name):
    gfile, bas, aux, kfile, jkfit = SYSTEMS[name]
    REF = validation_dir()
    g = json.load(open(os.path.join(REF, gfile)))
    atoms = [(s, (x, y, z)) for s, x, y, z in g["provenance"]["geometry_bohr"]]
    zs = [basis.SYMBOLS[s] for s, _ in atoms]
    rs = [c for _, c in atoms]
    t0 = time.time()
    sh = basis.shells_for(atoms, bas)
    S, T = integrals.overlap_kinetic(sh)
    V = integrals.nuclear(sh, zs, rs)
    eri = integrals.eri4(sh)
    enuc = scf.nuclear_repulsion(zs, rs)
    nocc = int(g["nocc"])
    e_rhf, eps, C = scf.rhf(S, T + V, nocc, enuc, scf.exact_jk(eri))
    b, v_aux, t3_aux = scf.dressed(basis.shells_for(atoms, aux), sh)
    bov = scf.b_ov(b, C, nocc)
    nvir = C.shape[1] - nocc
    e_os, e_ss, _ = orc.spin_components(bov, eps, nocc, nvir)
    out = dict(b_ov=bov, eps=eps, nocc=nocc, nvir=nvir,
               golden_e_rhf=g["e_rhf"], golden_e_os=g["dfmp2"]["e_os"], golden_e_ss=g["dfmp2"]["e_ss"],
               oracle_e_rhf=e_rhf, oracle_e_os=e_os, oracle_e_ss=e_ss)
    if kfile:
        k = json.load(open(os.path.join(REF, kfile)))
        out["kappa"] = np.array([r["kappa"] for r in k["kappa"]])
        out["golden_kappa_e_os"] = np.array([r["e_os"] for r in k["kappa"]])
        out["golden_kappa_e_ss"] = np.array([r["e_ss"] for r in k["kappa"]])
    if jkfit:
        # config 1: RHF with DF-JK (JK-fit basis), then RI-MP2 on its orbitals
        bjk, _, _ = scf.dressed(basis.shells_for(atoms, jkfit), sh)
        e_df, eps_df, c_df = scf.rhf(S, T + V, nocc, enuc, scf.df_jk(bjk))
        bov_df = scf.b_ov(b, c_df, nocc)
        d_os, d_ss, _ = orc.spin_components(bov_df, eps_df, nocc, nvir)
        # raw (P|mn), the metric and the exact-JK orbitals: inputs of the MO dressing
        out.update(b_jk=bjk, b_ri=b, h_core=T + V, s=S, e_nuc=enuc, oracle_e_dfrhf=e_df,
                   oracle_dfrhf_e_os=d_os, oracle_dfrhf_e_ss=d_ss, t3_ri=t3_aux, v_ri=v_aux, c=C)
    print(f"{name}: n {C.shape[0]} naux {bov.shape[0]} E_rhf {e_rhf:.12f} (golden {g['e_rhf']:.12f}) "
          f"E_os {e_os:.14f} (golden {g['dfmp2']['e_os']:.14f}) {time.time() - t0:.1f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


# open-shell systems: UHF (exact J/K) then unrestricted RI-MP2 (alpha-alpha,
# beta-beta, alpha-beta) against the reference's u_rimp2 goldens
U_SYSTEMS = {
    "oh_ump2": "u_rimp2/oh_cc-pvdz.json",
    "nh2_ump2": "u_rimp2/nh2_cc-pvdz.json",
}


def build_u(name):
    g = json.load(open(os.path.join(validation_dir(), U_SYSTEMS[name])))
    atoms = [(s, (x, y, z)) for s, x, y, z in g["provenance"]["geometry_bohr"]]
    zs = [basis.SYMBOLS[s] for s, _ in atoms]
    rs = [c for _, c in atoms]
    t0 = time.time()
    sh = basis.shells_for(atoms, g["basis"])
    S, T = integrals.overlap_kinetic(sh)
    V = integrals.nuclear(sh, zs, rs)
    eri = integrals.eri4(sh)
    enuc = scf.nuclear_repulsion(zs, rs)
    na, nb = int(g["uhf"]["nelec_alpha"]), int(g["uhf"]["nelec_beta"])
    # several starting orbitals (core Hamiltonian; RHF of the n-electron
    # cation- and anion-like closed shells), keep the lowest UHF solution, as
    # the goldens' generator scans guesses ("3 guesses + stability loop")
    tries = [scf.uhf(S, T + V, na, nb, enuc, eri)]
    for nc in sorted({nb, na}):
        _, _, c0 = scf.rhf(S, T + V, nc, enuc, scf.exact_jk(eri), tol=1e-9)
        tries.append(scf.uhf(S, T + V, na, nb, enuc, eri, guess=(c0, c0)))
    e_uhf, (epa, epb), (ca, cb) = min(tries, key=lambda r: r[0])
    b, _, _ = scf.dressed(basis.shells_for(atoms, g["aux_basis"]), sh)
    ba, bb = scf.b_ov(b, ca, na), scf.b_ov(b, cb, nb)
    e_aa = orc.u_same_spin(ba, epa[:na], epa[na:])
    e_bb = orc.u_same_spin(bb, epb[:nb], epb[nb:])
    e_ab = orc.u_opposite_spin(ba, epa[:na], epa[na:], bb, epb[:nb], epb[nb:])
    u = g["ump2"]
    out = dict(b_a=ba, b_b=bb, eps_a=epa, eps_b=epb, na=na, nb=nb,
               golden_e_uhf=g["uhf"]["energy"], golden_e_aa=u["e_aa"], golden_e_bb=u["e_bb"],
               golden_e_ab=u["e_ab"], oracle_e_uhf=e_uhf, oracle_e_aa=e_aa, oracle_e_bb=e_bb,
               oracle_e_ab=e_ab)
    print(f"{name}: E_uhf {e_uhf:.12f} (golden {g['uhf']['energy']:.12f}) e_aa {e_aa:.14f} "
          f"({u['e_aa']:.14f}) e_bb {e_bb:.14f} ({u['e_bb']:.14f}) e_ab {e_ab:.14f} ({u['e_ab']:.14f}) "
          f"{time.time() - t0:.1f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(SYSTEMS) + list(U_SYSTEMS)):
        (build_u if n in U_SYSTEMS else build)(n)

"""Basis-set loading for the oracle's golden pin (test infrastructure only).

Reads the reference's bundled MolSSI-BSE JSON files
(ferric-core/src/basis/bundled/*.json) at run time; nothing is copied into
this repository.  The directory is taken from ``FERRIC_BASIS_DIR``, else
from the reference checkout named by ``FERRIC_REFERENCE_ROOT``; with neither
set, ``available()`` is False and the callers skip.
"""
from __future__ import annotations

import json
import os

from .integrals import Shell

BOHR_PER_ANGSTROM = 1.0 / 0.52917721092   # the conversion the reference's JSONs record
SYMBOLS = {"H": 1, "He": 2, "C": 6, "N": 7, "O": 8, "F": 9}


def reference_root():
    """The reference checkout (``FERRIC_REFERENCE_ROOT``), or None."""
    return os.environ.get("FERRIC_REFERENCE_ROOT") or None


def basis_dir():
    d = os.environ.get("FERRIC_BASIS_DIR")
    if d:
        return d
    root = reference_root()
    if root is None:
        return None
    return os.path.join(root, "crates", "ferric-core", "src", "basis", "bundled")


def available():
    d = basis_dir()
    return d is not None and os.path.isdir(d)


def load(name):
    with open(os.path.join(basis_dir(), f"{name}.json")) as f:
        return json.load(f)["elements"]


def shells_for(atoms, name):
    """atoms: [(symbol, (x, y, z) bohr)] -> list of Shell."""
    data = load(name)
    out = []
    for sym, xyz in atoms:
        z = SYMBOLS[sym]
        for sh in data[str(z)]["electron_shells"]:
            exps = [float(e) for e in sh["exponents"]]
            spherical = sh["function_type"] == "gto_spherical"
            for l_idx, l in enumerate(sh["angular_momentum"]):
                # SP-style shells list one coefficient row per angular momentum
                rows = sh["coefficients"] if len(sh["angular_momentum"]) == 1 else [sh["coefficients"][l_idx]]
                cols = [[float(c) for c in row] for row in rows]
                coefs = list(map(list, zip(*cols)))          # (K, ncontr)
                out.append(Shell(xyz, l, exps, coefs, spherical or l >= 2 and sh["function_type"] != "gto_cartesian"))
    return out

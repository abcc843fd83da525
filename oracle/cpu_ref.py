"""ctypes front end of the oracle's C++ CPU arm (TEST INFRASTRUCTURE).

``oracle/cpu_ref.cpp`` restates the reference's host algorithms (per-i BLAS3
RI-MP2 with the adjoint, packed two-pass DF-J, DSYMM/DSYRK DF-K) with OpenMP
over work units and OpenBLAS at one thread per unit; this module builds it
on first use (``oracle.build_cpu_ref``) and exposes:

* ``physical_cores()`` -- the host's physical cores (``lscpu``), limited to
  the CPUs this process may run on;
* ``rimp2_units`` / ``rimp2_energy_grad`` -- units (i, j0, j1) of the RI-MP2
  energy + adjoint, and the whole of it (small cases, for the parity test);
* ``dfj`` / ``dfk`` -- one DF-J and one DF-K build.

Only ``tests/`` and ``bench.py`` (its CPU-baseline leg and reference arm)
use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import build_cpu_ref

_LIB = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int64)


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build_cpu_ref.build())
        L.cr_rimp2_units.restype = ctypes.c_double
        L.cr_rimp2_units.argtypes = [_D, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _D, _D, _I,
                                     ctypes.c_int64, ctypes.c_int, _D, _D, _D]
        L.cr_dfj.restype = ctypes.c_double
        L.cr_dfj.argtypes = [_D, ctypes.c_int64, ctypes.c_int64, _D, _D, ctypes.c_int]
        L.cr_dfk.restype = ctypes.c_double
        L.cr_dfk.argtypes = [_D, ctypes.c_int64, ctypes.c_int64, _D, ctypes.c_int64, ctypes.c_int64, _D,
                             ctypes.c_int]
        _LIB = L
    return _LIB


def physical_cores():
    """Physical cores per ``lscpu -p=core,socket`` among the CPUs this
    process may use (falls back to the affinity count)."""
    allowed = os.sched_getaffinity(0)
    try:
        out = subprocess.run(["lscpu", "-p=cpu,core,socket"], capture_output=True, text=True, check=True).stdout
        cores = set()
        for line in out.splitlines():
            if line.startswith("#"):
                continue
            cpu, core, sock = (int(x) for x in line.split(",")[:3])
            if cpu in allowed:
                cores.add((sock, core))
        if cores:
            return len(cores)
    except (OSError, subprocess.CalledProcessError, ValueError):
        pass
    return len(allowed)


def _d(a):
    return a.ctypes.data_as(_D)


def rimp2_units(b, eo, ev, units, threads, x_out=None, occ_out=True):
    """Run the units (i, j0, j1); returns (seconds, e[nunits, 2], occ[nunits])."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    eo = np.ascontiguousarray(eo, dtype=np.float64)
    ev = np.ascontiguousarray(ev, dtype=np.float64)
    u = np.ascontiguousarray(np.asarray(units, dtype=np.int64).reshape(-1, 3))
    e = np.zeros((len(u), 2))
    occ = np.zeros(len(u)) if occ_out else None
    secs = lib().cr_rimp2_units(_d(b), b.shape[0], len(eo), len(ev), _d(eo), _d(ev), u.ctypes.data_as(_I), len(u),
                                int(threads), _d(e), None if x_out is None else _d(x_out),
                                None if occ is None else _d(occ))
    return secs, e, occ


def rimp2_energy_grad(b, eo, ev, width=4, threads=4):
    """The whole RI-MP2 energy + Gamma + dE/deps_occ through the units (one
    thread per i at a time, so the x_ov updates of one i never overlap)."""
    nocc, nvir = len(eo), len(ev)
    x = np.zeros_like(np.asarray(b, dtype=np.float64))
    e_os = e_ss = 0.0
    d_o = np.zeros(nocc)
    for i in range(nocc):
        units = [(i, j0, min(nocc, j0 + width)) for j0 in range(0, nocc, width)]
        _, e, occ = rimp2_units(b, eo, ev, units, 1, x_out=x)
        e_os += e[:, 0].sum()
        e_ss += e[:, 1].sum()
        d_o[i] = -2.0 * occ.sum()
    return e_os, e_ss, 4.0 * x, d_o


def dfj(bp, d_weights, threads):
    """J (packed) = Bp^T (Bp w); returns (seconds, j_packed)."""
    bp = np.ascontiguousarray(bp, dtype=np.float64)
    w = np.ascontiguousarray(d_weights, dtype=np.float64)
    j = np.zeros(bp.shape[1])
    secs = lib().cr_dfj(_d(bp), bp.shape[0], bp.shape[1], _d(w), _d(j), int(threads))
    return secs, j


def dfk(b, c_occ, threads, qchunk=16):
    """K = sum_Q (B_Q C)(B_Q C)^T on the square tensor; returns (seconds, K)."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    c = np.ascontiguousarray(c_occ, dtype=np.float64)
    n = b.shape[1]
    k = np.zeros((n, n))
    secs = lib().cr_dfk(_d(b), b.shape[0], n, _d(c), c.shape[1], int(qchunk), _d(k), int(threads))
    return secs, k

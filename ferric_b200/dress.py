"""MO transform and metric dressing of the 3-index tensor (the step before the
RI-MP2 path): ``B[P, l*nr + r] = sum_Q M[P, Q] (Q|lr)`` with
``(Q|lr) = C_left^T (Q|mu nu) C_right`` -- stream_dressed_mo_band
(ferric-mp2/src/rimp2.rs:648-737).  ``fc_mo_dress`` / ``fc_mo_dress_dev``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FcStats, PRECISIONS, check, ptr


def mo_dress(eri3, m, c_left, c_right, precision="f64", stats=None, out=None):
    """``eri3`` (naux, n, n) symmetric in the AO pair, ``m`` (naux, naux),
    ``c_left`` (n, nl), ``c_right`` (n, nr); returns B (naux, nl*nr).  NumPy
    arrays use the host API, CUDA float64 tensors the device API."""
    _lib.ensure_init()
    naux, n = int(eri3.shape[0]), int(eri3.shape[1])
    nl, nr = int(c_left.shape[1]), int(c_right.shape[1])
    st = FcStats()
    prec = PRECISIONS[precision]
    if hasattr(eri3, "is_cuda") and eri3.is_cuda:
        import torch
        t, mm, cl, cr = (x.contiguous() for x in (eri3, m, c_left, c_right))
        b = torch.empty((naux, nl * nr), dtype=torch.float64, device=t.device) if out is None else out
        check(_lib.lib.fc_mo_dress_dev(ptr(t), naux, n, ptr(mm), ptr(cl), nl, ptr(cr), nr, prec, ptr(b),
                                       ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream),
                                       ctypes.byref(st)))
    else:
        t, mm, cl, cr = (np.ascontiguousarray(x, dtype=np.float64) for x in (eri3, m, c_left, c_right))
        b = np.empty((naux, nl * nr)) if out is None else out
        check(_lib.lib.fc_mo_dress(ptr(t), naux, n, ptr(mm), ptr(cl), nl, ptr(cr), nr, prec, ptr(b),
                                   ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return b

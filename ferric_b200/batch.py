"""Batched RI-MP2: many molecules of uneven size in one CUDA graph.

The reference loops over molecules, one ``spin_components`` call
(ferric-mp2/src/rimp2.rs:1445-1544) and one adjoint (rimp2.rs:1832-1836)
each.  ``Rimp2Batch`` records the split kernels, the persistent pair and
adjoint kernels over every molecule's tiles, and the reductions into one
graph (``fc_rimp2_batched_create``) and replays it.

Inputs are CUDA float64 tensors that must stay alive (and at the same
address) for the life of the batch; refill them in place and call
``run()`` again for new inputs.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FcBatchInfo, FcMolDesc, PRECISIONS, check


def _dev64(x):
    import torch
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float64):
        raise TypeError("Rimp2Batch takes CUDA float64 tensors")
    return x.contiguous()


class Rimp2Batch:
    """``mols``: sequence of ``(b_ov, eps_occ, eps_vir)`` CUDA float64 tensors
    (b_ov of shape (naux, nocc*nvir)).  ``grad=True`` also produces, per
    molecule, Gamma = dE/dB_ov and dE/deps (``self.gamma``, ``self.de_docc``,
    ``self.de_dvir``: tensors allocated here)."""

    def __init__(self, mols, grad=False, precision="mixed"):
        import torch
        _lib.ensure_init()
        self.grad = bool(grad)
        self._keep = []
        self.shapes = []
        self.gamma, self.de_docc, self.de_dvir = [], [], []
        descs = (FcMolDesc * len(mols))()
        for m, (b, eo, ev) in enumerate(mols):
            b, eo, ev = _dev64(b), _dev64(eo), _dev64(ev)
            nocc, nvir = int(eo.numel()), int(ev.numel())
            naux = int(b.shape[0])
            if b.dim() != 2 or b.shape[1] != nocc * nvir:
                raise ValueError(f"molecule {m}: b_ov must be (naux, nocc*nvir)")
            self._keep += [b, eo, ev]
            d = descs[m]
            d.b_ov, d.eps_occ, d.eps_vir = b.data_ptr(), eo.data_ptr(), ev.data_ptr()
            d.naux, d.nocc, d.nvir = naux, nocc, nvir
            if self.grad:
                g = torch.empty((naux, nocc * nvir), dtype=torch.float64, device=b.device)
                go = torch.empty(nocc, dtype=torch.float64, device=b.device)
                gv = torch.empty(nvir, dtype=torch.float64, device=b.device)
                self.gamma.append(g)
                self.de_docc.append(go)
                self.de_dvir.append(gv)
                d.gamma, d.de_deps_occ, d.de_deps_vir = g.data_ptr(), go.data_ptr(), gv.data_ptr()
            self.shapes.append((naux, nocc, nvir))
        torch.cuda.synchronize()
        self.nmol = len(mols)
        h = ctypes.c_void_p()
        check(_lib.lib.fc_rimp2_batched_create(descs, self.nmol, PRECISIONS[precision], ctypes.byref(h)))
        self._h = h

    def run(self, stream=None):
        """Enqueue one replay (``stream``: a torch.cuda.Stream, or None for the batch's own)."""
        s = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        check(_lib.lib.fc_rimp2_batched_replay(self._h, s))

    def energies(self):
        """(e_os, e_ss) numpy arrays of the last replay (waits for it)."""
        eo = np.zeros(self.nmol)
        es = np.zeros(self.nmol)
        check(_lib.lib.fc_rimp2_batched_energies(
            self._h, eo.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            es.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return eo, es

    def info(self):
        r = FcBatchInfo()
        check(_lib.lib.fc_rimp2_batched_info(self._h, ctypes.byref(r)))
        return r.as_dict()

    def plan(self):
        """Per size bucket: tile shape, the diagonal-tile exchange choice and
        whether it was measured (autotuner), defaulted or forced."""
        import json
        n = _lib.lib.fc_rimp2_batched_plan(self._h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        _lib.lib.fc_rimp2_batched_plan(self._h, buf, n + 1)
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib.fc_rimp2_batched_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

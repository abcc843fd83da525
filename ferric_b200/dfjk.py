"""DF-J / DF-K builders on the B200, behind the reference's builder traits.

``DfJ`` and ``DfK`` follow ``JBuilder`` / ``KBuilder`` (ferric-scf/src/fock.rs:10-52):
``build(d, j)`` writes J into the caller's (zeroed) matrix, ``build_from_occ(c_occ, k)``
writes ``K = sum_Q (B_Q C)(B_Q C)^T`` with no occupation factor, ``reset()`` is a
no-op.  Both hold one device-resident tensor (the reference's per-builder
``DeviceSlot``, ferric-scf/src/df_j_gpu.rs:1-5, df_k_gpu.rs:1-4); the tensor is
uploaded once at construction and only D / C_occ / J / K cross per build.

NumPy arguments use the host API; CUDA torch tensors use the device API on
the current stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FcStats, LAYOUTS, PRECISIONS, check, ptr


def _prec(p):
    return p if isinstance(p, int) else PRECISIONS[p]


class DfJK:
    """One device-resident 3-index tensor shared by J and K builds.

    ``b``: ``(naux, n, n)`` symmetric (``layout="square"``) or
    ``(naux, n(n+1)/2)`` packed lower rows (``layout="packed_lower"``, J only).
    ``metric_chol``: the lower Cholesky factor of the Coulomb metric for the
    raw ``(P|mn)`` form (``DfJ``, ferric-scf/src/df_j.rs:931); ``None`` for a
    dressed tensor.
    """

    def __init__(self, b, n=None, layout="square", precision="f64", metric_chol=None):
        _lib.ensure_init()
        self.layout = layout
        self.precision = precision
        self.naux = int(b.shape[0])
        if layout == "square":
            self.n = int(b.shape[1])
        else:
            if n is None:
                raise ValueError("packed_lower layout needs n")
            self.n = int(n)
        h = ctypes.c_void_p()
        if hasattr(b, "is_cuda") and b.is_cuda:
            import torch
            bb = b.contiguous()
            check(_lib.lib.fc_dfjk_create_dev(ptr(bb), self.naux, self.n, LAYOUTS[layout], _prec(precision),
                                              ctypes.c_void_p(torch.cuda.current_stream(bb.device).cuda_stream),
                                              ctypes.byref(h)))
        else:
            bb = np.ascontiguousarray(b, dtype=np.float64)
            check(_lib.lib.fc_dfjk_create(ptr(bb), self.naux, self.n, LAYOUTS[layout], _prec(precision),
                                          ctypes.byref(h)))
        self._h = h
        self.active = precision
        if metric_chol is not None:
            lc = np.ascontiguousarray(metric_chol, dtype=np.float64)
            check(_lib.lib.fc_dfj_set_metric_chol(self._h, ptr(lc)))

    def set_precision(self, precision):
        """Precision of the next builds: "f64" always, or the handle's own
        mixed precision (``fc_dfjk_set_precision``)."""
        check(_lib.lib.fc_dfjk_set_precision(self._h, _prec(precision)))
        self.active = precision

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib.fc_dfjk_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def j(self, d, out=None, stats=None):
        st = FcStats()
        if hasattr(d, "is_cuda") and d.is_cuda:
            import torch
            dd = d.contiguous()
            out = torch.empty_like(dd) if out is None else out
            check(_lib.lib.fc_dfj_build_dev(self._h, ptr(dd), ptr(out),
                                            ctypes.c_void_p(torch.cuda.current_stream(dd.device).cuda_stream),
                                            ctypes.byref(st)))
        else:
            dd = np.ascontiguousarray(d, dtype=np.float64)
            out = np.empty_like(dd) if out is None else out
            check(_lib.lib.fc_dfj_build(self._h, ptr(dd), ptr(out), ctypes.byref(st)))
        if stats is not None:
            stats.update(st.as_dict())
        return out

    def k_from_occ(self, c_occ, out=None, stats=None):
        st = FcStats()
        nocc = int(c_occ.shape[1])
        if hasattr(c_occ, "is_cuda") and c_occ.is_cuda:
            import torch
            cc = c_occ.contiguous()
            out = torch.empty((self.n, self.n), dtype=torch.float64, device=cc.device) if out is None else out
            check(_lib.lib.fc_dfk_build_occ_dev(self._h, ptr(cc), nocc, ptr(out),
                                                ctypes.c_void_p(torch.cuda.current_stream(cc.device).cuda_stream),
                                                ctypes.byref(st)))
        else:
            cc = np.ascontiguousarray(c_occ, dtype=np.float64)
            out = np.empty((self.n, self.n)) if out is None else out
            check(_lib.lib.fc_dfk_build_occ(self._h, ptr(cc), nocc, ptr(out), ctypes.byref(st)))
        if stats is not None:
            stats.update(st.as_dict())
        return out


    def jk_from_occ(self, c_occ, out=None, stats=None):
        """``(J, K)`` of one occupied-orbital matrix in one call
        (``fc_dfjk_build_occ``): K as ``k_from_occ`` and J = J(C C^T), J's
        first pass taken from K's stage-1 product.  ``out``: optional (J, K)
        buffers."""
        st = FcStats()
        nocc = int(c_occ.shape[1])
        if hasattr(c_occ, "is_cuda") and c_occ.is_cuda:
            import torch
            cc = c_occ.contiguous()
            if out is None:
                out = tuple(torch.empty((self.n, self.n), dtype=torch.float64, device=cc.device) for _ in range(2))
            check(_lib.lib.fc_dfjk_build_occ_dev(self._h, ptr(cc), nocc, ptr(out[0]), ptr(out[1]),
                                                 ctypes.c_void_p(torch.cuda.current_stream(cc.device).cuda_stream),
                                                 ctypes.byref(st)))
        else:
            cc = np.ascontiguousarray(c_occ, dtype=np.float64)
            if out is None:
                out = (np.empty((self.n, self.n)), np.empty((self.n, self.n)))
            check(_lib.lib.fc_dfjk_build_occ(self._h, ptr(cc), nocc, ptr(out[0]), ptr(out[1]), ctypes.byref(st)))
        if stats is not None:
            stats.update(st.as_dict())
        return out


class DfJ:
    """``JBuilder`` over a device-resident tensor (``DfJ``, ferric-scf/src/df_j.rs:127)."""

    def __init__(self, b, n=None, layout="packed_lower", precision="f64", metric_chol=None, shared=None):
        self.jk = shared if shared is not None else DfJK(b, n=n, layout=layout, precision=precision,
                                                          metric_chol=metric_chol)

    def build(self, d, j):
        """Build J of density ``d`` into ``j`` (returns 0 ERI quartets, as DF builders do)."""
        j[...] = self.jk.j(d)
        return 0

    def reset(self):
        pass


class DfK:
    """``KBuilder`` over a device-resident dressed tensor (``DfK``, ferric-scf/src/df_k.rs:299)."""

    def __init__(self, b, precision="f64", shared=None):
        self.jk = shared if shared is not None else DfJK(b, layout="square", precision=precision)

    def build_from_occ(self, c_occ, k):
        if c_occ.shape[0] != self.jk.n:
            raise ValueError(f"DfK::build_from_occ: c_occ rows ({c_occ.shape[0]}) != nao ({self.jk.n})")
        k[...] = self.jk.k_from_occ(c_occ)
        return 0

    def build(self, d, k):
        """Density path: K of a symmetric positive semi-definite ``d`` through its
        occupied factorisation ``d = C C^T`` (eigen-decomposition, FP64)."""
        w, v = np.linalg.eigh(np.asarray(d, dtype=np.float64))
        keep = w > 1e-14 * max(1.0, float(np.abs(w).max()))
        if np.any(w < -1e-12 * max(1.0, float(np.abs(w).max()))):
            raise ValueError("DfK.build: density is not positive semi-definite; use build_from_occ")
        c = v[:, keep] * np.sqrt(w[keep])
        return self.build_from_occ(c, k)

    def update_density(self, *_):
        pass

    def reset(self):
        pass

"""RI-MP2 on the B200, behind the reference's own entry points.

Mirrors, with the same argument meaning:

* ``spin_components_from_b_ov_kappa`` / ``try_spin_components_on_device``
  (ferric-mp2/src/rimp2.rs:1330-1375, rimp2_gpu.rs:105-170):
  ``b_ov`` (naux, nocc*nvir) with column ``i*nvir + a``, the full MO-energy
  vector ``eps`` indexed ``first_occ + i`` / ``nocc_total + a``, optional
  ``kappa``.  ``try_*`` returns ``None`` when the device declines (the
  reference's "run the CPU path"), with the reason counted in ``STATS``;
  the plain form raises :class:`FcError`.
* ``Mp2Intermediates::from_ri_densities`` inputs (rimp2.rs:1841-1883):
  :func:`rimp2_energy_grad` returns ``Gamma = dE/dB = 4 x_ov`` and
  ``dE/d eps`` (``2 diag(P_oo)``, ``2 diag(P_vv)``) without storing amplitudes;
  :func:`rimp2_energy_grad_dens` adds the full unrelaxed ``P_oo`` / ``P_vv``
  of ``build_mp2_density`` (ferric-mp2/src/oo_rimp2.rs:1170-1300), and
  :func:`ri_densities` returns exactly ``(x_ov, p_oo, p_vv, e_corr)``.

Inputs may be NumPy arrays (host API: the library copies) or CUDA torch
tensors (device API on torch's current stream).
"""
from __future__ import annotations

import collections
import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import FcError, FcStats, PRECISIONS, check, ptr

STATS = collections.Counter()


@dataclass
class SpinComponents:
    """``SpinComponents`` (ferric-mp2/src/rimp2.rs:134-141)."""
    e_os: float
    e_ss: float
    e_total: float


def _precision(p):
    if isinstance(p, int):
        return p
    try:
        return PRECISIONS[p]
    except KeyError as exc:
        raise ValueError(f"unknown precision {p!r}; expected one of {sorted(PRECISIONS)}") from exc


def _is_torch_cuda(x):
    return hasattr(x, "is_cuda") and x.is_cuda


def _stream_of(x):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)


def _split_eps(eps, nocc, nvir, first_occ, nocc_total):
    if nocc_total is None:
        nocc_total = first_occ + nocc
    return eps[first_occ:first_occ + nocc], eps[nocc_total:nocc_total + nvir]


def rimp2_energy(b_ov, eps_occ, eps_vir, kappa=None, precision="f64", stats=None):
    """``(e_os, e_ss)`` for ``b_ov`` and the active orbital energies.

    NumPy inputs use the host API; CUDA tensors (float64, contiguous) use
    the device API on the current stream.
    """
    _lib.ensure_init()
    nocc, nvir = int(eps_occ.shape[0]), int(eps_vir.shape[0])
    naux = int(b_ov.shape[0])
    if b_ov.shape[1] != nocc * nvir:
        raise ValueError(f"b_ov has {b_ov.shape[1]} columns, expected nocc*nvir = {nocc * nvir}")
    eo, es = ctypes.c_double(), ctypes.c_double()
    st = FcStats()
    prec = _precision(precision)
    hk, kv = (0, 0.0) if kappa is None else (1, float(kappa))
    if _is_torch_cuda(b_ov):
        b, o, v = (t.contiguous() for t in (b_ov, eps_occ, eps_vir))
        for t in (b, o, v):
            if t.dtype != __import__("torch").float64:
                raise TypeError("device inputs must be float64")
        check(_lib.lib.fc_rimp2_energy_dev(ptr(b), naux, nocc, nvir, ptr(o), ptr(v), hk, kv, prec,
                                           ctypes.byref(eo), ctypes.byref(es), _stream_of(b),
                                           ctypes.byref(st)))
    else:
        b = np.ascontiguousarray(b_ov, dtype=np.float64)
        o = np.ascontiguousarray(eps_occ, dtype=np.float64)
        v = np.ascontiguousarray(eps_vir, dtype=np.float64)
        check(_lib.lib.fc_rimp2_energy(ptr(b), naux, nocc, nvir, ptr(o), ptr(v), hk, kv, prec,
                                       ctypes.byref(eo), ctypes.byref(es), ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return eo.value, es.value


def spin_components_on_device(b_ov, eps, nocc, nvir, first_occ=0, nocc_total=None, kappa=None,
                              precision="f64", stats=None):
    """Device spin components; raises :class:`FcError` when the device cannot run
    (``spin_components_on_device``, ferric-mp2/src/rimp2_gpu.rs:198)."""
    if len(eps) < (first_occ + nocc if nocc_total is None else nocc_total) + nvir:
        raise ValueError("eps is shorter than nocc_total + nvir")
    eo, ev = _split_eps(eps, nocc, nvir, first_occ, nocc_total)
    e_os, e_ss = rimp2_energy(b_ov, eo, ev, kappa=kappa, precision=precision, stats=stats)
    return SpinComponents(e_os, e_ss, e_os + e_ss)


def try_spin_components_on_device(b_ov, eps, nocc, nvir, first_occ=0, nocc_total=None, kappa=None,
                                  mixed_ok=False, stats=None):
    """Dispatcher: ``None`` means "run the CPU path", with the reason counted.

    Same contract as ``try_spin_components_on_device``
    (ferric-mp2/src/rimp2_gpu.rs:105-170): mixed runs only when ``mixed_ok``
    and no kappa; a mixed kernel failure (``FC_ERR_KERNEL``/``FC_ERR_RANGE``)
    is retried in FP64 on the device, counted, never silent.
    """
    precision = "mixed" if (mixed_ok and kappa is None) else "f64"
    try:
        return spin_components_on_device(b_ov, eps, nocc, nvir, first_occ, nocc_total, kappa,
                                         precision, stats)
    except FcError as e:
        if precision != "f64" and e.name in ("FC_ERR_KERNEL", "FC_ERR_RANGE"):
            STATS[f"mixed_fallback:{e.name}"] += 1
            try:
                return spin_components_on_device(b_ov, eps, nocc, nvir, first_occ, nocc_total,
                                                 kappa, "f64", stats)
            except FcError as e2:
                STATS[f"cpu:{e2.name}"] += 1
                return None
        STATS[f"cpu:{e.name}"] += 1
        return None


def rimp2_energy_grad(b_ov, eps_occ, eps_vir, precision="f64", stats=None, out=None):
    """``(SpinComponents, gamma, de_docc, de_dvir)``.

    ``gamma[P, ia] = dE/dB[P, ia]`` (= 4 x_ov, ferric-mp2/src/rimp2.rs:1832-1836),
    ``de_docc[i] = dE/d eps_occ[i]``, ``de_dvir[a] = dE/d eps_vir[a]``.
    """
    _lib.ensure_init()
    nocc, nvir = int(eps_occ.shape[0]), int(eps_vir.shape[0])
    naux = int(b_ov.shape[0])
    if b_ov.shape[1] != nocc * nvir:
        raise ValueError(f"b_ov has {b_ov.shape[1]} columns, expected nocc*nvir = {nocc * nvir}")
    eo, es = ctypes.c_double(), ctypes.c_double()
    st = FcStats()
    prec = _precision(precision)
    if _is_torch_cuda(b_ov):
        import torch
        b, o, v = (t.contiguous() for t in (b_ov, eps_occ, eps_vir))
        if out is None:
            gamma = torch.empty_like(b)
            d_o = torch.empty_like(o)
            d_v = torch.empty_like(v)
        else:
            gamma, d_o, d_v = out
        check(_lib.lib.fc_rimp2_energy_grad_dev(
            ptr(b), naux, nocc, nvir, ptr(o), ptr(v), prec, ctypes.byref(eo), ctypes.byref(es),
            ptr(gamma), ptr(d_o), ptr(d_v), _stream_of(b), ctypes.byref(st)))
    else:
        b = np.ascontiguousarray(b_ov, dtype=np.float64)
        o = np.ascontiguousarray(eps_occ, dtype=np.float64)
        v = np.ascontiguousarray(eps_vir, dtype=np.float64)
        gamma = np.empty_like(b)
        d_o = np.empty(nocc)
        d_v = np.empty(nvir)
        check(_lib.lib.fc_rimp2_energy_grad(
            ptr(b), naux, nocc, nvir, ptr(o), ptr(v), prec, ctypes.byref(eo), ctypes.byref(es),
            ptr(gamma), ptr(d_o), ptr(d_v), ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return SpinComponents(eo.value, es.value, eo.value + es.value), gamma, d_o, d_v


def rimp2_energy_grad_dens(b_ov, eps_occ, eps_vir, precision="f64", stats=None):
    """``(SpinComponents, gamma, de_docc, de_dvir, p_oo, p_vv)``: as
    :func:`rimp2_energy_grad` plus the unrelaxed MP2 densities
    ``p_oo[i, j] = -sum_kab t_ik^ab (2 t_jk^ab - t_jk^ba)`` and
    ``p_vv[a, b] = sum_ijc t_ij^ac (2 t_ij^bc - t_ij^cb)``
    (build_mp2_density, ferric-mp2/src/oo_rimp2.rs:1170-1300)."""
    _lib.ensure_init()
    nocc, nvir = int(eps_occ.shape[0]), int(eps_vir.shape[0])
    naux = int(b_ov.shape[0])
    if b_ov.shape[1] != nocc * nvir:
        raise ValueError(f"b_ov has {b_ov.shape[1]} columns, expected nocc*nvir = {nocc * nvir}")
    eo, es = ctypes.c_double(), ctypes.c_double()
    st = FcStats()
    prec = _precision(precision)
    if _is_torch_cuda(b_ov):
        import torch
        b, o, v = (t.contiguous() for t in (b_ov, eps_occ, eps_vir))
        gamma, d_o, d_v = torch.empty_like(b), torch.empty_like(o), torch.empty_like(v)
        p_oo = torch.empty((nocc, nocc), dtype=torch.float64, device=b.device)
        p_vv = torch.empty((nvir, nvir), dtype=torch.float64, device=b.device)
        check(_lib.lib.fc_rimp2_energy_grad_dens_dev(
            ptr(b), naux, nocc, nvir, ptr(o), ptr(v), prec, ctypes.byref(eo), ctypes.byref(es),
            ptr(gamma), ptr(d_o), ptr(d_v), ptr(p_oo), ptr(p_vv), _stream_of(b), ctypes.byref(st)))
    else:
        b = np.ascontiguousarray(b_ov, dtype=np.float64)
        o = np.ascontiguousarray(eps_occ, dtype=np.float64)
        v = np.ascontiguousarray(eps_vir, dtype=np.float64)
        gamma, d_o, d_v = np.empty_like(b), np.empty(nocc), np.empty(nvir)
        p_oo, p_vv = np.empty((nocc, nocc)), np.empty((nvir, nvir))
        check(_lib.lib.fc_rimp2_energy_grad_dens(
            ptr(b), naux, nocc, nvir, ptr(o), ptr(v), prec, ctypes.byref(eo), ctypes.byref(es),
            ptr(gamma), ptr(d_o), ptr(d_v), ptr(p_oo), ptr(p_vv), ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return SpinComponents(eo.value, es.value, eo.value + es.value), gamma, d_o, d_v, p_oo, p_vv


def ri_densities(b_ov, eps_occ, eps_vir, precision="f64"):
    """``(x_ov, p_oo, p_vv, e_corr)``: the arguments
    ``Mp2Intermediates::from_ri_densities`` takes after ``rpa``
    (rimp2.rs:1841-1883), with ``x_ov = Gamma / 4``."""
    sc, gamma, _, _, p_oo, p_vv = rimp2_energy_grad_dens(b_ov, eps_occ, eps_vir, precision)
    return gamma / 4.0, p_oo, p_vv, sc.e_total


def ump2_energy(b_a, eps_occ_a, eps_vir_a, b_b, eps_occ_b, eps_vir_b, precision="f64", stats=None):
    """Unrestricted RI-MP2 energy components ``(e_aa, e_bb, e_ab)``
    (same_spin_block_energy / opposite_spin_block_energy,
    ferric-mp2/src/u_rimp2.rs:693-753); SCS/SOS weighting is the caller's."""
    _lib.ensure_init()
    noa, nva, nob, nvb = (int(x.shape[0]) for x in (eps_occ_a, eps_vir_a, eps_occ_b, eps_vir_b))
    naux = int(b_a.shape[0])
    if b_b.shape[0] != naux:
        raise ValueError("b_a and b_b must share naux")
    e1, e2, e3 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    st = FcStats()
    prec = _precision(precision)
    if _is_torch_cuda(b_a):
        ts = [t.contiguous() for t in (b_a, eps_occ_a, eps_vir_a, b_b, eps_occ_b, eps_vir_b)]
        check(_lib.lib.fc_ump2_energy_dev(ptr(ts[0]), noa, nva, ptr(ts[1]), ptr(ts[2]), ptr(ts[3]), nob, nvb,
                                          ptr(ts[4]), ptr(ts[5]), naux, prec, ctypes.byref(e1), ctypes.byref(e2),
                                          ctypes.byref(e3), _stream_of(ts[0]), ctypes.byref(st)))
    else:
        ts = [np.ascontiguousarray(x, dtype=np.float64)
              for x in (b_a, eps_occ_a, eps_vir_a, b_b, eps_occ_b, eps_vir_b)]
        check(_lib.lib.fc_ump2_energy(ptr(ts[0]), noa, nva, ptr(ts[1]), ptr(ts[2]), ptr(ts[3]), nob, nvb,
                                      ptr(ts[4]), ptr(ts[5]), naux, prec, ctypes.byref(e1), ctypes.byref(e2),
                                      ctypes.byref(e3), ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return e1.value, e2.value, e3.value


def rimp2_imat(x_ov, b_full, nocc, nvir, first_occ=0, precision="f64", stats=None):
    """RI Lagrangian Imat (nmo x nmo) from x_ov = Gamma / 4 and the dressed MO
    3-index tensor b_full (naux, nmo, nmo) (build_imat_ri,
    ferric-mp2/src/zvector.rs:735-832)."""
    _lib.ensure_init()
    naux, nmo = int(b_full.shape[0]), int(b_full.shape[1])
    st = FcStats()
    prec = _precision(precision)
    if _is_torch_cuda(b_full):
        import torch
        x, b = x_ov.contiguous(), b_full.contiguous()
        out = torch.empty((nmo, nmo), dtype=torch.float64, device=b.device)
        check(_lib.lib.fc_rimp2_imat_dev(ptr(x), ptr(b), naux, nmo, nocc, nvir, first_occ, prec, ptr(out),
                                         _stream_of(b), ctypes.byref(st)))
    else:
        x = np.ascontiguousarray(x_ov, dtype=np.float64)
        b = np.ascontiguousarray(b_full, dtype=np.float64)
        out = np.empty((nmo, nmo))
        check(_lib.lib.fc_rimp2_imat(ptr(x), ptr(b), naux, nmo, nocc, nvir, first_occ, prec, ptr(out),
                                     ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return out


def rimp2_response_2c(x_ov, b_ov, v_inv_sqrt, weight=2.0, stats=None):
    """``(y_ov, gamma_2c)`` of the RI 3c/2c response for one channel
    (ferric-mp2/src/gradient.rs:559-887): ``y_ov = V^{-1/2 T} x_ov`` and
    ``gamma_2c = -w (V^{-1/2 T} b_ov) y_ov^T``, FP64."""
    _lib.ensure_init()
    naux, nov = int(x_ov.shape[0]), int(x_ov.shape[1])
    st = FcStats()
    if _is_torch_cuda(x_ov):
        import torch
        x, b, v = (t.contiguous() for t in (x_ov, b_ov, v_inv_sqrt))
        y = torch.empty_like(x)
        g = torch.empty((naux, naux), dtype=torch.float64, device=x.device)
        check(_lib.lib.fc_rimp2_response_2c_dev(ptr(x), ptr(b), ptr(v), naux, nov, float(weight), ptr(y), ptr(g),
                                                _stream_of(x), ctypes.byref(st)))
    else:
        x, b, v = (np.ascontiguousarray(t, dtype=np.float64) for t in (x_ov, b_ov, v_inv_sqrt))
        y = np.empty_like(x)
        g = np.empty((naux, naux))
        check(_lib.lib.fc_rimp2_response_2c(ptr(x), ptr(b), ptr(v), naux, nov, float(weight), ptr(y), ptr(g),
                                            ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return y, g


def rimp2_response_3c(y_ov, c_occ, c_vir, p0=0, np_=None, weight=2.0, stats=None):
    """The 3-centre weight ``g3c[P] = w (G_P + G_P^T)``, ``G_P = C_occ Y_P
    C_vir^T``, for the aux slab ``[p0, p0 + np_)`` (np_, nbf, nbf)
    (ferric-mp2/src/gradient.rs:772-804), FP64."""
    _lib.ensure_init()
    naux = int(y_ov.shape[0])
    nbf, nocc = int(c_occ.shape[0]), int(c_occ.shape[1])
    nvir = int(c_vir.shape[1])
    np_ = naux - p0 if np_ is None else int(np_)
    st = FcStats()
    if _is_torch_cuda(y_ov):
        import torch
        y, co, cv = (t.contiguous() for t in (y_ov, c_occ, c_vir))
        out = torch.empty((np_, nbf, nbf), dtype=torch.float64, device=y.device)
        check(_lib.lib.fc_rimp2_response_3c_dev(ptr(y), ptr(co), ptr(cv), naux, nocc, nvir, nbf, p0, np_,
                                                float(weight), ptr(out), _stream_of(y), ctypes.byref(st)))
    else:
        y, co, cv = (np.ascontiguousarray(t, dtype=np.float64) for t in (y_ov, c_occ, c_vir))
        out = np.empty((np_, nbf, nbf))
        check(_lib.lib.fc_rimp2_response_3c(ptr(y), ptr(co), ptr(cv), naux, nocc, nvir, nbf, p0, np_, float(weight),
                                            ptr(out), ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return out

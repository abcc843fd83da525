"""One RI-MP2 system or DF-JK build over the processes of a torch.distributed
group, one GPU each (NCCL over NVLink in production; any backend works for
the composition).

RI-MP2 (energy, or energy + Gamma + dE/deps): every process holds all of
B_ov and computes a balanced share of the occupied pairs
(``fc_rimp2_*_shard_dev``); the results are sums over the shares, so the
only collectives are on them -- one all-reduce of the scalars and dE/deps,
and a reduce-scatter of Gamma by aux rows (each process keeps its band, as
the next step of an analytic gradient wants) or an all-reduce of the whole
Gamma.  The reference's MPI path (ferric-mp2/src/mpi_rimp2.rs:16-43) cuts
aux bands and all-reduces per-i intermediates instead.

DF-JK: each process holds an aux band of B (the reference's partition,
ferric-scf/src/parallel.rs:215-231) and all-reduces its J and K (df_j.rs:101-115,
df_k.rs:1522-1526); dressed tensors only (no metric solve across bands).

Collectives run on the tensors' devices in a fixed order on every rank; their
summation order is the backend's.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FcStats, PRECISIONS, check, ptr


def _prec(p):
    return p if isinstance(p, int) else PRECISIONS[p]


def shard_pairs(nocc, nvir, shard, nshards, precision="mixed", grad=True):
    """The occupied pairs (i <= j), as an (n, 2) int32 array, that shard
    ``shard`` of ``nshards`` computes (host only: no GPU needed)."""
    n = ctypes.c_int64()
    args = (int(nocc), int(nvir), _prec(precision), int(bool(grad)), int(shard), int(nshards))
    check(_lib.lib.fc_rimp2_shard_pairs(*args, None, 0, ctypes.byref(n)))
    out = np.zeros((max(1, n.value), 2), dtype=np.int32)
    check(_lib.lib.fc_rimp2_shard_pairs(*args, ptr(out), n.value, ctypes.byref(n)))
    return out[:n.value]


def aux_band(naux, rank, world):
    """Aux rows [lo, hi) of band ``rank`` of ``world`` (equal bands, the last
    one shorter)."""
    nb = -(-naux // world)
    return min(naux, rank * nb), min(naux, (rank + 1) * nb)


def rimp2_energy_shard(b_ov, eps_occ, eps_vir, shard, nshards, precision="mixed"):
    """This shard's partial (E_os, E_ss) for device tensors (CUDA torch)."""
    import torch
    e_os, e_ss = ctypes.c_double(), ctypes.c_double()
    naux, nov = b_ov.shape
    nocc, nvir = eps_occ.numel(), eps_vir.numel()
    stream = torch.cuda.current_stream(b_ov.device).cuda_stream
    check(_lib.lib.fc_rimp2_energy_shard_dev(ptr(b_ov), naux, nocc, nvir, ptr(eps_occ), ptr(eps_vir), 0, 0.0,
                                             _prec(precision), int(shard), int(nshards), ctypes.byref(e_os),
                                             ctypes.byref(e_ss), ctypes.c_void_p(stream), None))
    return e_os.value, e_ss.value


def rimp2_energy_grad_shard(b_ov, eps_occ, eps_vir, shard, nshards, precision="mixed", stats=None):
    """This shard's partial (E_os, E_ss, Gamma, dE/deps_occ, dE/deps_vir) for
    device tensors; Gamma is the full (naux, nocc*nvir) array holding only this
    shard's contributions."""
    import torch
    b_ov = b_ov.contiguous()
    naux, nov = b_ov.shape
    nocc, nvir = eps_occ.numel(), eps_vir.numel()
    gamma = torch.empty_like(b_ov)
    d_o = torch.empty_like(eps_occ)
    d_v = torch.empty_like(eps_vir)
    e_os, e_ss = ctypes.c_double(), ctypes.c_double()
    st = FcStats()
    stream = torch.cuda.current_stream(b_ov.device).cuda_stream
    check(_lib.lib.fc_rimp2_energy_grad_shard_dev(ptr(b_ov), naux, nocc, nvir, ptr(eps_occ), ptr(eps_vir),
                                                  _prec(precision), int(shard), int(nshards), ctypes.byref(e_os),
                                                  ctypes.byref(e_ss), ptr(gamma), ptr(d_o), ptr(d_v),
                                                  ctypes.c_void_p(stream), ctypes.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return e_os.value, e_ss.value, gamma, d_o, d_v


def combine_shards(e_os, e_ss, gamma, de_docc, de_dvir, group=None, gamma_layout="band"):
    """Sum the shards' partials over ``group``: one all-reduce of
    [E_os, E_ss, dE/deps_occ, dE/deps_vir] and, for Gamma, a reduce-scatter by
    aux rows (``gamma_layout="band"``: this rank gets rows ``aux_band(...)``,
    returned with their offset) or an all-reduce (``"full"``).

    Returns ``(e_os, e_ss, gamma_out, row0, de_docc, de_dvir)``."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nocc, nvir = de_docc.numel(), de_dvir.numel()
    vec = torch.cat([torch.tensor([e_os, e_ss], dtype=torch.float64, device=de_docc.device),
                     de_docc.reshape(-1), de_dvir.reshape(-1)])
    dist.all_reduce(vec, group=group)
    naux = gamma.shape[0]
    if gamma_layout == "full":
        dist.all_reduce(gamma, group=group)
        g_out, row0 = gamma, 0
    elif gamma_layout == "band":
        nb = -(-naux // world)
        src = gamma
        if nb * world != naux:  # equal bands for the collective; the padding rows are zero
            src = torch.zeros((nb * world, gamma.shape[1]), dtype=gamma.dtype, device=gamma.device)
            src[:naux] = gamma
        band = torch.empty((nb, gamma.shape[1]), dtype=gamma.dtype, device=gamma.device)
        dist.reduce_scatter_tensor(band, src.contiguous(), group=group)
        lo, hi = aux_band(naux, rank, world)
        g_out, row0 = band[:hi - lo], lo
    else:
        raise ValueError("gamma_layout is 'band' or 'full'")
    return (float(vec[0]), float(vec[1]), g_out, row0, vec[2:2 + nocc].clone(), vec[2 + nocc:].clone())


def rimp2_energy_grad_sharded(b_ov, eps_occ, eps_vir, precision="mixed", group=None, gamma_layout="band"):
    """E, Gamma and dE/deps of one system over the ranks of ``group`` (each
    rank passes the same B_ov, eps on its own GPU).  Returns
    ``(e_os, e_ss, gamma_band_or_full, row0, de_docc, de_dvir)``."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    part = rimp2_energy_grad_shard(b_ov, eps_occ, eps_vir, rank, world, precision)
    return combine_shards(*part, group=group, gamma_layout=gamma_layout)


def rimp2_energy_sharded(b_ov, eps_occ, eps_vir, precision="mixed", group=None):
    """(E_os, E_ss) of one system over the ranks of ``group``."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    e = rimp2_energy_shard(b_ov, eps_occ, eps_vir, rank, world, precision)
    vec = torch.tensor(e, dtype=torch.float64, device=b_ov.device)
    dist.all_reduce(vec, group=group)
    return float(vec[0]), float(vec[1])


class DfJKShard:
    """A DF-JK builder over the aux band this rank holds: ``j(d)`` and
    ``k_from_occ(c)`` return the whole J and K, all-reduced over ``group``.
    ``b_band`` is (naux_band, n, n) on this rank's GPU (a dressed tensor)."""

    def __init__(self, b_band, precision="f64", group=None):
        from .dfjk import DfJK
        self.group = group
        self.jk = DfJK(b_band, layout="square", precision=precision)

    def j(self, d):
        import torch.distributed as dist
        j = self.jk.j(d)
        dist.all_reduce(j, group=self.group)
        return j

    def k_from_occ(self, c_occ):
        import torch.distributed as dist
        k = self.jk.k_from_occ(c_occ)
        dist.all_reduce(k, group=self.group)
        return k

    def close(self):
        self.jk.close()

"""ctypes binding of libferric_cuda.so (the C ABI declared in include/ferric_cuda.h).

Loading is strict: a missing or unloadable library raises ``ImportError`` --
there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FERRIC_CUDA_LIB", os.path.join(_HERE, "libferric_cuda.so"))

FC_OK = 0
STATUS_NAMES = {
    0: "FC_OK", 1: "FC_ERR_DRIVER", 2: "FC_ERR_BLAS", 3: "FC_ERR_DEVICE", 4: "FC_ERR_POOL_FULL",
    5: "FC_ERR_LAYOUT", 6: "FC_ERR_CUDA", 7: "FC_ERR_KERNEL", 8: "FC_ERR_RANGE", 9: "FC_ERR_TIMEOUT",
    10: "FC_ERR_INVALID",
}
PRECISIONS = {"f64": 0, "mixed": 1, "mixed_fast": 2}
LAYOUTS = {"square": 0, "packed_lower": 1}

# Every symbol include/ferric_cuda.h declares, with its ctypes signature.
_c = ctypes
_P = _c.c_void_p
_I64 = _c.c_int64
_I32 = _c.c_int32
_D = _c.c_double
_DP = _c.POINTER(_c.c_double)
SIGNATURES = {
    "fc_init": (_I32, [_I32, _c.c_uint64]),
    "fc_release_workspace": (_I32, []),
    "fc_pool_used": (_c.c_uint64, []),
    "fc_check_recip": (_I32, [_P, _I64, _P]),
    "fc_last_error": (_c.c_size_t, [_c.c_char_p, _c.c_size_t]),
    "fc_version": (_c.c_char_p, []),
    "fc_rimp2_energy": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _D, _I32, _DP, _DP, _P]),
    "fc_rimp2_energy_dev": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _D, _I32, _DP, _DP, _P, _P]),
    "fc_rimp2_energy_grad": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _DP, _DP, _P, _P, _P, _P]),
    "fc_rimp2_energy_grad_dev": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _DP, _DP, _P, _P, _P, _P, _P]),
    "fc_rimp2_response_2c": (_I32, [_P, _P, _P, _I64, _I64, _D, _P, _P, _P]),
    "fc_rimp2_response_2c_dev": (_I32, [_P, _P, _P, _I64, _I64, _D, _P, _P, _P, _P]),
    "fc_rimp2_response_3c": (_I32, [_P, _P, _P, _I64, _I64, _I64, _I64, _I64, _I64, _D, _P, _P]),
    "fc_rimp2_response_3c_dev": (_I32, [_P, _P, _P, _I64, _I64, _I64, _I64, _I64, _I64, _D, _P, _P, _P]),
    "fc_rimp2_energy_grad_dens": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _DP, _DP, _P, _P, _P, _P, _P, _P]),
    "fc_rimp2_energy_grad_dens_dev": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _DP, _DP, _P, _P, _P, _P, _P, _P,
                                             _P]),
    "fc_rimp2_energy_shard_dev": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _D, _I32, _I32, _I32, _DP, _DP, _P,
                                         _P]),
    "fc_rimp2_energy_grad_shard_dev": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _I32, _I32, _DP, _DP, _P, _P, _P,
                                              _P, _P]),
    "fc_rimp2_shard_pairs": (_I32, [_I64, _I64, _I32, _I32, _I32, _I32, _P, _I64, _c.POINTER(_I64)]),
    "fc_dfjk_create": (_I32, [_P, _I64, _I64, _I32, _I32, _c.POINTER(_P)]),
    "fc_dfjk_create_dev": (_I32, [_P, _I64, _I64, _I32, _I32, _P, _c.POINTER(_P)]),
    "fc_dfj_set_metric_chol": (_I32, [_P, _P]),
    "fc_dfj_build": (_I32, [_P, _P, _P, _P]),
    "fc_dfj_build_dev": (_I32, [_P, _P, _P, _P, _P]),
    "fc_dfk_build_occ": (_I32, [_P, _P, _I64, _P, _P]),
    "fc_dfk_build_occ_dev": (_I32, [_P, _P, _I64, _P, _P, _P]),
    "fc_dfjk_build_occ": (_I32, [_P, _P, _I64, _P, _P, _P]),
    "fc_dfjk_build_occ_dev": (_I32, [_P, _P, _I64, _P, _P, _P, _P]),
    "fc_dfjk_set_precision": (_I32, [_P, _I32]),
    "fc_dfjk_destroy": (_I32, [_P]),
    "fc_rimp2_energy_noalloc": (_I32, [_P, _I64, _I64, _I64, _P, _P, _I32, _D, _DP, _DP, _P]),
    "fc_ump2_energy": (_I32, [_P, _I64, _I64, _P, _P, _P, _I64, _I64, _P, _P, _I64, _I32, _DP, _DP, _DP, _P]),
    "fc_ump2_energy_dev": (_I32, [_P, _I64, _I64, _P, _P, _P, _I64, _I64, _P, _P, _I64, _I32, _DP, _DP, _DP, _P,
                                  _P]),
    "fc_rimp2_imat": (_I32, [_P, _P, _I64, _I64, _I64, _I64, _I64, _I32, _P, _P]),
    "fc_rimp2_imat_dev": (_I32, [_P, _P, _I64, _I64, _I64, _I64, _I64, _I32, _P, _P, _P]),
    "fc_mo_dress": (_I32, [_P, _I64, _I64, _P, _P, _I64, _P, _I64, _I32, _P, _P]),
    "fc_mo_dress_dev": (_I32, [_P, _I64, _I64, _P, _P, _I64, _P, _I64, _I32, _P, _P, _P]),
    "fc_rimp2_batched_create": (_I32, [_P, _I64, _I32, _c.POINTER(_P)]),
    "fc_rimp2_batched_replay": (_I32, [_P, _P]),
    "fc_rimp2_batched_energies": (_I32, [_P, _DP, _DP]),
    "fc_rimp2_batched_info": (_I32, [_P, _P]),
    "fc_rimp2_batched_plan": (_c.c_size_t, [_P, _c.c_char_p, _c.c_size_t]),
    "fc_rimp2_batched_destroy": (_I32, [_P]),
    "fc_rimp2_batched": (_I32, [_P, _I64, _I32, _DP, _DP]),
}


class FcMolDesc(ctypes.Structure):
    """``fc_mol_desc``: one molecule of a batch (device pointers)."""
    _fields_ = [
        ("b_ov", ctypes.c_void_p), ("eps_occ", ctypes.c_void_p), ("eps_vir", ctypes.c_void_p),
        ("naux", ctypes.c_int64), ("nocc", ctypes.c_int64), ("nvir", ctypes.c_int64),
        ("gamma", ctypes.c_void_p), ("de_deps_occ", ctypes.c_void_p), ("de_deps_vir", ctypes.c_void_p),
    ]


class FcBatchInfo(ctypes.Structure):
    """``fc_batch_info``."""
    _fields_ = [
        ("nmol", ctypes.c_int64), ("items", ctypes.c_int64), ("gemm_tiles", ctypes.c_int64),
        ("launches", ctypes.c_int32), ("groups", ctypes.c_int32), ("pair_launches", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("grad", ctypes.c_int32),
        ("tile_m", ctypes.c_int32), ("tile_n", ctypes.c_int32), ("k_panel", ctypes.c_int32),
        ("flops", ctypes.c_double), ("last_ms", ctypes.c_double), ("bytes", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FcStats(ctypes.Structure):
    _fields_ = [
        ("kernel_ms", ctypes.c_double), ("flops", ctypes.c_double),
        ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("precision", ctypes.c_int32), ("launches", ctypes.c_int32),
        ("tile_m", ctypes.c_int32), ("tile_n", ctypes.c_int32),
        ("k_panel", ctypes.c_int32), ("main_launches", ctypes.c_int32),
        ("main_ms", ctypes.c_double), ("main_flops", ctypes.c_double),
        ("main_bytes", ctypes.c_double),
        ("aux_launches", ctypes.c_int32), ("reserved_", ctypes.c_int32),
        ("aux_ms", ctypes.c_double), ("aux_flops", ctypes.c_double), ("aux_bytes", ctypes.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FcError(RuntimeError):
    """A non-zero fc_status: the device path did not run (the reference's GpuError)."""

    def __init__(self, status, message):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {message}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libferric_cuda.so not found at {LIB_PATH}; build it with `python -m ferric_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()
_init_lock = threading.Lock()
_initialised = None


def last_error():
    n = lib.fc_last_error(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib.fc_last_error(buf, n + 1)
    return buf.value.decode(errors="replace")


def check(status):
    if status != FC_OK:
        raise FcError(status, last_error())


def init(device=0, pool_bytes=0):
    """Bind the library to ``device`` (idempotent)."""
    global _initialised
    with _init_lock:
        if _initialised == (device, pool_bytes):
            return
        check(lib.fc_init(device, pool_bytes))
        _initialised = (device, pool_bytes)


def ensure_init():
    if _initialised is None:
        dev = 0
        try:
            import torch
            if torch.cuda.is_available():
                dev = torch.cuda.current_device()
        except Exception:  # noqa: BLE001 - torch is optional for the host API
            pass
        init(dev, int(os.environ.get("FERRIC_GPU_MEM_BYTES", "0")))


def ptr(a):
    """Address of a contiguous numpy array or torch tensor."""
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)

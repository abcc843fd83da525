"""The C ABI without a GPU: the library loads, exports every symbol that
include/ferric_cuda.h declares, and refuses bad calls before touching a device."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ferric_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\*?\s+\*?(fc_[a-z_0-9]+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("fc_init", "fc_rimp2_energy", "fc_rimp2_energy_grad", "fc_dfjk_create",
                 "fc_dfj_build", "fc_dfk_build_occ", "fc_dfjk_destroy", "fc_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from ferric_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding has a signature for each
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_string():
    from ferric_b200 import _lib
    assert b"sm_100a" in _lib.lib.fc_version()


def test_invalid_arguments_refused_before_device():
    from ferric_b200 import _lib
    L = _lib.lib
    eo, es = ctypes.c_double(), ctypes.c_double()
    # null outputs
    assert L.fc_rimp2_energy(None, 1, 1, 1, None, None, 0, 0.0, 0, None, None, None) == 10
    # negative dimension
    assert L.fc_rimp2_energy(None, -1, 1, 1, None, None, 0, 0.0, 0, ctypes.byref(eo), ctypes.byref(es), None) == 5
    # kappa with mixed precision
    b = np.zeros((2, 2))
    e = np.zeros(2)
    st = L.fc_rimp2_energy(_lib.ptr(b), 2, 1, 2, _lib.ptr(e), _lib.ptr(e), 1, 1.0, 1,
                           ctypes.byref(eo), ctypes.byref(es), None)
    assert st == 10 and "kappa" in _lib.last_error()
    # unknown precision
    st = L.fc_rimp2_energy(_lib.ptr(b), 2, 1, 2, _lib.ptr(e), _lib.ptr(e), 0, 0.0, 9,
                           ctypes.byref(eo), ctypes.byref(es), None)
    assert st == 10
    # overflowing sizes
    st = L.fc_rimp2_energy(_lib.ptr(b), 1 << 40, 1 << 20, 1 << 20, _lib.ptr(e), _lib.ptr(e), 0, 0.0, 0,
                           ctypes.byref(eo), ctypes.byref(es), None)
    assert st == 5
    # handle creation with bad layout
    h = ctypes.c_void_p()
    assert L.fc_dfjk_create(_lib.ptr(b), 2, 2, 7, 0, ctypes.byref(h)) == 10
    assert L.fc_dfjk_destroy(None) == 0


def test_no_cpu_fallback_without_device():
    """Without a usable device the product path errors; it never computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        return
    from ferric_b200 import _lib
    b = np.ones((4, 6))
    e = np.array([-1.0, -2.0, 0.5, 1.0, 2.0])
    eo, es = ctypes.c_double(), ctypes.c_double()
    st = _lib.lib.fc_rimp2_energy(_lib.ptr(b), 4, 2, 3, _lib.ptr(e), _lib.ptr(e[2:]), 0, 0.0, 0,
                                  ctypes.byref(eo), ctypes.byref(es), None)
    assert st != 0

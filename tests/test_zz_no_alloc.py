"""fc_rimp2_energy_noalloc: the FP64 RI-MP2 energy for callers that cannot call
cudaMalloc (their device memory belongs to another allocator, or an inner loop
must not take cudaMalloc's device synchronisation).  Its scratch is a fixed
array inside the library.  The test calls it through the C ABI twice in a row
and checks both results against the workspace entry point fc_rimp2_energy_dev
and against the FP64 oracle, and that the library's workspace pool and the
device's free memory do not change across the calls.  Collected last so a
failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu


def _noalloc(L, b, eo, ev, stream, kappa=None):
    e_os, e_ss = ctypes.c_double(), ctypes.c_double()
    hk, kv = (0, 0.0) if kappa is None else (1, float(kappa))
    st = L.lib.fc_rimp2_energy_noalloc(L.ptr(b), b.shape[0], eo.shape[0], ev.shape[0], L.ptr(eo), L.ptr(ev),
                                       hk, kv, ctypes.byref(e_os), ctypes.byref(e_ss), stream)
    return st, e_os.value, e_ss.value


def _reference(L, b, eo, ev, stream, kappa=None):
    e_os, e_ss = ctypes.c_double(), ctypes.c_double()
    hk, kv = (0, 0.0) if kappa is None else (1, float(kappa))
    L.check(L.lib.fc_rimp2_energy_dev(L.ptr(b), b.shape[0], eo.shape[0], ev.shape[0], L.ptr(eo), L.ptr(ev),
                                      hk, kv, 0, ctypes.byref(e_os), ctypes.byref(e_ss), stream, None))
    return e_os.value, e_ss.value


@pytest.mark.parametrize("naux,nocc,nvir,kappa", [(200, 7, 65, None), (480, 12, 110, None), (130, 6, 33, 1.1)])
def test_noalloc_matches_workspace_entry_point(fc, naux, nocc, nvir, kappa):
    import torch
    L = fc
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    tb, to, tv = (torch.from_numpy(x).cuda() for x in (b, eo, ev))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = _reference(L, tb, to, tv, stream, kappa)
    o_os, o_ss, _ = orc.spin_components(b, np.concatenate([eo, ev]), nocc, nvir, kappa=kappa)
    torch.cuda.synchronize()
    pool0 = L.lib.fc_pool_used()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        st, e_os, e_ss = _noalloc(L, tb, to, tv, stream, kappa)
        assert st == 0, L.last_error()
        # same kernel and reduction order as the workspace path: FP64 tolerance of the plain set
        assert abs(e_os - ref[0]) <= 1e-12 * abs(ref[0]) + 1e-15
        assert abs(e_ss - ref[1]) <= 1e-12 * abs(ref[0]) + 1e-15
        # and the FP64 oracle to the plain set's parity bar
        assert abs(e_os - o_os) <= 1e-10 + 1e-13 * abs(o_os)
        assert abs(e_ss - o_ss) <= 1e-10 + 1e-13 * abs(o_os)
    torch.cuda.synchronize()
    assert L.lib.fc_pool_used() == pool0
    assert free0 - torch.cuda.mem_get_info()[0] < (1 << 20)


def test_noalloc_refuses_beyond_its_scratch(fc):
    import torch
    L = fc
    # nocc 120, nvir 1100: 7260 pairs x 18^2 tiles, far past the fixed scratch
    tb = torch.zeros((2, 120 * 1100), dtype=torch.float64, device="cuda")
    to = torch.full((120,), -1.0, dtype=torch.float64, device="cuda")
    tv = torch.ones(1100, dtype=torch.float64, device="cuda")
    st, _, _ = _noalloc(L, tb, to, tv, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 5
    assert "scratch" in L.last_error()

"""RI-MP2 parity on the B200: the FP64 plain kernels against the FP64 oracle,
through the C ABI (host API) and the device API (torch CUDA tensors)."""
import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

# FP64 plain set: within 1e-10 Eh of the FP64 oracle (absolute), and a
# relative floor for the large-magnitude synthetic cases.
E_TOL = 1e-10

SHAPES = [
    (96, 5, 23),      # nvir < one tile, odd
    (84, 5, 19),      # water-sized
    (130, 3, 64),     # exact tile edge, naux not a multiple of 16
    (200, 7, 65),     # one past a tile edge
    (480, 12, 110),   # scaled-down synthetic RI-MP2 (1/10 of naux 4800, nocc 120, nvir 1100)
    (17, 1, 1),       # degenerate: one occupied, one virtual
]


def _tol(e):
    return E_TOL + 1e-13 * abs(e)


@pytest.mark.parametrize("naux,nocc,nvir", SHAPES)
def test_energy_f64_matches_oracle(fc, naux, nocc, nvir):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    eps = np.concatenate([eo, ev])
    ref = orc.spin_components(b, eps, nocc, nvir)
    st = {}
    sc = rimp2.spin_components_on_device(b, eps, nocc, nvir, precision="f64", stats=st)
    assert abs(sc.e_os - ref[0]) < _tol(ref[0])
    assert abs(sc.e_ss - ref[1]) < _tol(ref[1])
    assert abs(sc.e_total - ref[2]) < _tol(ref[2])
    assert st["launches"] >= 2 and st["precision"] == 0


def test_energy_is_deterministic(fc):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(200, 7, 65)
    r = [rimp2.rimp2_energy(b, eo, ev) for _ in range(3)]
    assert r[0] == r[1] == r[2]


@pytest.mark.parametrize("kappa", [0.5, 1.1, 2.0])
def test_kappa_energy_matches_oracle(fc, kappa):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(130, 6, 33)
    eps = np.concatenate([eo, ev])
    ref = orc.spin_components(b, eps, 6, 33, kappa=kappa)
    sc = rimp2.spin_components_on_device(b, eps, 6, 33, kappa=kappa)
    assert abs(sc.e_os - ref[0]) < _tol(ref[0])
    assert abs(sc.e_ss - ref[1]) < _tol(ref[1])


def test_frozen_core_indexing(fc):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(96, 4, 23)
    eps = np.concatenate([[-60.0, -30.0], eo, ev])   # two frozen cores before the active block
    ref = orc.spin_components(b, eps, 4, 23, first_occ=2, nocc_total=6)
    sc = rimp2.spin_components_on_device(b, eps, 4, 23, first_occ=2, nocc_total=6)
    assert abs(sc.e_total - ref[2]) < _tol(ref[2])


@pytest.mark.parametrize("naux,nocc,nvir", [(96, 5, 23), (200, 7, 65), (130, 3, 64)])
def test_gradient_f64_matches_oracle(fc, naux, nocc, nvir):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    e_os, e_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
    sc, g, go, gv = rimp2.rimp2_energy_grad(b, eo, ev, precision="f64")
    assert abs(sc.e_os - e_os) < _tol(e_os)
    assert abs(sc.e_ss - e_ss) < _tol(e_ss)
    scale = np.abs(gamma).max()
    assert np.abs(g - gamma).max() <= 1e-12 * scale
    assert np.abs(go - d_o).max() <= 1e-12 * np.abs(d_o).max()
    assert np.abs(gv - d_v).max() <= 1e-12 * np.abs(d_v).max()


def test_gradient_chunked_matches_single_chunk(fc, monkeypatch):
    """Small amplitude budget -> occupied chunks of 2 (9 = 2+2+2+2+1), 15
    chunk pairs; Gamma is accumulated over the chunk pairs in FP64, so it
    matches one chunk to rounding."""
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(160, 9, 40)
    one = rimp2.rimp2_energy_grad(b, eo, ev)
    monkeypatch.setenv("FERRIC_CUDA_CHUNK_BYTES", str(2 * 3 * 40 * 3 * 40 * 8 - 1))
    many = rimp2.rimp2_energy_grad(b, eo, ev)
    assert abs(one[0].e_total - many[0].e_total) < 1e-14 * abs(one[0].e_total) + 1e-16
    for k in (1, 2, 3):
        assert np.allclose(one[k], many[k], rtol=0, atol=1e-13 * np.abs(one[k]).max())
    e_os, e_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
    assert np.abs(many[1] - gamma).max() <= 1e-12 * np.abs(gamma).max()


def test_device_api_matches_host_api(fc):
    import torch
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(200, 7, 65)
    host = rimp2.rimp2_energy(b, eo, ev)
    dev = rimp2.rimp2_energy(torch.from_numpy(b).cuda(), torch.from_numpy(eo).cuda(),
                             torch.from_numpy(ev).cuda())
    assert host == dev
    sc, g, go, gv = rimp2.rimp2_energy_grad(torch.from_numpy(b).cuda(), torch.from_numpy(eo).cuda(),
                                           torch.from_numpy(ev).cuda())
    sc2, g2, go2, gv2 = rimp2.rimp2_energy_grad(b, eo, ev)
    assert np.array_equal(g.cpu().numpy(), g2)


def test_dispatcher_returns_components(fc):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(96, 5, 23)
    eps = np.concatenate([eo, ev])
    sc = rimp2.try_spin_components_on_device(b, eps, 5, 23, mixed_ok=False)
    ref = orc.spin_components(b, eps, 5, 23)
    assert sc is not None and abs(sc.e_total - ref[2]) < _tol(ref[2])


def test_zero_sizes(fc):
    from ferric_b200 import rimp2
    b = np.zeros((10, 0))
    e_os, e_ss = rimp2.rimp2_energy(b, np.zeros(0), np.zeros(5))
    assert e_os == 0.0 and e_ss == 0.0


def test_pool_cap_refuses_before_transfer(fc):
    import ferric_b200._lib as L
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(96, 5, 23)
    L.lib.fc_release_workspace()
    L.init(0, 1024)             # 1 KiB pool: the B upload cannot fit
    try:
        with pytest.raises(L.FcError) as ei:
            rimp2.rimp2_energy(b, eo, ev)
        assert ei.value.name == "FC_ERR_POOL_FULL"
        assert rimp2.try_spin_components_on_device(b, np.concatenate([eo, ev]), 5, 23) is None
    finally:
        L.init(0, 0)

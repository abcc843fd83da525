"""Exact integer-slice RI-MP2 kernels (tcgen05 kind::i8) against the FP64
oracle and against an exact NumPy emulation of the split algorithm.

FC_PREC_MIXED splits every pair-operand row into four int8 integers at a
power-of-two scale and sums the ten slice products of level <= 3 exactly in
int32 (the adjoint contraction keeps three slices and six products); the
device energy must equal the emulation (slices in NumPy, integer products
summed exactly, (ia|ia) of the i == j blocks in FP64) to FP64 rounding, and
the FP64 oracle to the slice truncation error.
"""
import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

# Energy bound of the split: four int8 slices carry ~31 bits of each element
# relative to its row maximum.  For small systems, where a few elements
# dominate E, the relative energy error reaches ~5e-10 (largest over the
# shapes below and 120 seeded random systems of 2-4 occupied orbitals,
# emulated exactly on the CPU); large systems sit near 1e-12 (config 3:
# ~5e-8 Eh of 1.9e5 Eh, emulated on sampled pairs).
MIXED_E_REL = 2e-9
# Gamma (max-normalised) and dE/deps bounds: the adjoint contraction's three
# slices (measured max x 5)
MIXED_G_REL = 1e-5
MIXED_D_REL = 1e-6
# absolute floor (Eh) for tiny systems
MIXED_E_ABS = 1e-13
FAST_E_REL = 2e-4     # hi+lo, FP32 accumulation (accumulation-bound)


def chunk_budget(nvir, chunk):
    """FERRIC_CUDA_CHUNK_BYTES for occupied chunks of `chunk` orbitals: the
    gradient driver's memory model per chunk-pair element (two FP32 amplitude
    blocks, three int8 slices) at amplitude pitch nvir rounded up to 16."""
    tp = (nvir + 15) // 16 * 16
    return (chunk + 1) ** 2 * (tp * tp * 11 + 1024 * tp) - 1


def pair_slices(b):
    """The FC_PREC_MIXED split of every column of b (power-of-two scale with
    max|x|/s in (63.5, 127], four int8 slices at weights 1/254^k)."""
    mx = np.abs(b).max(axis=0)
    k = np.frexp(np.where(mx > 0, mx, 1.0))[1]
    s = np.ldexp(1.0, k - 7)
    s = np.where(mx > 127.0 * s, 2.0 * s, s)
    s = np.where(mx > 0, s, 1.0)
    r = b / s[None, :]
    cs = []
    for _ in range(4):
        c = np.rint(r)
        assert np.abs(c).max() <= 127
        cs.append(c)
        r = (r - c) * 254.0
    return s, cs


def emulate_fixed_slices(b):
    """G = B^T B as the pair kernel forms it: the exact level sums of the ten
    products of level <= 3, combined as s_r s_r' (((L0 254 + L1) 254 + L2) 254
    + L3) / 254^3."""
    s, c = pair_slices(b)
    lev = [sum(c[k].T @ c[l - k] for k in range(l + 1)) for l in range(4)]
    v = ((lev[0] * 254.0 + lev[1]) * 254.0 + lev[2]) * 254.0 + lev[3]
    return (np.outer(s, s) * (1.0 / 254.0 ** 3)) * v


def energy_from_g(g, eo, ev, b=None):
    """The device's energy from the emulated G: per pair i <= j the X element
    (ia|jb) and the Y element (ib|ja) in FP64; i == j uses X only, with the
    exact (ia|ia) = sum_Q B_Q,ia^2 on its diagonal (when b is given)."""
    nocc, nvir = len(eo), len(ev)
    e_os = e_ss = 0.0
    for i in range(nocc):
        for j in range(i, nocc):
            x = g[i * nvir:(i + 1) * nvir, j * nvir:(j + 1) * nvir].copy()
            d = eo[i] + eo[j] - ev[:, None] - ev[None, :]
            if i == j:
                if b is not None:
                    x[np.diag_indices(nvir)] = (b[:, i * nvir:(i + 1) * nvir] ** 2).sum(axis=0)
                e_os += np.sum(x * x / d)
            else:
                y = g[j * nvir:(j + 1) * nvir, i * nvir:(i + 1) * nvir]   # G_ji[a, b] = (ib|ja)
                e_os += 2.0 * np.sum(x * x / d)
                e_ss += 2.0 * np.sum(x * (x - y) / d)
    return e_os, e_ss


# nvir 190 and 192: the last virtual tile trimmed to 64 columns (its limit);
# 193: 80 columns, the stacked form
SHAPES = [(96, 5, 23), (84, 5, 19), (200, 7, 65), (300, 4, 130), (130, 3, 128), (480, 12, 110),
          (260, 4, 190), (260, 3, 193)]


@pytest.mark.parametrize("xt", ["0", "1"])
@pytest.mark.parametrize("naux,nocc,nvir", SHAPES)
def test_mixed_energy_matches_oracle_and_emulation(fc, monkeypatch, naux, nocc, nvir, xt):
    """xt = 1: diagonal tiles in one phase, Y = X^T read back from the X tile."""
    from ferric_b200 import rimp2
    monkeypatch.setenv("FERRIC_CUDA_XT", xt)
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    ref = orc.spin_components(b, np.concatenate([eo, ev]), nocc, nvir)
    st = {}
    e_os, e_ss = rimp2.rimp2_energy(b, eo, ev, precision="mixed", stats=st)
    assert st["precision"] == 1 and st["launches"] > 0
    assert abs(e_os + e_ss - ref[2]) <= MIXED_E_REL * abs(ref[2]) + MIXED_E_ABS
    em = energy_from_g(emulate_fixed_slices(b), eo, ev, b)
    # exact accumulation: device == emulation to summation rounding
    assert abs(e_os - em[0]) <= 1e-12 * abs(em[0]) + 1e-15
    assert abs(e_ss - em[1]) <= 1e-12 * abs(em[0]) + 1e-15


@pytest.mark.parametrize("xt", ["0", "1"])
@pytest.mark.parametrize("naux,nocc,nvir", [(96, 5, 23), (200, 7, 65), (300, 4, 130), (520, 6, 300),
                                            (260, 4, 192)])
def test_mixed_gradient_matches_oracle(fc, monkeypatch, naux, nocc, nvir, xt):
    from ferric_b200 import rimp2
    monkeypatch.setenv("FERRIC_CUDA_XT", xt)
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    e_os, e_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
    sc, g, go, gv = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert abs(sc.e_total - (e_os + e_ss)) <= MIXED_E_REL * abs(e_os + e_ss) + MIXED_E_ABS
    assert np.abs(g - gamma).max() <= MIXED_G_REL * np.abs(gamma).max()
    assert np.abs(go - d_o).max() <= MIXED_D_REL * np.abs(d_o).max()
    assert np.abs(gv - d_v).max() <= MIXED_D_REL * np.abs(d_v).max()
    # the gradient call's energy is the energy call's energy (the same FP64
    # terms), up to the order of the partial sums
    e2 = rimp2.rimp2_energy(b, eo, ev, precision="mixed")
    assert abs(sum(e2) - sc.e_total) <= 1e-13 * abs(sc.e_total)


def test_mixed_gradient_chunked(fc, monkeypatch):
    """A small chunk budget: several occupied chunks (the last one shorter),
    most chunk pairs off the diagonal (each unordered pair feeds the
    amplitude rows of both its chunks).  The amplitudes are the same; each amplitude block is split at
    its own row scales (the row maximum over the block's columns), so Gamma
    differs from the one-chunk Gamma by the slicing error; dE/deps come from
    the pair kernel in FP64 and differ only in summation order."""
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(160, 9, 40)
    one = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    monkeypatch.setenv("FERRIC_CUDA_CHUNK_BYTES", str(chunk_budget(40, 2)))  # chunks of 2
    many = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert abs(one[0].e_total - many[0].e_total) <= 1e-14 * abs(one[0].e_total)
    assert np.abs(one[1] - many[1]).max() <= 4e-6 * np.abs(one[1]).max()
    assert np.abs(one[2] - many[2]).max() <= 1e-13 * np.abs(one[2]).max()
    assert np.abs(one[3] - many[3]).max() <= 1e-13 * np.abs(one[3]).max()
    e_os, e_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
    assert np.abs(many[1] - gamma).max() <= MIXED_G_REL * np.abs(gamma).max()
    assert np.abs(many[2] - d_o).max() <= MIXED_D_REL * np.abs(d_o).max()
    assert np.abs(many[3] - d_v).max() <= MIXED_D_REL * np.abs(d_v).max()


def test_mixed_gradient_pinned_upload(fc, monkeypatch):
    """A page-locked B_ov goes up chunk by chunk on a copy stream while the
    gradient runs, each chunk's operands made after its arrival event: with
    several chunks the host API's result is the device API's bit for bit,
    and a pageable B_ov (one copy before the compute) gives the same."""
    import torch
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(160, 9, 40)
    monkeypatch.setenv("FERRIC_CUDA_CHUNK_BYTES", str(chunk_budget(40, 2)))  # chunks of 2
    pinned = torch.empty(b.shape, dtype=torch.float64).pin_memory()
    pinned.numpy()[:] = b
    up = rimp2.rimp2_energy_grad(pinned.numpy(), eo, ev, precision="mixed")
    dev = rimp2.rimp2_energy_grad(torch.from_numpy(b).cuda(), torch.from_numpy(eo).cuda(),
                                  torch.from_numpy(ev).cuda(), precision="mixed")
    paged = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    for other in (dev, paged):
        assert (up[0].e_os, up[0].e_ss) == (other[0].e_os, other[0].e_ss)
        for x, y in zip(up[1:], other[1:]):
            y = y.cpu().numpy() if hasattr(y, "cpu") else y
            assert np.array_equal(x, y)


def test_adjoint_k_segments(fc, monkeypatch):
    """The adjoint contraction keeps its int32 level sums exact by running K
    in segments (32768 by default) that each add into Gamma; with 128-column
    segments Gamma matches the one-segment result to FP64 rounding."""
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(200, 9, 60)
    one = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    monkeypatch.setenv("FERRIC_CUDA_KSEG", "128")
    seg = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert one[0].e_total == seg[0].e_total
    assert np.abs(one[1] - seg[1]).max() <= 1e-13 * np.abs(one[1]).max()


def test_mixed_refuses_naux_beyond_exact_int32(fc):
    """The pair kernel's level sums are exact while 4 * 127^2 * naux <= 2^31 - 1
    (naux <= 33286): at naux = 33286 a constant B whose four slices all sit at
    +-127 (x / s = 127 - 127/254 + 127/254^2 - 127/254^3, so level 3 sums
    -4 * 127^2 per aux function, 2147479576 in magnitude) still equals the
    exact emulation -- an int32 wrap would be off by 2^32 -- and FP64 to the
    dropped level-4 products (3 127^2 / 254^4 of each term here, where the
    two occupied rows are equal); naux = 33287 is refused (FC_ERR_LAYOUT,
    nothing launched), and FP64 takes it."""
    import ferric_b200._lib as L
    from ferric_b200 import rimp2
    c = 127.0 - 127.0 / 254 + 127.0 / 254 ** 2 - 127.0 / 254 ** 3
    _, sl = pair_slices(np.full((4, 1), c))
    assert [int(x[0, 0]) for x in sl] == [127, -127, 127, -127]
    eo, ev = np.array([-1.0, -0.8]), np.array([0.5])
    b = np.full((33286, 2), c)
    e = rimp2.rimp2_energy(b, eo, ev, precision="mixed")
    em = energy_from_g(emulate_fixed_slices(b), eo, ev, b)
    assert abs(e[0] - em[0]) <= 1e-12 * abs(em[0]) and abs(e[1] - em[1]) <= 1e-12 * abs(em[0])
    ref = orc.spin_components(b, np.concatenate([eo, ev]), 2, 1)
    assert abs(sum(e) - ref[2]) <= 2.0 * 3.0 * 127 ** 2 / 254.0 ** 4 / 127 ** 2 * abs(ref[2])
    rng = np.random.default_rng(3)
    b = rng.standard_normal((33287, 2)) * 1e-3
    eo, ev = np.array([-1.0]), np.array([0.5, 0.9])
    with pytest.raises(L.FcError) as ei:
        rimp2.rimp2_energy(b, eo, ev, precision="mixed")
    assert ei.value.name == "FC_ERR_LAYOUT"
    e = rimp2.rimp2_energy(b, eo, ev, precision="f64")
    ref = orc.spin_components(b, np.concatenate([eo, ev]), 1, 2)
    assert abs(sum(e) - ref[2]) <= 1e-12 * abs(ref[2])


def test_mixed_deterministic(fc):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(200, 7, 65)
    r = [rimp2.rimp2_energy(b, eo, ev, precision="mixed") for _ in range(3)]
    assert r[0] == r[1] == r[2]
    g1 = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    g2 = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert np.array_equal(g1[1], g2[1])


@pytest.mark.parametrize("naux,nocc,nvir", [(96, 5, 23), (200, 7, 65), (480, 12, 110)])
def test_mixed_fast_energy(fc, naux, nocc, nvir):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir)
    ref = orc.spin_components(b, np.concatenate([eo, ev]), nocc, nvir)
    e = rimp2.rimp2_energy(b, eo, ev, precision="mixed_fast")
    assert abs(sum(e) - ref[2]) <= FAST_E_REL * abs(ref[2])


def test_mixed_refuses_nonfinite(fc):
    import ferric_b200._lib as L
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(96, 5, 23)
    b[3, 7] = np.inf
    with pytest.raises(L.FcError) as ei:
        rimp2.rimp2_energy(b, eo, ev, precision="mixed")
    assert ei.value.name == "FC_ERR_RANGE"
    # the dispatcher retries in FP64 on the device; FP64 then sees the inf too
    sc = rimp2.try_spin_components_on_device(b, np.concatenate([eo, ev]), 5, 23, mixed_ok=True)
    assert sc is None or not np.isfinite(sc.e_total)


def test_mixed_fast_has_no_adjoint(fc):
    import ferric_b200._lib as L
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(96, 5, 23)
    with pytest.raises(L.FcError) as ei:
        rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed_fast")
    assert ei.value.name == "FC_ERR_KERNEL"


def test_exchange_matches_two_phases(fc, monkeypatch):
    """The diagonal-tile exchange reads Y = X^T back from the FP64 X tile; the
    two-phase schedule computes Y with the operands swapped, whose level sums
    are the same integers (the kept products are symmetric in the two
    operands), so both give the same energy, Gamma and dE/deps_occ bits."""
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(520, 7, 300)
    out = {}
    for xt in ("0", "1"):
        monkeypatch.setenv("FERRIC_CUDA_XT", xt)
        out[xt] = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert out["0"][0].e_os == out["1"][0].e_os and out["0"][0].e_ss == out["1"][0].e_ss
    assert np.array_equal(out["0"][1], out["1"][1]) and np.array_equal(out["0"][2], out["1"][2])
    # dE/deps_vir: a two-phase tile sums its column terms in FP32 over a warp's
    # rows, the exchanged tile adds them to its rows in FP64
    assert np.abs(out["0"][3] - out["1"][3]).max() <= 1e-7 * np.abs(out["0"][3]).max()


EDGE = [
    (17, 1, 1),       # one occupied, one virtual
    (1, 3, 4),        # one aux function
    (65, 2, 129),     # one virtual past a 128-row tile: two tiles, ragged
    (64, 4, 128),     # exact tile and k-step edges
    (700, 33, 169),   # the largest batched alkane (C8H18 in cc-pVDZ / -RI)
]


@pytest.mark.parametrize("naux,nocc,nvir", EDGE)
def test_mixed_edge_shapes(fc, naux, nocc, nvir):
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(naux, nocc, nvir, seed_b=11, seed_eps=12)
    e_os, e_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
    e = rimp2.rimp2_energy(b, eo, ev, precision="mixed")
    assert abs(sum(e) - (e_os + e_ss)) <= MIXED_E_REL * abs(e_os + e_ss) + MIXED_E_ABS
    sc, g, go, gv = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
    assert abs(sc.e_total - (e_os + e_ss)) <= MIXED_E_REL * abs(e_os + e_ss) + MIXED_E_ABS
    assert np.abs(g - gamma).max() <= MIXED_G_REL * np.abs(gamma).max()
    assert np.abs(go - d_o).max() <= MIXED_D_REL * np.abs(d_o).max()
    assert np.abs(gv - d_v).max() <= MIXED_D_REL * np.abs(d_v).max()


def test_mixed_zero_sizes(fc):
    from ferric_b200 import rimp2
    e_os, e_ss = rimp2.rimp2_energy(np.zeros((10, 0)), np.zeros(0), np.zeros(5), precision="mixed")
    assert e_os == 0.0 and e_ss == 0.0


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_gamma_streamed_to_pinned_host(fc, monkeypatch, precision):
    """With a pinned host Gamma the host API copies each occupied chunk's
    columns out while later chunk pairs still run; the result is the same
    bits as the copy-at-the-end path (pageable Gamma)."""
    import ctypes
    import torch
    import ferric_b200._lib as L
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(160, 9, 40)
    monkeypatch.setenv("FERRIC_CUDA_CHUNK_BYTES", str(chunk_budget(40, 2)))
    ref = rimp2.rimp2_energy_grad(b, eo, ev, precision=precision)
    g = torch.empty(b.shape, dtype=torch.float64, pin_memory=True)
    g.fill_(np.nan)
    do, dv = np.empty(9), np.empty(40)
    e1, e2 = ctypes.c_double(), ctypes.c_double()
    L.check(L.lib.fc_rimp2_energy_grad(L.ptr(b), 160, 9, 40, L.ptr(eo), L.ptr(ev), L.PRECISIONS[precision],
                                       ctypes.byref(e1), ctypes.byref(e2), ctypes.c_void_p(g.data_ptr()),
                                       L.ptr(do), L.ptr(dv), None))
    assert np.array_equal(g.numpy(), ref[1])
    assert np.array_equal(do, ref[2]) and np.array_equal(dv, ref[3])


def test_epilogue_reciprocal_within_one_ulp(fc):
    """The pair epilogue's 1 / D (an FP32 seed and a third-order
    Newton-Raphson step) against the correctly rounded FP64 quotient (CUDA's
    and NumPy's division), over denominators of both signs from 1e-30 to 1e30
    and a dense sample of the orbital-energy range."""
    from ferric_b200 import _lib
    rng = np.random.default_rng(5)
    mag = np.concatenate([rng.uniform(0.05, 200.0, 200000), np.logspace(-30, 30, 6001),
                          1.0 + np.arange(-50, 51) * 2.0 ** -52, [1.0, 2.0, 0.5, 3.0, 1.0 / 3.0]])
    d = np.ascontiguousarray(np.concatenate([-mag, mag]))
    out = np.empty_like(d)
    _lib.check(_lib.lib.fc_check_recip(_lib.ptr(d), len(d), _lib.ptr(out)))
    ref = 1.0 / d
    assert np.all(np.abs(out - ref) <= np.spacing(np.abs(ref)))

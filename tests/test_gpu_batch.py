"""Batched RI-MP2 (one CUDA graph over many molecules of uneven size)
against the FP64 oracle per molecule, against the single-molecule device
calls, and on the reference's golden molecules.

Shapes: linear alkanes C_nH_2n+2 in cc-pVDZ / cc-pVDZ-RI have naux 84n+28,
nocc 4n+1, nvir 20n+9; synthetic B_ov of those shapes stand in for the SCF
tensors, plus the real CH4 and water B_ov of the golden fixtures.
"""
import os

import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
# Energy bound of the split (the pair kernel's four int8 slices, ~31 bits of
# each element relative to its row maximum): for small systems, where a few
# elements dominate E, E's relative error reaches ~5e-10 (emulated exactly);
# large systems sit near 1e-12.
MIXED_E_REL = 2e-9
MIXED_G_REL = 1e-5
MIXED_D_REL = 1e-6
MIXED_E_ABS = 1e-12  # Eh, tiny systems


def alkane_shape(n):
    return 84 * n + 28, 4 * n + 1, 20 * n + 9


def _mols(ns, seed0=100):
    out = []
    for k, n in enumerate(ns):
        naux, nocc, nvir = alkane_shape(n)
        out.append(synthetic.rimp2_inputs(naux, nocc, nvir, seed_b=seed0 + k, seed_eps=seed0 + 50 + k))
    return out


def _to_dev(mols):
    import torch
    return [tuple(torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in m) for m in mols]


def test_batch_energy_matches_oracle_and_single(fc):
    from ferric_b200 import rimp2
    from ferric_b200.batch import Rimp2Batch
    ns = [3, 1, 4, 2, 1, 5, 3]
    mols = _mols(ns)
    bt = Rimp2Batch(_to_dev(mols), grad=False)
    bt.run()
    e_os, e_ss = bt.energies()
    info = bt.info()
    assert info["nmol"] == len(ns) and info["pair_launches"] == 1 and info["grad"] == 0
    for m, (b, eo, ev) in enumerate(mols):
        ref = orc.spin_components(b, np.concatenate([eo, ev]), len(eo), len(ev))
        assert abs(e_os[m] + e_ss[m] - ref[2]) <= MIXED_E_REL * abs(ref[2])
        single = rimp2.rimp2_energy(b, eo, ev, precision="mixed")
        # same tiles and slices as the single-molecule call; only the order
        # of the per-tile partial sums differs
        assert abs(e_os[m] - single[0]) <= 1e-13 * abs(single[0])
        assert abs(e_ss[m] - single[1]) <= 1e-13 * abs(single[0])
    bt.close()


def test_batch_gradient_matches_oracle_and_single(fc):
    from ferric_b200 import rimp2
    from ferric_b200.batch import Rimp2Batch
    ns = [2, 1, 4, 3, 1]
    mols = _mols(ns, seed0=200)
    bt = Rimp2Batch(_to_dev(mols), grad=True)
    bt.run()
    e_os, e_ss = bt.energies()
    info = bt.info()
    assert info["grad"] == 1 and info["groups"] >= 1 and info["gemm_tiles"] > 0
    for m, (b, eo, ev) in enumerate(mols):
        r_os, r_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
        g = bt.gamma[m].cpu().numpy()
        go = bt.de_docc[m].cpu().numpy()
        gv = bt.de_dvir[m].cpu().numpy()
        assert abs(e_os[m] + e_ss[m] - (r_os + r_ss)) <= MIXED_E_REL * abs(r_os + r_ss)
        assert np.abs(g - gamma).max() <= MIXED_G_REL * np.abs(gamma).max()
        assert np.abs(go - d_o).max() <= MIXED_D_REL * np.abs(d_o).max()
        assert np.abs(gv - d_v).max() <= MIXED_D_REL * np.abs(d_v).max()
        sc, g1, go1, gv1 = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
        # the same integer slices and exact level sums: only the amplitude
        # pitch and the summation order of partials differ
        assert np.abs(g - g1).max() <= 1e-12 * np.abs(g1).max()
        assert np.abs(go - go1).max() <= 1e-12 * np.abs(go1).max()
        assert np.abs(gv - gv1).max() <= 1e-12 * np.abs(gv1).max()
        assert abs(e_os[m] + e_ss[m] - sc.e_total) <= 1e-12 * abs(sc.e_total)
    bt.close()


def test_batch_groups_and_replay(fc, monkeypatch):
    """Small amplitude budget: one group per molecule; results equal the
    one-group batch.  Replays are deterministic, and follow inputs refilled in
    place (B scaled by 2 -> E scaled by exactly 16: the split scales are
    powers of two)."""
    from ferric_b200.batch import Rimp2Batch
    mols = _mols([2, 3, 1], seed0=300)
    dev = _to_dev(mols)
    one = Rimp2Batch(dev, grad=True)
    one.run()
    e1 = one.energies()
    g1 = [g.cpu().numpy() for g in one.gamma]
    monkeypatch.setenv("FERRIC_CUDA_BATCH_GROUP_BYTES", "1")
    many = Rimp2Batch(dev, grad=True)
    assert many.info()["groups"] == 3
    many.run()
    e2 = many.energies()
    for m in range(3):
        assert abs(e1[0][m] - e2[0][m]) <= 1e-14 * abs(e1[0][m])
        assert np.array_equal(g1[m], many.gamma[m].cpu().numpy())
    many.run()
    assert np.array_equal(many.energies()[0], e2[0])
    for b, _, _ in dev:
        b.mul_(2.0)
    many.run()
    e3 = many.energies()
    assert np.allclose(e3[0], 16.0 * e2[0], rtol=1e-13, atol=0)
    assert np.allclose(e3[1], 16.0 * e2[1], rtol=1e-13, atol=0)
    one.close()
    many.close()


def test_batch_golden_molecules(fc):
    """CH4 and water (cc-pVDZ / -RI, the reference's validation molecules)
    batched with synthetic alkanes: each within the mixed bound of its
    golden DF-MP2 energy."""
    from ferric_b200.batch import Rimp2Batch
    fx = [np.load(os.path.join(HERE, "golden", f + ".npz")) for f in ("ch4_ccpvdz", "h2o_ccpvdz")]
    mols = []
    for d in fx:
        nocc, nvir = int(d["nocc"]), int(d["nvir"])
        eps = d["eps"]
        mols.append((np.ascontiguousarray(d["b_ov"]), eps[:nocc].copy(), eps[nocc:nocc + nvir].copy()))
    mols += _mols([2, 1])
    bt = Rimp2Batch(_to_dev(mols), grad=True)
    bt.run()
    e_os, e_ss = bt.energies()
    for m, d in enumerate(fx):
        assert abs(e_os[m] - float(d["golden_e_os"])) < 1e-6
        assert abs(e_ss[m] - float(d["golden_e_ss"])) < 1e-6
        assert abs(e_os[m] - float(d["oracle_e_os"])) <= MIXED_E_REL * abs(float(d["oracle_e_os"]))
    bt.close()


def test_batch_refusals(fc):
    import torch
    import ferric_b200._lib as L
    from ferric_b200.batch import Rimp2Batch
    dev = _to_dev(_mols([1, 2]))
    with pytest.raises(L.FcError) as ei:
        Rimp2Batch(dev, precision="f64")
    assert ei.value.name == "FC_ERR_KERNEL"
    bad = [list(m) for m in dev]
    bad[1][0] = bad[1][0].clone()
    bad[1][0][0, 0] = float("inf")
    bt = Rimp2Batch([tuple(m) for m in bad])
    bt.run()
    with pytest.raises(L.FcError) as ei:
        bt.energies()
    assert ei.value.name == "FC_ERR_RANGE"
    bt.close()
    with pytest.raises(ValueError):
        Rimp2Batch([(dev[0][0], dev[1][1], dev[0][2])])
    torch.cuda.synchronize()


def test_batch_autotuner_plan(fc, monkeypatch, tmp_path):
    """FERRIC_CUDA_AUTOTUNE=1: every size bucket's exchange choice is measured
    (both choices timed on a trial sub-batch), reported by plan(), written to
    the cache file, and the results stay within the mixed bars whichever
    choice won."""
    import json
    from ferric_b200.batch import Rimp2Batch
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("FERRIC_CUDA_AUTOTUNE", "1")
    monkeypatch.setenv("FERRIC_CUDA_AUTOTUNE_CACHE", str(cache))
    mols = _mols([1, 6, 1, 6], seed0=400)
    bt = Rimp2Batch(_to_dev(mols), grad=True)
    plan = bt.plan()
    assert sum(p["molecules"] for p in plan) == 4 and len(plan) == 2
    for p in plan:
        assert p["source"] == "tuned" and p["exchange"] in (0, 1)
        assert p["ms_two_phase"] > 0 and p["ms_exchange"] > 0
        assert p["exchange"] == int(p["ms_exchange"] < p["ms_two_phase"])
    bt.run()
    e_os, e_ss = bt.energies()
    for m, (b, eo, ev) in enumerate(mols):
        r_os, r_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
        assert abs(e_os[m] + e_ss[m] - (r_os + r_ss)) <= MIXED_E_REL * abs(r_os + r_ss)
        assert np.abs(bt.gamma[m].cpu().numpy() - gamma).max() <= MIXED_G_REL * np.abs(gamma).max()
        assert np.abs(bt.de_dvir[m].cpu().numpy() - d_v).max() <= MIXED_D_REL * np.abs(d_v).max()
    bt.close()
    if cache.exists():  # written unless an earlier batch of this process tuned these buckets
        data = json.loads(cache.read_text())
        assert all(k.startswith(("grad_", "energy_")) for k in data)


@pytest.mark.parametrize("grad", [False, True])
def test_batch_exchange_forced(fc, monkeypatch, grad):
    """Both schedules of the diagonal tiles give the same energies: Y = X^T
    read back from the FP64 X tile equals the swapped-operand phase's Y."""
    from ferric_b200.batch import Rimp2Batch
    mols = _to_dev(_mols([2, 5, 3], seed0=500))
    res = {}
    for xt in ("0", "1"):
        monkeypatch.setenv("FERRIC_CUDA_XT", xt)
        bt = Rimp2Batch(mols, grad=grad)
        assert all(p["source"] == "forced" and p["exchange"] == int(xt) for p in bt.plan())
        bt.run()
        res[xt] = bt.energies()
        bt.close()
    assert np.array_equal(res["0"][0], res["1"][0])
    assert np.array_equal(res["0"][1], res["1"][1])


def test_batch_single_and_degenerate_molecules(fc):
    """A batch of one, and molecules with one occupied / one virtual orbital."""
    from ferric_b200.batch import Rimp2Batch
    mols = [synthetic.rimp2_inputs(17, 1, 1, seed_b=61, seed_eps=62),
            synthetic.rimp2_inputs(40, 1, 30, seed_b=63, seed_eps=64),
            synthetic.rimp2_inputs(90, 6, 2, seed_b=65, seed_eps=66)]
    for group in (mols[:1], mols):
        bt = Rimp2Batch(_to_dev(group), grad=True)
        bt.run()
        e_os, e_ss = bt.energies()
        for m, (b, eo, ev) in enumerate(group):
            r_os, r_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
            assert abs(e_os[m] + e_ss[m] - (r_os + r_ss)) <= MIXED_E_REL * abs(r_os + r_ss) + MIXED_E_ABS
            assert np.abs(bt.gamma[m].cpu().numpy() - gamma).max() <= MIXED_G_REL * np.abs(gamma).max()
            assert np.abs(bt.de_docc[m].cpu().numpy() - d_o).max() <= MIXED_D_REL * np.abs(d_o).max()
        bt.close()


def test_batch_on_oracle_alkane_tensors(fc):
    """Real SCF tensors: the oracle's RHF B_ov and orbital energies of
    all-trans CH4, C2H6 and C3H8 in cc-pVDZ / cc-pVDZ-RI (committed fixture,
    tests/golden/make_alkanes.py), several copies each in one batch: every
    molecule's mixed energy within the bar of the oracle's FP64 RI-MP2
    energy, and the FP64 device path within 1e-10 Eh of it."""
    import torch
    from ferric_b200 import rimp2
    from ferric_b200.batch import Rimp2Batch
    d = dict(np.load(os.path.join(HERE, "golden", "alkanes_c1_c3.npz")))
    ns = [3, 1, 2, 2, 3, 1]
    mols = [(d[f"c{n}_b_ov"], d[f"c{n}_eps_occ"], d[f"c{n}_eps_vir"]) for n in ns]
    bt = Rimp2Batch(_to_dev(mols), grad=True)
    bt.run()
    e_os, e_ss = bt.energies()
    for m, n in enumerate(ns):
        ref = float(d[f"c{n}_e_os"] + d[f"c{n}_e_ss"])
        assert abs(e_os[m] + e_ss[m] - ref) <= MIXED_E_REL * abs(ref) + MIXED_E_ABS
        b, eo, ev = mols[m]
        sc, g, _, _ = rimp2.rimp2_energy_grad(b, eo, ev, precision="f64")
        assert abs(sc.e_total - ref) <= 1e-10
        assert np.abs(bt.gamma[m].cpu().numpy() - g).max() <= MIXED_G_REL * np.abs(g).max()
    bt.close()

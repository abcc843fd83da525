"""Sharded RI-MP2 and DF-JK on one B200: the shards' partials, computed one
after another on the same GPU, add up to the unsharded call; the composition
over a torch.distributed NCCL group of one rank is the identity; DF-JK aux
bands add up to the full J and K."""
import datetime
import os

import numpy as np
import pytest
import torch

from oracle import dfjk as orc_jk
from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu

MIXED_G_REL = 1e-5


def _dev(b, eo, ev):
    return tuple(torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (b, eo, ev))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("nshards", [2, 3])
def test_energy_shards_sum(fc, precision, nshards):
    from ferric_b200 import rimp2, sharded
    b, eo, ev = synthetic.rimp2_inputs(150, 11, 45)
    db, deo, dev = _dev(b, eo, ev)
    full = rimp2.rimp2_energy(db, deo, dev, precision=precision)
    parts = [sharded.rimp2_energy_shard(db, deo, dev, s, nshards, precision) for s in range(nshards)]
    assert all(p[0] != 0.0 for p in parts)
    tot = np.sum(parts, axis=0)
    assert abs(tot[0] - full[0]) <= 1e-12 * abs(full[0])
    assert abs(tot[1] - full[1]) <= 1e-12 * abs(full[1])


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("nshards", [2, 3])
def test_gradient_shards_sum(fc, precision, nshards):
    """Shards cap the occupied chunk size (>= 8 chunk pairs each); FP64 sums
    match the unsharded call to summation order, the mixed Gamma to the
    slicing of its smaller amplitude blocks (each split at its own row
    scales), and both the oracle."""
    from ferric_b200 import rimp2, sharded
    b, eo, ev = synthetic.rimp2_inputs(160, 12, 40)
    db, deo, dev = _dev(b, eo, ev)
    one = rimp2.rimp2_energy_grad(db, deo, dev, precision=precision)
    acc = None
    for s in range(nshards):
        part = sharded.rimp2_energy_grad_shard(db, deo, dev, s, nshards, precision)
        assert part[0] != 0.0
        vals = [part[0], part[1]] + [x.cpu().numpy() for x in part[2:]]
        acc = vals if acc is None else [a + v for a, v in zip(acc, vals)]
    e_tol = 1e-12 if precision == "f64" else 1e-9
    assert abs(acc[0] + acc[1] - one[0].e_total) <= e_tol * abs(one[0].e_total)
    g1 = one[1].cpu().numpy()
    g_tol = 1e-12 if precision == "f64" else 4e-6
    assert np.abs(acc[2] - g1).max() <= g_tol * np.abs(g1).max()
    assert np.abs(acc[3] - one[2].cpu().numpy()).max() <= 1e-12 * np.abs(acc[3]).max()
    assert np.abs(acc[4] - one[3].cpu().numpy()).max() <= 1e-12 * np.abs(acc[4]).max()
    e_os, e_ss, gamma, d_o, d_v = orc.energy_gamma_deps(b, eo, ev)
    assert np.abs(acc[2] - gamma).max() <= (1e-12 if precision == "f64" else MIXED_G_REL) * np.abs(gamma).max()


@pytest.fixture
def nccl_group():
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(29900 + os.getpid() % 50)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    yield dist.group.WORLD
    dist.destroy_process_group()


def test_sharded_over_one_rank_nccl(fc, nccl_group):
    from ferric_b200 import rimp2, sharded
    b, eo, ev = synthetic.rimp2_inputs(96, 7, 33)
    db, deo, dev = _dev(b, eo, ev)
    one = rimp2.rimp2_energy_grad(db, deo, dev, precision="f64")
    for layout in ("band", "full"):
        e_os, e_ss, g, row0, d_o, d_v = sharded.rimp2_energy_grad_sharded(db, deo, dev, precision="f64",
                                                                           gamma_layout=layout)
        assert row0 == 0 and g.shape == db.shape
        assert abs(e_os + e_ss - one[0].e_total) <= 1e-13 * abs(one[0].e_total)
        assert torch.equal(g, one[1])
        assert torch.equal(d_o, one[2]) and torch.equal(d_v, one[3])
    e = sharded.rimp2_energy_sharded(db, deo, dev, precision="mixed")
    e1 = rimp2.rimp2_energy(db, deo, dev, precision="mixed")
    assert abs(sum(e) - sum(e1)) <= 1e-13 * abs(sum(e1))
    jk = sharded.DfJKShard(torch.from_numpy(synthetic.dfjk_inputs(30, 40, 5)[0]).cuda())
    bb, c, d = synthetic.dfjk_inputs(30, 40, 5)
    j = jk.j(torch.from_numpy(d).cuda()).cpu().numpy()
    assert np.abs(j - orc_jk.df_j_square(bb, d)).max() < 1e-10
    jk.close()


def test_dfjk_aux_bands_sum(fc):
    """Aux bands of B (the ranks' shares) give J and K that add up to the
    full builds: what DfJKShard's all-reduce computes across GPUs."""
    from ferric_b200.dfjk import DfJK
    from ferric_b200 import sharded
    bb, c, d = synthetic.dfjk_inputs(50, 90, 7)
    j = np.zeros((50, 50))
    k = np.zeros((50, 50))
    for r in range(3):
        lo, hi = sharded.aux_band(90, r, 3)
        jk = DfJK(np.ascontiguousarray(bb[lo:hi]), precision="f64")
        j += jk.j(d)
        k += jk.k_from_occ(c)
        jk.close()
    assert np.abs(j - orc_jk.df_j_square(bb, d)).max() < 1e-10
    assert np.abs(k - orc_jk.df_k_occ(bb, c)).max() < 1e-10

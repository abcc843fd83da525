"""Occupied-pair sharding of one RI-MP2 system, on the CPU: the partition the
library plans (host only) covers every pair i <= j exactly once and is
balanced, and the composition of per-rank partials (all-reduce of the
scalars and dE/deps, reduce-scatter or all-reduce of Gamma) over gloo,
world size 2, reproduces the unsharded oracle -- each rank's partial is the
oracle restricted to that rank's pairs."""
import os
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("grad", [False, True])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("nocc,nvir,nshards", [(1, 5, 1), (7, 30, 2), (30, 60, 3), (120, 1100, 8), (5, 9, 8)])
def test_shard_pairs_partition(nocc, nvir, nshards, precision, grad):
    sys.path.insert(0, ROOT)
    from ferric_b200 import sharded
    got = []
    sizes = []
    for s in range(nshards):
        p = sharded.shard_pairs(nocc, nvir, s, nshards, precision=precision, grad=grad)
        assert np.all(p[:, 0] <= p[:, 1])
        got += [tuple(x) for x in p]
        sizes.append(len(p))
    assert sorted(got) == [(i, j) for i in range(nocc) for j in range(i, nocc)]
    if nocc * (nocc + 1) // 2 >= 64 * nshards:
        assert max(sizes) <= 1.1 * sum(sizes) / nshards


def test_shard_pairs_refuses_bad_shard():
    sys.path.insert(0, ROOT)
    import ferric_b200._lib as L
    from ferric_b200 import sharded
    with pytest.raises(L.FcError):
        sharded.shard_pairs(10, 10, 2, 2)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    from ferric_b200 import sharded
    from oracle import rimp2 as orc
    from oracle import synthetic
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        b, eo, ev = synthetic.rimp2_inputs(37, 9, 11)   # naux 37: unequal aux bands
        nocc = len(eo)
        pairs = sharded.shard_pairs(nocc, len(ev), rank, world, precision="f64", grad=True)
        e_os, e_ss, g, d_o, d_v = orc.energy_gamma_deps_pairs(b, eo, ev, [tuple(x) for x in pairs])
        full = orc.energy_gamma_deps(b, eo, ev)
        res = []
        for layout in ("band", "full"):
            out = sharded.combine_shards(e_os, e_ss, torch.from_numpy(g.copy()), torch.from_numpy(d_o),
                                         torch.from_numpy(d_v), gamma_layout=layout)
            c_os, c_ss, gout, row0, c_o, c_v = out
            lo, hi = sharded.aux_band(b.shape[0], rank, world) if layout == "band" else (0, b.shape[0])
            res.append((layout, row0 == lo,
                        abs(c_os - full[0]) / abs(full[0]), abs(c_ss - full[1]) / abs(full[1]),
                        float(np.abs(gout.numpy() - full[2][lo:hi]).max() / np.abs(full[2]).max()),
                        float(np.abs(c_o.numpy() - full[3]).max() / np.abs(full[3]).max()),
                        float(np.abs(c_v.numpy() - full[4]).max() / np.abs(full[4]).max()),
                        len(pairs)))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_shard_composition_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert sum(r[1][0][7] for r in out) == 9 * 10 // 2     # the two shards hold every pair
    for rank, res in out:
        for layout, row_ok, eos, ess, g, do, dv, npair in res:
            assert row_ok and npair > 0, (rank, layout)
            assert eos < 1e-12 and ess < 1e-12 and g < 1e-12 and do < 1e-12 and dv < 1e-12, (rank, layout)

"""Failure detection without a GPU fault: a bounded wait that nothing will
end returns FC_ERR_TIMEOUT and leaves the context usable.

The pair kernel's MMA warp waits for each operand stage with a limit
(FERRIC_CUDA_WAIT_MS, default 4 s); FERRIC_CUDA_TEST_DROP_LOAD=1 makes CTA 0's
producer issue no load for its first stage, so that wait runs out with
nothing in flight.  The other roles see the CTA's abort flag and leave their
loops; the producer waits (long limit) for every load it did issue, and TMEM
is released.  The call returns FC_ERR_TIMEOUT within the short limit, the
dispatcher declines to the CPU path on it, and the next call, without the
switch, gives the right energy."""
import time

import numpy as np
import pytest

from oracle import rimp2 as orc
from oracle import synthetic

pytestmark = pytest.mark.gpu


def test_pair_wait_runs_out_and_context_recovers(fc, monkeypatch):
    import ferric_b200._lib as L
    from ferric_b200 import rimp2
    b, eo, ev = synthetic.rimp2_inputs(200, 7, 65)
    ref = orc.spin_components(b, np.concatenate([eo, ev]), 7, 65)
    monkeypatch.setenv("FERRIC_CUDA_WAIT_MS", "50")
    monkeypatch.setenv("FERRIC_CUDA_TEST_DROP_LOAD", "1")
    for call in (lambda: rimp2.rimp2_energy(b, eo, ev, precision="mixed"),
                 lambda: rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")):
        t0 = time.perf_counter()
        with pytest.raises(L.FcError) as ei:
            call()
        assert ei.value.name == "FC_ERR_TIMEOUT"
        assert time.perf_counter() - t0 < 3.0      # the 50 ms limit ended it, not the 4 s default
    before = rimp2.STATS["cpu:FC_ERR_TIMEOUT"]
    assert rimp2.try_spin_components_on_device(b, np.concatenate([eo, ev]), 7, 65, mixed_ok=True) is None
    assert rimp2.STATS["cpu:FC_ERR_TIMEOUT"] == before + 1
    monkeypatch.delenv("FERRIC_CUDA_TEST_DROP_LOAD")
    for _ in range(2):
        e = rimp2.rimp2_energy(b, eo, ev, precision="mixed")
        assert abs(sum(e) - ref[2]) <= 2e-9 * abs(ref[2])
        sc, g, _, _ = rimp2.rimp2_energy_grad(b, eo, ev, precision="mixed")
        assert abs(sc.e_total - ref[2]) <= 2e-9 * abs(ref[2])

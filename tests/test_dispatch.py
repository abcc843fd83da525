"""The device dispatcher's decline and retry rules on the host, with the
device calls replaced by fakes that raise the library's status codes
(rimp2_gpu.rs:105-179): a mixed run that fails with FC_ERR_KERNEL or
FC_ERR_RANGE is retried in FP64 on the device and counted; any other status,
or a failing FP64 retry, declines to the CPU path (None) with the reason
counted; kappa or mixed_ok=False never tries the mixed form."""
import numpy as np
import pytest

from ferric_b200 import _lib, rimp2


def _fake(fail_on):
    calls = []

    def fake(b_ov, eps, nocc, nvir, first_occ=0, nocc_total=None, kappa=None, precision="f64", stats=None):
        calls.append(precision)
        if precision in fail_on:
            raise _lib.FcError(fail_on[precision], "injected")
        return rimp2.SpinComponents(-1.0, -0.5, -1.5)
    return fake, calls


def _run(**kw):
    return rimp2.try_spin_components_on_device(np.zeros((4, 6)), np.zeros(5), 2, 3, **kw)


@pytest.mark.parametrize("status,name", [(8, "FC_ERR_RANGE"), (7, "FC_ERR_KERNEL")])
def test_mixed_failure_retries_in_fp64(monkeypatch, status, name):
    fake, calls = _fake({"mixed": status})
    monkeypatch.setattr(rimp2, "spin_components_on_device", fake)
    before = rimp2.STATS[f"mixed_fallback:{name}"]
    sc = _run(mixed_ok=True)
    assert calls == ["mixed", "f64"]
    assert sc == rimp2.SpinComponents(-1.0, -0.5, -1.5)
    assert rimp2.STATS[f"mixed_fallback:{name}"] == before + 1


@pytest.mark.parametrize("status,name", [(4, "FC_ERR_POOL_FULL"), (9, "FC_ERR_TIMEOUT"), (5, "FC_ERR_LAYOUT")])
def test_other_failures_decline_to_cpu(monkeypatch, status, name):
    fake, calls = _fake({"mixed": status})
    monkeypatch.setattr(rimp2, "spin_components_on_device", fake)
    before = rimp2.STATS[f"cpu:{name}"]
    assert _run(mixed_ok=True) is None
    assert calls == ["mixed"]
    assert rimp2.STATS[f"cpu:{name}"] == before + 1


def test_failed_fp64_retry_declines(monkeypatch):
    fake, calls = _fake({"mixed": 8, "f64": 6})
    monkeypatch.setattr(rimp2, "spin_components_on_device", fake)
    before = rimp2.STATS["cpu:FC_ERR_CUDA"]
    assert _run(mixed_ok=True) is None
    assert calls == ["mixed", "f64"]
    assert rimp2.STATS["cpu:FC_ERR_CUDA"] == before + 1


@pytest.mark.parametrize("kw", [dict(mixed_ok=False), dict(mixed_ok=True, kappa=1.1)])
def test_fp64_only_without_mixed_permission(monkeypatch, kw):
    fake, calls = _fake({})
    monkeypatch.setattr(rimp2, "spin_components_on_device", fake)
    assert _run(**kw) is not None
    assert calls == ["f64"]

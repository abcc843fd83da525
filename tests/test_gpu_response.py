"""The GEMM-shaped RI 3c/2c response (fc_rimp2_response_2c / _3c) against the
oracle's restatement of ri_response_gradient_channels
(ferric-mp2/src/gradient.rs:559-887): FP64 to 1e-12 of the largest element,
tile edges on every dimension, aux slabs, host and device forms."""
import numpy as np
import pytest

from oracle import rimp2 as orc

pytestmark = pytest.mark.gpu


def _inputs(naux, nocc, nvir, nbf, seed=5):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((naux, nocc * nvir)) * 1e-2
    b = rng.standard_normal((naux, nocc * nvir)) * 0.05
    a = rng.standard_normal((naux, naux))
    v = np.linalg.cholesky(a @ a.T / naux + np.eye(naux))  # stands in for V^-1/2 (any square factor)
    c_occ = rng.standard_normal((nbf, nocc)) * 0.3
    c_vir = rng.standard_normal((nbf, nvir)) * 0.3
    return x, b, v, c_occ, c_vir


@pytest.mark.parametrize("naux,nocc,nvir,nbf", [(130, 7, 30, 70), (64, 3, 5, 9), (300, 12, 61, 140)])
def test_response_2c_matches_oracle(fc, naux, nocc, nvir, nbf):
    from ferric_b200 import rimp2
    x, b, v, _, _ = _inputs(naux, nocc, nvir, nbf)
    y_ref, g_ref = orc.response_2c(x, b, v, 2.0)
    st = {}
    y, g = rimp2.rimp2_response_2c(x, b, v, 2.0, stats=st)
    assert np.abs(y - y_ref).max() <= 1e-12 * np.abs(y_ref).max()
    assert np.abs(g - g_ref).max() <= 1e-12 * np.abs(g_ref).max()
    assert st["launches"] == 3 and st["kernel_ms"] > 0


@pytest.mark.parametrize("naux,nocc,nvir,nbf", [(130, 7, 30, 70), (64, 3, 5, 9), (300, 12, 61, 140)])
@pytest.mark.parametrize("p0,np_", [(0, None), (5, 1), (17, 40)])
def test_response_3c_matches_oracle(fc, naux, nocc, nvir, nbf, p0, np_):
    from ferric_b200 import rimp2
    x, b, v, co, cv = _inputs(naux, nocc, nvir, nbf)
    y, _ = orc.response_2c(x, b, v, 2.0)
    n = naux - p0 if np_ is None else np_
    ref = orc.response_3c(y, co, cv, p0, n, 2.0)
    out = rimp2.rimp2_response_3c(y, co, cv, p0, n, 2.0)
    assert out.shape == (n, nbf, nbf)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.array_equal(out, out.transpose(0, 2, 1))


def test_response_device_api(fc):
    import torch
    from ferric_b200 import rimp2
    x, b, v, co, cv = _inputs(130, 7, 30, 70)
    y, g = rimp2.rimp2_response_2c(x, b, v, 1.0)
    yd, gd = rimp2.rimp2_response_2c(*(torch.from_numpy(t).cuda() for t in (x, b, v)), 1.0)
    assert np.array_equal(y, yd.cpu().numpy()) and np.array_equal(g, gd.cpu().numpy())
    o = rimp2.rimp2_response_3c(y, co, cv, 3, 50, 1.0)
    od = rimp2.rimp2_response_3c(torch.from_numpy(y).cuda(), torch.from_numpy(co).cuda(),
                                 torch.from_numpy(cv).cuda(), 3, 50, 1.0)
    assert np.array_equal(o, od.cpu().numpy())


def test_response_refusals(fc):
    from ferric_b200 import rimp2, _lib
    x, b, v, co, cv = _inputs(64, 3, 5, 9)
    y, _ = orc.response_2c(x, b, v)
    with pytest.raises(_lib.FcError) as e:
        rimp2.rimp2_response_3c(y, co, cv, 60, 10)
    assert e.value.name == "FC_ERR_LAYOUT"

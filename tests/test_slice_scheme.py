"""CPU check of the integer-slice contraction the mixed adjoint uses.

Operand rows are split at a power-of-two scale s (max|x|/s in (63.5, 127])
into three int8 slices at weights 1/254, the six slice products are summed
exactly in integers as three levels, and the levels are combined in FP64:
    sum_k a_k b_k ~ s_a s_b ((L0 254 + L1) 254 + L2) / 254^2.
The Q-row operand gets one scale per (Q row, occupied chunk of columns), so
a chunk can be sliced as soon as its columns are on the device; this test
shows that scale is never worse than one per Q row and stays inside the
slice error bound of the exact FP64 product.
"""
import numpy as np

W = 254


def pow2_scale(mx):
    """Power of two with mx / s in (63.5, 127] (1 for an all-zero row)."""
    s = np.ones_like(mx)
    nz = mx > 0
    k = np.frexp(mx[nz])[1]                 # mx = m 2^k, m in [0.5, 1)
    s[nz] = np.ldexp(1.0, k - 7)            # mx / s in [64, 128)
    over = mx > 127.0 * s
    s[over] *= 2.0
    return s


def slices(x, s):
    """Three integer slices of x / s (rows of x, scale per row)."""
    y = x / s[:, None]
    c1 = np.rint(y)
    y2 = (y - c1) * W
    c2 = np.rint(y2)
    c3 = np.rint((y2 - c2) * W)
    for c in (c1, c2, c3):
        assert np.abs(c).max() <= 127
    return [c.astype(np.int64) for c in (c1, c2, c3)]


def sliced_product(a, b):
    """a b^T through the slices: per-row scales of a and b, exact levels."""
    sa, sb = pow2_scale(np.abs(a).max(axis=1)), pow2_scale(np.abs(b).max(axis=1))
    a1, a2, a3 = slices(a, sa)
    b1, b2, b3 = slices(b, sb)
    l0 = a1 @ b1.T
    l1 = a1 @ b2.T + a2 @ b1.T
    l2 = a1 @ b3.T + a2 @ b2.T + a3 @ b1.T
    v = (l0.astype(np.float64) * W + l1) * W + l2
    return v * np.outer(sa, sb) / W**2


def test_chunk_scales_within_bound_and_no_worse():
    rng = np.random.default_rng(11)
    m, n, k, chunk = 48, 40, 360, 120
    a = rng.standard_normal((m, k))          # amplitude rows (i, a) over (j, b)
    b = rng.standard_normal((n, k))          # Q rows over (j, b)
    b[:, 2 * chunk:] *= 1e-3                 # a chunk of much smaller columns
    exact = a @ b.T
    per_row = sliced_product(a, b)
    per_chunk = sum(sliced_product(a[:, c:c + chunk], b[:, c:c + chunk]) for c in range(0, k, chunk))
    # |x - slices(x)| <= s / (2 254^2) per element, plus the three dropped
    # slice products; per-row scales bound the per-chunk ones from above
    sa, sb = pow2_scale(np.abs(a).max(axis=1)), pow2_scale(np.abs(b).max(axis=1))
    da, db = sa / (2 * W**2), sb / (2 * W**2)
    bound = (np.abs(a).sum(axis=1)[:, None] * db[None, :] + da[:, None] * np.abs(b).sum(axis=1)[None, :]
             + k * np.outer(da, db) + k * 127.0**2 * (2.0 / W**3 + 1.0 / W**4) * np.outer(sa, sb))
    err_row = np.abs(per_row - exact)
    err_chunk = np.abs(per_chunk - exact)
    assert (err_row <= bound).all()
    assert (err_chunk <= bound).all()
    # the small chunk's own scale resolves it: the per-chunk error is smaller
    assert err_chunk.max() < err_row.max()


def test_dropped_products_bounded():
    """The six kept products of the slices against the product of the
    slice-reconstructed operands: the difference is the three dropped
    products (c2 c3', c3 c2', c3 c3'), at most 127^2 (2/254^3 + 1/254^4) of
    the row scales per term."""
    rng = np.random.default_rng(5)
    a = rng.standard_normal((16, 96))
    b = rng.standard_normal((12, 96))
    sa, sb = pow2_scale(np.abs(a).max(axis=1)), pow2_scale(np.abs(b).max(axis=1))
    ra = sum(c * w for c, w in zip(slices(a, sa), (1.0, 1.0 / W, 1.0 / W**2))) * sa[:, None]
    rb = sum(c * w for c, w in zip(slices(b, sb), (1.0, 1.0 / W, 1.0 / W**2))) * sb[:, None]
    full = ra @ rb.T
    dropped = np.abs(full - sliced_product(a, b)) / np.outer(sa, sb)
    assert dropped.max() <= 96 * 127.0**2 * (2.0 / W**3 + 1.0 / W**4)

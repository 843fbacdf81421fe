"""The integer-slice product scheme of the mixed path's Gram and rotation
kernels, restated in numpy (no GPU): each band scaled by sigma = 2^e so that
|x| / sigma < 1/2, rounded to a 28-bit fixed-point integer, cut into four
balanced 7-bit digits; a product keeps the digit pairs with t + u <= 3.
Checks the digit range, the reconstruction bound (28 bits of each operand),
that the products (whose error the dropped pairs set, about 2^-21 |a||b|)
are as accurate as an FP32 GEMM of the same operands, and the bias of the
dropped squares on a Gram diagonal (which is why the kernels take that
diagonal from FP64 sums of squares)."""
import numpy as np

S = 4


def digits(x):
    """Per-row sigma and the S balanced base-128 digits, most significant first."""
    m = np.max(np.abs(x), axis=1)
    e = np.where(m > 0, np.frexp(m)[1] + 1, 0)
    sigma = np.ldexp(1.0, e)
    v = np.rint(x / sigma[:, None] * 2.0 ** (7 * S)).astype(np.int64)
    d = np.zeros((S,) + x.shape, dtype=np.int64)
    for t in range(S - 1, 0, -1):
        q = ((v + 64) & 127) - 64
        d[t] = q
        v = (v - q) >> 7
    d[0] = v
    return sigma, d


def product(sa, da, sb, db):
    """sum_k a_k b_k over the kept digit pairs, exact integer accumulation."""
    acc = np.zeros((da.shape[1], db.shape[1]))
    for t in range(S):
        for u in range(S - t):
            acc += (da[t] @ db[u].T).astype(np.float64) * 2.0 ** (-7 * (t + u + 2))
    return acc * sa[:, None] * sb[None, :]


def bands(rng, n=16, k=4000):
    # band-like rows: a few large low-G components and a long small tail
    x = rng.standard_normal((n, k)) / (1.0 + np.arange(k))[None, :] ** 0.7
    return x / np.linalg.norm(x, axis=1)[:, None]


def test_digits_are_int8_and_reconstruct_to_28_bits():
    x = bands(np.random.default_rng(1))
    sigma, d = digits(x)
    assert d.min() >= -64 and d.max() <= 64
    rec = sum(d[t] * 2.0 ** (-7 * (t + 1)) for t in range(S)) * sigma[:, None]
    assert np.max(np.abs(rec - x) / sigma[:, None]) <= 2.0 ** -29 + 1e-18


def test_products_are_as_accurate_as_fp32():
    rng = np.random.default_rng(2)
    a, b = bands(rng), bands(rng)
    sa, da = digits(a)
    sb, db = digits(b)
    exact = a @ b.T
    err = np.abs(product(sa, da, sb, db) - exact)
    assert err.max() < 2.0 ** -21  # unit bands: |a||b| = 1
    f32 = np.abs((a.astype(np.float32) @ b.astype(np.float32).T).astype(np.float64) - exact)
    assert err.max() <= f32.max()


def test_dropped_squares_bias_a_gram_diagonal():
    x = bands(np.random.default_rng(3), n=8, k=60000)
    s, d = digits(x)
    g = product(s, d, s, d)
    exact = x @ x.T
    diag_err = np.diag(g) - np.diag(exact)
    off = g - exact
    np.fill_diagonal(off, 0.0)
    # the diagonal is systematically low (the dropped d_t d_t squares), far
    # beyond the off-diagonal noise
    assert np.all(diag_err < 0)
    assert np.abs(diag_err).min() > 5 * np.abs(off).max()

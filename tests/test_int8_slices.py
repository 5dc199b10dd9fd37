"""The arithmetic of the int8 digit-slice synthesis (gd_ozaki.cu), restated in
numpy and checked on the CPU.

Per operand row (table) or column (coefficients): a power-of-two scale 2^e
with |x| < 2^e, X = rint(x 2^(7G-1-e)) written as G balanced base-128 digits
(d_0 in [-64, 64], the rest in [-64, 63]); products of digit pairs (i, j)
summed per group g = i + j < G (exact in int32), the groups combined exactly
in int64 as sum_g acc_g 128^(G-1-g), one rounding to FP64, times
2^(e_row - 12 - 7(G-1)) 2^(e_col).  Checked: the digits reconstruct X
exactly, every group sum fits int32 with the kernel's K, the combination fits
int64, and the product matches the FP64 product to the scheme's bound
(about K 2^(2-7G) of row max x column max; 6 digits: about 1e-11 of the
largest product on Legendre-like data)."""
import numpy as np
import pytest


def digits(x, e, G):
    """Balanced base-128 digits of rint(x 2^(7G-1-e)), most significant first."""
    X = np.rint(np.ldexp(x, 7 * G - 1 - e)).astype(np.int64)
    out = np.zeros((G,) + X.shape, dtype=np.int64)
    for i in range(G - 1, 0, -1):
        d = ((X + 64) & 127) - 64
        out[i] = d
        X = (X - d) >> 7
    out[0] = X
    return out


def exponent(amax):
    """Smallest e with |x| < 2^e (0 for an all-zero row)."""
    e = np.where(amax > 0, np.frexp(np.where(amax > 0, amax, 1.0))[1], 0)
    return e.astype(np.int64)


def int8_product(A, B, G):
    """A (M x K) times B (K x N) by the digit-slice scheme of the kernel."""
    ea = exponent(np.max(np.abs(A), axis=1))            # per row
    eb = exponent(np.max(np.abs(B), axis=0))            # per column
    da = digits(A, ea[:, None], G)                      # G x M x K
    db = digits(B, eb[None, :], G)                      # G x K x N
    acc = []
    for g in range(G):
        s = sum(da[i] @ db[g - i] for i in range(g + 1))
        assert np.max(np.abs(s)) < 2 ** 31                # the TMEM accumulators are int32
        acc.append(s)
    S = acc[0].copy()
    for g in range(1, G):
        S = S * 128 + acc[g]                            # exact in int64
    assert np.max(np.abs(S)) < 2 ** 62
    return np.ldexp(S.astype(np.float64), (ea - 12 - 7 * (G - 1))[:, None] + eb[None, :]), ea, eb


def legendre_like(rng, M, K):
    # rows of very different magnitude along K, like Pbar_l^m(theta) near the poles
    scale = np.exp(-rng.uniform(0, 30, size=(M, 1)) * np.linspace(0, 1, K)[None, :] ** 2)
    return rng.standard_normal((M, K)) * scale


@pytest.mark.parametrize("G", [5, 6])
def test_digits_reconstruct_exactly(G):
    rng = np.random.default_rng(G)
    x = rng.standard_normal(4096) * np.exp(rng.uniform(-20, 20, 4096))
    e = exponent(np.abs(x))
    d = digits(x, e, G)
    assert d[0].min() >= -64 and d[0].max() <= 64
    assert d[1:].min() >= -64 and d[1:].max() <= 63
    X = np.rint(np.ldexp(x, 7 * G - 1 - e)).astype(np.int64)
    rec = np.zeros_like(X)
    for i in range(G):
        rec = rec * 128 + d[i]
    assert np.array_equal(rec, X)
    # the rounding leaves at most half a unit of the last digit
    assert np.all(np.abs(np.ldexp(X.astype(np.float64), e - (7 * G - 1)) - x) <= np.ldexp(0.5, e - (7 * G - 1)))


@pytest.mark.parametrize("G,bound", [(6, 5e-11), (5, 5e-9)])
def test_product_matches_fp64(G, bound):
    rng = np.random.default_rng(10 + G)
    M, K, N = 128, 128, 32                               # one tile, one parity of lmax 255
    A = legendre_like(rng, M, K)
    B = rng.standard_normal((K, N)) * (np.arange(K)[:, None] + 1.0) ** -2
    C, ea, eb = int8_product(A, B, G)
    ref = A @ B
    scale = np.max(np.abs(A), axis=1)[:, None] * np.max(np.abs(B), axis=0)[None, :]
    err = np.abs(C - ref) / scale
    # the scheme's bound: each of K terms within a few units of 2^-7G of row x column max
    assert np.max(err) <= K * 2.0 ** (2 - 7 * G)
    assert np.max(np.abs(C - ref)) / np.max(np.abs(ref)) < bound


def test_zero_rows_and_columns():
    A = np.zeros((8, 32))
    A[1] = 1.0
    B = np.zeros((32, 4))
    B[:, 2] = -3.5
    C, _, _ = int8_product(A, B, 6)
    assert np.array_equal(C, A @ B)

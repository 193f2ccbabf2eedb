"""Integer-tensor-core products of FP64 matrices (scy_ozaki_matmul) on the GPU.

The product splits every row of X and W into S signed 8-bit digit planes
scaled by a power of two, multiplies the planes exactly on the tensor cores
(tcgen05.mma kind::i8, 32-bit accumulators) and combines the digit-weight
groups in FP64.  ``emulate`` restates that arithmetic in numpy: with exact
integer products and the same combination order the device must agree with
it to the last bit (up to one rounding of the final FP64 sums); against the
plain FP64 product the error per row is about 100^-S.
"""
import ctypes as C

import numpy as np
import pytest

from scycle_b200 import _lib as S

pytestmark = pytest.mark.gpu


def digits(X, s):
    m = np.abs(X).max(axis=1)
    _, p = np.frexp(m)  # m = f 2^p, f in [1/2, 1): ilogb(m) = p - 1
    e = np.where(m > 0, p.astype(np.int64) + 1, 0)
    t = np.ldexp(X, (7 - e)[:, None])
    D = []
    for _ in range(s):
        d = np.rint(t)
        D.append(d.astype(np.int64))
        t = (t - d) * 128.0
    return D, e


def emulate(X, W, s):
    dx, ex = digits(X, s)
    dw, ew = digits(W, s)
    acc = np.zeros((X.shape[0], W.shape[0]))
    for g in range(s - 1, -1, -1):
        P = np.zeros(acc.shape, dtype=np.int64)
        for i in range(1, g + 2):
            P += dx[i - 1] @ dw[g + 1 - i].T
        assert np.abs(P).max() < 2 ** 31
        acc += P.astype(np.float64) * 2.0 ** (-7 * (g + 2))
    return np.ldexp(acc, ex[:, None] + ew[None, :])


BOUND = {3: 1e-4, 4: 1e-6, 5: 1e-8, 6: 1e-10, 7: 1e-12}


def _matmul(X, W, s, ldx=None, ldd=None, ctas=1, bf16=0):
    import torch
    rows, K = X.shape[0], W.shape[1]
    cols = W.shape[0]
    ldx = ldx or X.shape[1]
    ldd = ldd or cols
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    Dd = torch.zeros((rows, ldd), dtype=torch.float64, device="cuda")
    S.check(S.lib().scy_ozaki_matmul(C.c_void_p(Xd.data_ptr()), ldx, rows, K, S.as_dptr(np.ascontiguousarray(W)), K,
                                     cols, s, C.c_void_p(Dd.data_ptr()), ldd, ctas, bf16))
    return Dd.cpu().numpy()


@pytest.mark.parametrize("s", [3, 4, 5, 6, 7])
@pytest.mark.parametrize("rows,K,cols", [(300, 401, 401), (1000, 129, 200)])
def test_ozaki_matmul_matches_emulation_and_fp64(s, rows, K, cols):
    rng = np.random.default_rng(s * 100 + K)
    X = rng.standard_normal((rows, K)) * np.exp(3 * rng.standard_normal((rows, 1)))
    X[:, : K // 8] *= 1e-5
    X[7] = 0.0  # an all-zero row
    Q, _ = np.linalg.qr(rng.standard_normal((K, K)))
    W = np.ascontiguousarray(np.vstack([Q, Q])[:cols])
    D = _matmul(X, W, s)
    E = emulate(X, W, s)
    assert np.all(np.isfinite(D))
    assert np.all(D[7] == 0.0)
    np.testing.assert_allclose(D, E, rtol=1e-15, atol=1e-300)
    exact = X @ W.T
    rel = np.linalg.norm(D - exact, axis=1) / np.maximum(np.linalg.norm(exact, axis=1), 1e-300)
    assert rel.max() <= BOUND[s], rel.max()


def test_ozaki_matmul_strided_rows():
    """Row strides larger than K (the padded layouts the preconditioner uses)."""
    rng = np.random.default_rng(5)
    rows, K, cols, ldx, ldd = 257, 401, 401, 404, 404
    Xfull = rng.standard_normal((rows, ldx))
    W = rng.standard_normal((cols, K))
    D = _matmul(Xfull, W, 7, ldx=ldx, ldd=ldd)
    np.testing.assert_allclose(D[:, :cols], emulate(Xfull[:, :K], W, 7), rtol=1e-15, atol=1e-300)
    assert np.all(D[:, cols:] == 0.0)


@pytest.mark.parametrize("s", [3, 4, 5])
def test_ozaki_two_ctas_per_sm_shape_gives_the_same_product(s):
    """The two-CTAs-per-SM shape (narrower column tiles, half the tensor
    memory each) gives bit-for-bit the product of the one-CTA shape: the
    digit products are exact integers and the epilogue combines them in the
    same order."""
    rng = np.random.default_rng(40 + s)
    rows, K, cols = 700, 401, 401
    X = rng.standard_normal((rows, K)) * np.exp(2 * rng.standard_normal((rows, 1)))
    W = rng.standard_normal((cols, K))
    D1 = _matmul(X, W, s, ctas=1)
    D2 = _matmul(X, W, s, ctas=2)
    assert np.array_equal(D1, D2)
    np.testing.assert_allclose(D2, emulate(X, W, s), rtol=1e-15, atol=1e-300)


@pytest.mark.parametrize("s", [3, 4, 5])
@pytest.mark.parametrize("rows,K,cols", [(700, 401, 401), (5000, 401, 401), (1500, 129, 200)])
@pytest.mark.parametrize("bf16", [0, 1])
def test_ozaki_persistent_shape_gives_the_same_product(s, rows, K, cols, bf16):
    """The persistent shape (one CTA per SM walking the tiles, two
    accumulator sets in tensor memory, one tile's epilogue under the next
    tile's products) gives bit-for-bit the product of the one-CTA-per-tile
    shape: with fewer tiles than SMs, with several tiles per CTA (5000 rows:
    40 x 9 tiles), and with a narrow last column tile."""
    rng = np.random.default_rng(80 + s + rows)
    X = rng.standard_normal((rows, K)) * np.exp(2 * rng.standard_normal((rows, 1)))
    X[3] = 0.0
    W = rng.standard_normal((cols, K))
    D1 = _matmul(X, W, s, ctas=1, bf16=bf16)
    D0 = _matmul(X, W, s, ctas=0, bf16=bf16)
    assert np.array_equal(D0, D1)
    assert np.all(D0[3] == 0.0)


@pytest.mark.parametrize("s", [3, 4, 5, 6, 7])
@pytest.mark.parametrize("ctas", [1, 2])
def test_ozaki_bf16_digits_give_the_same_product(s, ctas):
    """The digits held in bf16 and multiplied with FP32 accumulation
    (kind::f16) give bit-for-bit the integer product (kind::i8): every
    partial sum stays below 2^24 at K = 401."""
    if ctas == 2 and s > 5:
        pytest.skip("two CTAs per SM only for S <= 5")
    rng = np.random.default_rng(60 + s)
    rows, K, cols = 600, 401, 401
    X = rng.standard_normal((rows, K)) * np.exp(2 * rng.standard_normal((rows, 1)))
    X[5] = 0.0
    W = rng.standard_normal((cols, K))
    D8 = _matmul(X, W, s, ctas=ctas, bf16=0)
    D16 = _matmul(X, W, s, ctas=ctas, bf16=1)
    assert np.array_equal(D8, D16)

"""The FP64 product on the integer tensor cores (tpe_gemm_nt_device with
TPE_GEMM_INT8_EMULATED), the building block of the large-constraint-set mixed
solve. Every integer digit product is exact, so the result is checked bit for
bit against a numpy restatement of the same splitting and summation order
(level sums formed exactly in float64: every partial sum stays below 2^53), and
against the plain FP64 product within the scheme's error bound. Covers ragged
shapes, K longer than one launch (4096), the triangular K ranges, lower-tile
updates with the upper triangle left alone, B as a band of A's rows (shared
digits), alpha/beta, and NaN propagation. The FP64 tensor-core method is checked
against numpy too."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from repulsive_test2_b200 import abi
from repulsive_test2_b200 import api as T

pytestmark = pytest.mark.gpu

S = 8
MAX_K = 4096


def split_np(X):
    """Row scales e (|x| < 2^e) and the eight digits of each element."""
    m = np.max(np.abs(X), axis=1)
    e = np.where(m > 0, np.frexp(m)[1], 0).astype(np.int64)
    y = np.ldexp(X, (7 - e)[:, None])
    f = np.floor(y)
    digits = [f]
    r = y - f
    for _ in range(1, S):
        r = r * 256.0
        f = np.floor(r)
        digits.append(f)
        r = r - f
    return digits, e


def ozaki_np(A, B, C0, alpha, beta):
    """The emulated product, in the kernel's order (launch by launch over K)."""
    K = A.shape[1]
    out = C0.copy()
    for c, k0 in enumerate(range(0, K, MAX_K)):
        k1 = min(K, k0 + MAX_K)
        dA, ea = split_np(A)
        dB, eb = split_np(B)
        acc = np.zeros((A.shape[0], B.shape[0]))
        for g in range(S - 1, -1, -1):
            lvl = sum(dA[p][:, k0:k1] @ dB[g - p][:, k0:k1].T for p in range(g + 1))
            acc = acc + lvl * 2.0 ** -(14 + 8 * g)
        y = alpha * np.ldexp(acc, ea[:, None] + eb[None, :])
        b = beta if c == 0 else 1.0
        if b != 0.0:
            y = y + b * out
        out = y
    return out


def _gemm(method, A, B, C0, alpha=1.0, beta=0.0, mode=0, b_rows_of_a=None):
    import torch

    ctx = T.context()
    dev = torch.device("cuda", 0)
    dA = torch.from_numpy(np.ascontiguousarray(A)).to(dev)
    if b_rows_of_a is None:
        dB = torch.from_numpy(np.ascontiguousarray(B)).to(dev)
        pb, N = dB.data_ptr(), B.shape[0]
    else:
        off, N = b_rows_of_a
        pb = dA.data_ptr() + off * A.shape[1] * 8
    dC = torch.from_numpy(np.ascontiguousarray(C0)).to(dev)
    torch.cuda.synchronize()
    M, K = A.shape
    rc = ctx.lib.tpe_gemm_nt_device(ctx.ptr, method, M, N, K, dA.data_ptr(), K, pb, K,
                                    dC.data_ptr(), N, alpha, beta, mode)
    torch.cuda.synchronize()
    assert rc == 0, ctx.lib.tpe_last_error(ctx.ptr)
    return dC.cpu().numpy()


def _bound(A, B):
    K = A.shape[1]
    return 4.0 * K * 2.0 ** -53 * np.max(np.abs(A), axis=1)[:, None] * np.max(np.abs(B), axis=1)[None, :]


@pytest.mark.parametrize("M,N,K", [(200, 150, 300), (128, 64, 64), (130, 70, 4200), (1, 3, 5)])
def test_int8_emulated_bitexact(M, N, K):
    rng = np.random.default_rng(M * 7 + N + K)
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-8, 8, (M, 1)))
    B = rng.standard_normal((N, K)) * np.exp(rng.uniform(-8, 8, (N, 1)))
    C0 = rng.standard_normal((M, N))
    for alpha, beta in [(1.0, 0.0), (-1.0, 1.0), (0.75, -0.5)]:
        got = _gemm(abi.GEMM_INT8_EMULATED, A, B, C0, alpha, beta)
        want = ozaki_np(A, B, C0, alpha, beta)
        np.testing.assert_array_equal(got, want)
        exact = alpha * (A @ B.T) + beta * C0
        assert np.all(np.abs(got - exact) <= abs(alpha) * _bound(A, B) + 1e-15 * np.abs(exact))


def test_int8_emulated_triangular_and_lower_update():
    rng = np.random.default_rng(3)
    n, K = 300, 260
    A = rng.standard_normal((n, K))
    # triangular operands: the skipped K ranges hold zeros, so the product is unchanged
    U = np.triu(rng.standard_normal((n, n)))
    L = np.tril(rng.standard_normal((n, n)))
    Bf = rng.standard_normal((n, n))
    C0 = np.zeros((n, n))
    for mode, Aop, Bop in [(2, U, Bf), (4, L, Bf), (8, Bf, U), (16, Bf, L)]:
        got = _gemm(abi.GEMM_INT8_EMULATED, Aop, Bop, C0, 1.0, 0.0, mode)
        np.testing.assert_array_equal(got, ozaki_np(Aop, Bop, C0, 1.0, 0.0))
    # symmetric lower update C -= A A^T (lower tiles, column <= row), upper part untouched
    C0 = rng.standard_normal((n, n))
    got = _gemm(abi.GEMM_INT8_EMULATED, A, A, C0, -1.0, 1.0, 1 | 32)
    want = ozaki_np(A, A, C0, -1.0, 1.0)
    low = np.tril(np.ones((n, n), dtype=bool))
    np.testing.assert_array_equal(got[low], want[low])
    np.testing.assert_array_equal(got[~low], C0[~low])


def test_int8_emulated_shared_rows_and_nan():
    rng = np.random.default_rng(4)
    M, K, off, N = 333, 190, 130, 70
    A = rng.standard_normal((M, K))
    C0 = np.zeros((M, N))
    got = _gemm(abi.GEMM_INT8_EMULATED, A, None, C0, 1.0, 0.0, 0, b_rows_of_a=(off, N))
    np.testing.assert_array_equal(got, ozaki_np(A, A[off:off + N], C0, 1.0, 0.0))
    A[5, 17] = np.nan
    B = rng.standard_normal((40, K))
    got = _gemm(abi.GEMM_INT8_EMULATED, A, B, np.zeros((M, 40)), 1.0, 0.0)
    assert np.all(np.isnan(got[5])) and np.all(np.isfinite(np.delete(got, 5, axis=0)))


def test_fp64_method_matches_numpy():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((257, 300))
    B = rng.standard_normal((129, 300))
    C0 = rng.standard_normal((257, 129))
    got = _gemm(abi.GEMM_FP64, A, B, C0, -1.0, 1.0)
    want = C0 - A @ B.T
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))

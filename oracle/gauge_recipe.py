"""Synthetic gauge field of the benchmark workloads, restated in numpy.

Test and baseline infrastructure only: the reference arm of bench.py and the
tests use it to build their inputs without loading the CUDA library.  The
product's generator is `cvcb_gauge_random` (cvc_b200/csrc/host_geometry.cpp);
tests/test_host.py checks that the two agree.

Recipe (the reference has no generator for it; its pieces are the
reference's own): random numbers from ranlxd (ranlxd.c) after
rlxd_init(1, seed), drawn with the reference library when it is given, else
with the oracle's restatement; per link (site-major, mu = 0..3) eight
normal deviates w_a from four Box-Muller pairs in rangauss's order
(cvc_utils.c:2734-2760); H = sum_a w_a lambda_a / 2 (Gell-Mann matrices);
U = exp(i eps H) by scaling and squaring of a 16-term Taylor series (Moler
and Van Loan, method 3), then rows 0, 1 Gram-Schmidt orthonormalised and
row 2 = conj(row0 x row1), so that U is special unitary up to rounding.
Link U_mu(x) is stored at 18*(4x + mu), row-major, (re, im) pairs
(global.h:55-61).
"""
import numpy as np

_S3 = 1.0 / np.sqrt(3.0)


def _gell_mann_h(w):
    """H = sum_a w_a lambda_a / 2 without the 1/2 (applied with eps)."""
    n = w.shape[0]
    H = np.zeros((n, 3, 3), np.complex128)
    H[:, 0, 1] += w[:, 0]; H[:, 1, 0] += w[:, 0]
    H[:, 0, 1] += -1j * w[:, 1]; H[:, 1, 0] += 1j * w[:, 1]
    H[:, 0, 0] += w[:, 2]; H[:, 1, 1] += -w[:, 2]
    H[:, 0, 2] += w[:, 3]; H[:, 2, 0] += w[:, 3]
    H[:, 0, 2] += -1j * w[:, 4]; H[:, 2, 0] += 1j * w[:, 4]
    H[:, 1, 2] += w[:, 5]; H[:, 2, 1] += w[:, 5]
    H[:, 1, 2] += -1j * w[:, 6]; H[:, 2, 1] += 1j * w[:, 6]
    H[:, 0, 0] += w[:, 7] * _S3; H[:, 1, 1] += w[:, 7] * _S3; H[:, 2, 2] += -2 * w[:, 7] * _S3
    return H


def _expm(A):
    """exp(A) for a stack of 3x3 matrices: scaling and squaring of a
    16-term Taylor series, the scale chosen per matrix so that the l1 sum
    of |Re| + |Im| over its entries is <= 1/2."""
    nrm = np.sum(np.abs(A.real) + np.abs(A.imag), axis=(1, 2))
    s = np.zeros(A.shape[0], np.int64)
    x = nrm.copy()
    while True:
        m = x > 0.5
        if not m.any():
            break
        x[m] *= 0.5
        s[m] += 1
    out = np.empty_like(A)
    for sv in np.unique(s):
        idx = np.nonzero(s == sv)[0]
        a = A[idx] * np.ldexp(1.0, -int(sv))
        term = np.broadcast_to(np.eye(3, dtype=np.complex128), a.shape).copy()
        total = term.copy()
        for k in range(1, 17):
            term = np.matmul(term, a) / k
            total += term
        for _ in range(int(sv)):
            total = np.matmul(total, total)
        out[idx] = total
    return out


def _reunitarise(U):
    r0 = U[:, 0, :] / np.linalg.norm(U[:, 0, :], axis=1, keepdims=True)
    p = np.sum(np.conj(r0) * U[:, 1, :], axis=1, keepdims=True)
    r1 = U[:, 1, :] - p * r0
    r1 = r1 / np.linalg.norm(r1, axis=1, keepdims=True)
    r2 = np.conj(np.cross(r0, r1))
    return np.stack([r0, r1, r2], axis=1)


def gauge_random(T, LX, LY, LZ, eps, seed, ranlxd, chunk=1 << 18):
    """72*V doubles; `ranlxd(n, seed)` returns the first n numbers of the
    ranlxd stream at level 1 (the reference's generator or a restatement)."""
    V = T * LX * LY * LZ
    nlink = 4 * V
    r = np.asarray(ranlxd(8 * nlink, seed), np.float64).reshape(nlink, 4, 2)
    g = np.empty((nlink, 3, 3), np.complex128)
    for a in range(0, nlink, chunk):
        b = min(nlink, a + chunk)
        x1, x2 = r[a:b, :, 0], r[a:b, :, 1]
        rad = np.sqrt(-2.0 * np.log(x1))
        w = np.empty((b - a, 8))
        w[:, 0::2] = rad * np.cos(2 * np.pi * x2)
        w[:, 1::2] = rad * np.sin(2 * np.pi * x2)
        A = 0.5j * eps * _gell_mann_h(w)
        g[a:b] = _reunitarise(_expm(A))
    return g.view(np.float64).reshape(-1).copy()

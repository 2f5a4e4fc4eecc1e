"""CPU oracle of the split-precision BSE GEMM (TEST INFRASTRUCTURE ONLY).

The reference's BSE is an FP64 ZGEMM (parquet_BSE.f90:72-128).  The
library's split mode emulates it with int8 slices (Ozaki's error-free
splitting, Ozaki, Ogita, Oishi & Rump, Numer. Algorithms 59 (2012)):

* the complex product C = A B (M x K times K x N) is written as one real
  product C' = A' B' with A' = [Re A | Im A] (M x 2K) and B' whose column
  2j is [Re B_j ; -Im B_j] and column 2j+1 is [Im B_j ; Re B_j], so that
  C'[:, 2j] = Re C_j and C'[:, 2j+1] = Im C_j;
* each row of A' is scaled by 2^-e (e the smallest integer with
  max|row| < 2^e) and cut into s int8 slices of 7 bits,
  a = sum_i 2^(-7(i+1)) a_i, a_i = trunc(2^7 r_i) with the running
  remainder r_i (exact in FP64); columns of B' likewise;
* the slice products with i + j = d (d < s) are summed exactly in int32
  and combined in FP64: C' = 2^(e+f) sum_d 2^(-7(d+2)) D_d.

The GPU path must produce the same int8 slices (bit-exact) and the same
FP64 result up to the order of the final FP64 additions.
"""
from __future__ import annotations

import numpy as np

SLICE_BITS = 7


def exponents(maxabs: np.ndarray) -> np.ndarray:
    """Smallest integer e with maxabs < 2^e (0 for an all-zero line)."""
    m, e = np.frexp(maxabs)       # maxabs = m 2^e, 0.5 <= m < 1  ->  maxabs < 2^e
    return np.where(maxabs > 0, e, 0).astype(np.int64)


def slice_lines(X: np.ndarray, s: int) -> tuple[np.ndarray, np.ndarray]:
    """Rows of the real matrix X -> (s, rows, cols) int8 slices and row exponents."""
    e = exponents(np.max(np.abs(X), axis=1))
    r = np.ldexp(X, -e[:, None])          # |r| < 1
    out = np.zeros((s,) + X.shape, dtype=np.int8)
    for i in range(s):
        x = r * 2.0 ** SLICE_BITS           # |x| < 128
        a = np.trunc(x)
        out[i] = a.astype(np.int8)
        r = x - a
    return out, e


def real_forms(A: np.ndarray, B: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """A' (M x 2K) and B'^T (2N x 2K, one row per column of B')."""
    Ap = np.concatenate([A.real, A.imag], axis=1)
    K, N = B.shape
    Bt = np.empty((2 * N, 2 * K))
    Bt[0::2] = np.concatenate([B.real, -B.imag], axis=0).T
    Bt[1::2] = np.concatenate([B.imag, B.real], axis=0).T
    return Ap, Bt


def ozaki_zgemm(A: np.ndarray, B: np.ndarray, s: int) -> np.ndarray:
    """Complex A @ B through s int8 slices per operand (triangular, i + j < s)."""
    Ap, Bt = real_forms(A, B)
    sa, ea = slice_lines(Ap, s)
    sb, eb = slice_lines(Bt, s)
    acc = np.zeros((Ap.shape[0], Bt.shape[0]))
    for d in range(s):
        D = np.zeros((Ap.shape[0], Bt.shape[0]), dtype=np.int64)
        for i in range(d + 1):
            D += sa[i].astype(np.int64) @ sb[d - i].astype(np.int64).T
        assert np.max(np.abs(D)) < 2 ** 31          # int32 accumulation is exact
        acc = acc + np.ldexp(D.astype(np.float64), -SLICE_BITS * (d + 2))
    Cp = np.ldexp(np.ldexp(acc, ea[:, None]), eb[None, :])
    return Cp[:, 0::2] + 1j * Cp[:, 1::2]


def bse_split(gamma: np.ndarray, F: np.ndarray, chi: np.ndarray, scale: float, f: float, s: int) -> np.ndarray:
    """One damped BSE update (parquet_BSE.f90:72-128) for one (q, r) with the
    GEMM [Gamma chi | F] [F ; chi Gamma] in split precision:
    Phi = scale [.] + (1 - f)(F - Gamma), scale = c_r f / (beta Nx Ny)."""
    A = np.concatenate([gamma @ chi, F], axis=1)
    B = np.concatenate([F, chi @ gamma], axis=0)
    return scale * ozaki_zgemm(A, B, s) + (1.0 - f) * (F - gamma)

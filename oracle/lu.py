"""FP64 LU oracle of the BSE's LU form (TEST INFRASTRUCTURE ONLY).

F = (1 - c Gamma chi)^{-1} Gamma with LAPACK zgetrf/zgetrs (scipy), the
dense chi built from its nu-diagonal blocks.  The reference has no LU mode
(its BSE is the damped update of parquet_BSE.f90:72-128); the two agree at
the fixed point, which ``damped_fixed_point`` reproduces by iterating that
update until it stops moving.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla


def chi_dense(chi_blocks: np.ndarray) -> np.ndarray:
    nl, _, nf = chi_blocks.shape
    n = nl * nf
    out = np.zeros((n, n), dtype=np.complex128)
    nu = np.arange(nf)
    for a in range(nl):
        for b in range(nl):
            out[a * nf + nu, b * nf + nu] = chi_blocks[a, b, :]
    return out


def bse_lu(gamma: np.ndarray, chi_blocks: np.ndarray, scale: float = 1.0) -> np.ndarray:
    """F = (I - scale Gamma chi)^{-1} Gamma via zgetrf/zgetrs."""
    n = gamma.shape[0]
    A = np.eye(n, dtype=np.complex128) - scale * (gamma @ chi_dense(chi_blocks))
    lu, piv = sla.lu_factor(A, check_finite=False)
    return sla.lu_solve((lu, piv), gamma, check_finite=False)


def damped_fixed_point(gamma: np.ndarray, chi_blocks: np.ndarray, scale: float, f: float = 0.5,
                       tol: float = 1e-14, max_iter: int = 100000) -> np.ndarray:
    """Iterate the reference's BSE update (parquet_BSE.f90:72-128) with Gamma
    held fixed, Phi <- f c' [Gamma chi F + F chi Gamma] + (1 - f) Phi,
    F = Gamma + Phi, where c' = scale/2 per ordering (c_r/(beta N) = scale/2
    for the symmetric two-ordering form); returns F at the fixed point."""
    chi = chi_dense(chi_blocks)
    phi = np.zeros_like(gamma)
    for _ in range(max_iter):
        F = gamma + phi
        new = f * 0.5 * scale * (gamma @ chi @ F + F @ chi @ gamma) + (1.0 - f) * phi
        if np.max(np.abs(new - phi)) <= tol * max(np.max(np.abs(new)), 1e-300):
            return gamma + new
        phi = new
    raise RuntimeError("damped BSE iteration did not converge")

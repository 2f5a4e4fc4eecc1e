"""CPU oracle of the learned warm start (TEST INFRASTRUCTURE ONLY).

The reference has no warm start: its loop starts from Sigma = 0 (or a DMFT
Sigma) and F_r = Gamma_r = Lambda_r on the (l=1, l=1) nu-block
(preprocessing.f90:100-116).  The library's warm start replaces that state
at the same hook; this module restates it in numpy:

* ``warm_start``: Sigma <- sigma, mu by the bisection of calc_Gkw_Grt
  (parquet_chi.f90:18-210), Gamma_r <- gamma_l1[r] on the (l=1, l=1)
  nu-block, and F_r = (1 - 2 c_r/(beta Nx Ny) Gamma_r chi_r)^{-1} Gamma_r,
  the fixed point of the damped BSE update (parquet_BSE.f90:72-128).
* ``mlp_*``: the network the library trains, in float64 — SiLU hidden
  layers, linear output, mean-squared-error loss, flat parameters
  [W_0, b_0, W_1, b_1, ...] with W_l (out, in) row-major.
"""
from __future__ import annotations

import numpy as np

from . import tups_oracle as O


def warm_start(st: O.State, sigma: np.ndarray, gamma_l1) -> None:
    Nf, Nz = st.Nf, st.Nz
    st.Sigma[:] = np.asarray(sigma, dtype=np.complex128).reshape(-1)
    O.calc_Gkw_Grt(st, 0, False)
    alpha = 1.0 / (st.p.beta * st.Nx * st.Ny)
    for r, g in zip("dmst", np.asarray(gamma_l1, dtype=np.complex128).reshape(4)):
        st.G[r][...] = 0.0
        st.G[r][:Nf, :Nf, :] = g
    eye = np.eye(Nz, dtype=np.complex128)
    for iq in range(st.Nb):
        qx, qy, w = (int(v) for v in st.ibz[iq])
        cph, cpp = O.calc_chi(st, qx, qy, w)
        for r in "dmst":
            chi = cph if r in "dm" else cpp
            gam = st.G[r][:, :, iq]
            s = 2.0 * O.BSE_COEF[r] * alpha
            st.F[r][:, :, iq] = np.linalg.solve(eye - s * (gam @ chi), gam)


def mlp_layout(widths):
    """[(w_off, b_off, fan_in, fan_out)] per linear layer and the total size."""
    out, off = [], 0
    for fin, fout in zip(widths[:-1], widths[1:]):
        out.append((off, off + fin * fout, fin, fout))
        off += fin * fout + fout
    return out, off


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mlp_forward(params: np.ndarray, widths, x: np.ndarray):
    """Returns (y, cache) for x (batch, n_in)."""
    layout, n = mlp_layout(widths)
    assert params.size == n
    p = params.astype(np.float64)
    a = x.astype(np.float64)
    cache = [(a, None)]
    for i, (wo, bo, fin, fout) in enumerate(layout):
        W = p[wo:wo + fin * fout].reshape(fout, fin)
        b = p[bo:bo + fout]
        z = a @ W.T + b
        if i < len(layout) - 1:
            a = _silu(z)
        else:
            a = z
        cache.append((a, z))
    return a, cache


def mlp_loss_grad(params: np.ndarray, widths, x: np.ndarray, t: np.ndarray):
    """Mean squared error over batch x n_out and its gradient (float64)."""
    layout, n = mlp_layout(widths)
    y, cache = mlp_forward(params, widths, x)
    d = y - t.astype(np.float64)
    loss = float(np.mean(d * d))
    grad = np.zeros(n)
    dz = 2.0 * d / d.size
    p = params.astype(np.float64)
    for i in range(len(layout) - 1, -1, -1):
        wo, bo, fin, fout = layout[i]
        a_in = cache[i][0]
        grad[wo:wo + fin * fout] = (dz.T @ a_in).reshape(-1)
        grad[bo:bo + fout] = dz.sum(axis=0)
        if i > 0:
            W = p[wo:wo + fin * fout].reshape(fout, fin)
            dz = (dz @ W) * _dsilu(cache[i][1])
    return loss, grad


"""Frequency-dependent Lambda tables for the DGA input tests.

The PA constants (d = U, m = -U, s = 2U, t = 0) plus a smooth perturbation
that decays with the fermionic frequencies and the bosonic index: real part
symmetric under nu1 <-> nu2 and under the mirror nu -> Nf + 1 - nu of both,
imaginary part odd under that mirror, as a local vertex of the Hubbard model
has them.  Seeded amplitudes per channel.
"""
from __future__ import annotations

import numpy as np

from oracle import tups_oracle as O


def dga_tables(Nf: int, U: float, seed: int = 0, eps: float = 0.2) -> dict:
    rng = np.random.default_rng(seed)
    x = np.arange(1, Nf + 1) - (Nf + 1) / 2.0
    x1, x2 = np.meshgrid(x, x, indexing="ij")
    w = np.arange(Nf // 2)
    env = np.exp(-(x1 ** 2 + x2 ** 2) / (0.5 * Nf * Nf))[:, :, None] / (1.0 + w[None, None, :] ** 2 / 4.0)
    odd = ((x1 + x2) / Nf)[:, :, None]
    base = {"d": U, "m": -U, "s": 2.0 * U, "t": 0.0}
    out = {}
    for r in "dmst":
        a, b = rng.uniform(0.5, 1.0, size=2)
        out[r] = (base[r] + eps * U * (a * env + 1j * b * odd * env)).astype(np.complex128)
    return out


def write_dga_files(stem: str, L: dict) -> None:
    """``stem``_ph.init holds (d, m), ``stem``_pp.init holds (s, t)."""
    O.write_lambda_file(stem + "_ph.init", L["d"], L["m"])
    O.write_lambda_file(stem + "_pp.init", L["s"], L["t"])

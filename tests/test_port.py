"""The compiled port of the oracle's crossing and Phi(R) phases (the CPU
baseline of the benchmark) against the numpy oracle, phase by phase and over
whole iterations."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import port as P
from oracle import tups_oracle as O


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("case", [
    dict(Nx=4, Nf=8, neighbours=2),
    dict(Nx=8, Nf=8, neighbours=3, tprime=-0.2),
    dict(Nx=4, Nf=16, neighbours=1),
], ids=["nl5", "nl9_tprime", "nl1"])
def test_port_phases_match_oracle(case):
    p = O.Params(beta=2.0, U=2.0, nParticle=0.9, f_damping=0.5, ite_max=10, **case)
    st = O.initialize(p)
    O.iteration(st, 0)
    O.calc_Gkw_Grt(st, 1, False)
    O.bse(st, 1)
    O.calc_PhiR(st)
    ref = {r: st.PhiR[r].copy() for r in "dmst"}
    P.calc_PhiR(st)
    assert max(_rel(st.PhiR[r], ref[r]) for r in "dmst") < 1e-13
    O.calculate_PAE(st)
    ref = {r: st.F[r].copy() for r in "dmst"}
    P.calculate_PAE(st)
    assert max(_rel(st.F[r], ref[r]) for r in "dmst") < 1e-13


def test_port_iterations_match_oracle():
    p = O.Params(beta=2.0, U=2.0, nParticle=0.95, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=10)
    a, b = O.initialize(p), O.initialize(p)
    for ite in range(4):
        ca, _ = O.iteration(a, ite)
        cb, _ = P.iteration(b, ite)
        assert ca == cb
    assert _rel(b.Sigma, a.Sigma) < 1e-12
    for r in "dmst":
        assert _rel(b.F[r], a.F[r]) < 1e-12

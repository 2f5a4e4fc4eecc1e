"""Parity with the CPU oracle at the tile shapes of the largest workloads.

* 8x8 k, 9 form factors, 32 frequencies (Nz = 288): two full iterations
  phase by phase, so the BSE of the second iteration runs on vertices with
  every (l1, l2) block filled.
* 16x16 k, 9 form factors, 64 frequencies, t' = -0.2, n = 0.85 (Nz = 576,
  1440 slots, 61 GB of vertices): the oracle cannot hold the vertices, so
  three sampled slots get random Gamma_r and F_r, and the BSE of those slots,
  Phi(R) at one frequency and the crossing (F_r of those slots, from the
  device's Phi(R)) are compared with the oracle restricted to them
  (``bse_slot``, ``phir_at_w``, ``crossing_slot``).  This runs the Nz = 576
  BSE tiles and the 81-column crossing tiles.

Max-norm relative error per phase <= 1e-12.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import tups_oracle as O
import parity

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_nl9_workload_two_iterations(gpu_lib):
    """Iteration 0, then iteration 1 started on both sides from the oracle's
    state (Sigma, mu, F_r, Gamma_r), so every phase of both iterations is
    compared on identical inputs; the second iteration's BSE runs on
    vertices with every (l1, l2) block filled."""
    p = O.Params(beta=5.0, U=2.0, nParticle=1.0, Nx=8, Nf=32, neighbours=3, f_damping=0.5, ite_max=100)
    st = O.initialize(p)
    from tups_b200 import Solver
    sol = Solver(parity.to_solver_params(p))
    for ite in range(2):
        if ite > 0:
            sol.Sigma = st.Sigma
            sol.mu = st.mu
            for r in "dmst":
                sol.set_vertex(r, 0, st.F[r])
                sol.set_vertex(r, 1, st.G[r])
        errs: dict = {}
        parity.iteration_phases(sol, st, ite, errs)
        bad = {k: max(v) for k, v in errs.items() if k not in ("conv_rel_sig", "conv_flag_mismatch")
               and max(v) > TOL}
        assert not bad, (ite, bad)
    sol.close()


def test_16x16_sampled_slots(gpu_lib):
    from tups_b200 import Solver
    p = O.Params(beta=10.0, U=3.0, nParticle=0.85, Nx=16, Nf=64, neighbours=3, tprime=-0.2, f_damping=0.5,
                 ite_max=10)
    st = O.initialize(p, vertices=False)
    sol = Solver(parity.to_solver_params(p))
    assert (sol.Nz, sol.Nb, st.Nz, st.Nb) == (576, 1440, 576, 1440)
    nh, Nz = st.Nf // 2, st.Nz
    O.calc_Gkw_Grt(st, 0, False)
    sol.calc_Gkw_Grt(0, False)
    assert abs(sol.mu - st.mu) <= 1e-15
    assert parity.rel(sol.Gkw, st.Gkw) <= TOL

    slots = [0, 20 * nh + 10, st.Nb - 1]
    rng = np.random.default_rng(576)
    gam, fv, chi = {}, {}, {}
    for iq in slots:
        qx, qy, w = (int(v) for v in st.ibz[iq])
        chi[iq] = O.calc_chi(st, qx, qy, w)
        gph, gpp = sol.calc_chi(iq + 1)
        assert max(parity.rel(gph, chi[iq][0]), parity.rel(gpp, chi[iq][1])) <= TOL, iq
        for r in "dmst":
            g = 10.0 * (rng.standard_normal((Nz, Nz)) + 1j * rng.standard_normal((Nz, Nz)))
            f = 10.0 * (rng.standard_normal((Nz, Nz)) + 1j * rng.standard_normal((Nz, Nz)))
            gam[iq, r], fv[iq, r] = g, f
            sol.set_vertex_slots(r, 1, iq, g)
            sol.set_vertex_slots(r, 0, iq, f)

    # BSE on every slot; the sampled ones against the oracle
    sol.BSE(0)
    phi = {}
    for iq in slots:
        for r in "dmst":
            phi[iq, r] = sol.vertex_slots(r, 1, iq)[:, :, 0]
            ref = O.bse_slot(st, r, gam[iq, r], fv[iq, r], chi[iq][0] if r in "dm" else chi[iq][1])
            assert parity.rel(phi[iq, r], ref) <= TOL, ("BSE", iq, r, parity.rel(phi[iq, r], ref))

    # Phi(R) at the bosonic frequency of the middle slot, from Phi of all 45 momenta
    O.calculate_expSqR(st)
    O.calculate_expqSR(st)
    sol.calculate_expSqR()
    sol.calculate_expqSR()
    sol.calc_PhiR(0)
    w0 = int(st.ibz[slots[1], 2])
    PhiR = {}
    for r in "dmst":
        PhiR[r] = sol.PhiR(r)
        cols = [sol.vertex_slots(r, 1, Q * nh + w0 - 1)[:, :, 0].reshape(-1, order="F") for Q in range(st.NIBZ)]
        ref = O.phir_at_w(st, np.stack(cols, axis=1))
        assert parity.rel(PhiR[r][:, w0 - 1, :], ref) <= TOL, ("PhiR", r)

    # crossing: F_r of the sampled slots from the device's Phi and Phi(R)
    O.calc_M(st)
    for f in (sol.calc_M_phbar_to_ph, sol.calc_M_pp_to_ph, sol.calc_M_ph_to_pp, sol.calc_M_phbar_to_pp):
        f()
    sol.calculate_PAE()
    for iq in slots:
        ref = O.crossing_slot(st, iq, {r: phi[iq, r] for r in "dmst"}, PhiR)
        for r in "dmst":
            got = sol.vertex_slots(r, 0, iq)[:, :, 0]
            assert parity.rel(got, ref[r]) <= TOL, ("PAE", iq, r, parity.rel(got, ref[r]))
    sol.close()

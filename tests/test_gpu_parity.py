"""Parity of the CUDA library with the CPU oracle (run on a B200).

Per phase: max-norm relative error <= 1e-12 (FP64 paths; the only
differences are summation orders).  End to end over several iterations:
self-energy and vertices <= 1e-10 relative.  Integer tables: equal.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import tups_oracle as O
import parity

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
PHASE_TOL = 1e-12
E2E_TOL = 1e-10


def _check(errs):
    bad = {k: max(v) for k, v in errs.items() if k not in ("conv_rel_sig", "conv_flag_mismatch")
           and max(v) > PHASE_TOL}
    assert not bad, bad
    assert "conv_flag_mismatch" not in errs
    assert max(errs["conv_rel_sig"]) < 1e-9


@pytest.mark.parametrize("case", [
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=16, neighbours=1),   # 4x4, 1 form factor
    dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2),    # 5 form factors, off half filling
    dict(beta=3.0, U=1.5, nParticle=0.95, Nx=8, Nf=8, neighbours=3, tprime=-0.2),  # 9 form factors, t'
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=10, neighbours=2, f_range=1),    # enlarged SDE box
    dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, Ngrain=3),      # coarse graining
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=8, neighbours=2, use_U2=False),  # no U^2 term
    dict(beta=10.0, U=3.0, nParticle=0.85, Nx=16, Nf=8, neighbours=3, tprime=-0.2),  # 16x16 k, 9 FF
    dict(beta=3.0, U=2.0, nParticle=0.9, Nx=4, Nf=64, neighbours=1),  # Nz = 64: two BSE tiles per dimension
], ids=["nl1", "nl5_n09", "nl9_tprime", "frange1", "ngrain3", "noU2", "nx16_nl9", "nz64"])
def test_phases_side_by_side(gpu_lib, case):
    p = O.Params(f_damping=0.5, ite_max=10, **case)
    errs, st, sol = parity.run_side_by_side(p, 2 if p.Nx >= 16 else 3)
    _check(errs)
    sol.close()


@pytest.mark.parametrize("case", [
    dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2),
    dict(beta=3.0, U=1.5, nParticle=0.95, Nx=8, Nf=8, neighbours=3, tprime=-0.2),
], ids=["nl5", "nl9_tprime"])
def test_four_product_crossing_side_by_side(gpu_lib, case):
    """The crossing GEMM with four real products per complex one meets the
    same per-phase bound as the three-product (Gauss) default."""
    p = O.Params(f_damping=0.5, ite_max=10, **case)
    errs, st, sol = parity.run_side_by_side(p, 3, crossing_products=4)
    _check(errs)
    sol.close()


def test_tables_bit_exact(gpu_lib):
    from tups_b200 import Solver
    p = O.Params(Nx=8, Nf=8, neighbours=3)
    st = O.initialize(p)
    sol = Solver(parity.to_solver_params(p))
    t = sol.tables()
    for k in ("signs", "reps", "lsym", "ibz"):
        assert np.array_equal(t[k], getattr(st, k)), k
    for k in ("FF", "FF_inv", "lfac"):
        assert np.array_equal(t[k], getattr(st, k)), k
    sol.close()


@pytest.mark.parametrize("name", ["pa_4x4_nl1", "pa_4x4_nl5"])
def test_golden_fixtures(gpu_lib, name):
    """The committed oracle fixtures, reproduced by the CUDA path."""
    from tups_b200 import Solver, read_prms
    g = np.load(GOLD / f"golden_{name}.npz")
    sol = Solver(read_prms(str(GOLD / f"prms_{name}")))
    sol.calc_Gkw_Grt(0, False)
    assert abs(sol.mu - float(g["ite0_mu"])) <= 1e-15
    assert parity.rel(sol.Gkw, g["ite0_Gkw"]) < PHASE_TOL
    assert parity.rel(sol.Grt, g["ite0_Grt"]) < PHASE_TOL
    ph, pp = sol.calc_chi(sol.Nb)
    assert parity.rel(ph, g["ite0_chi_ph_last"]) < PHASE_TOL
    assert parity.rel(pp, g["ite0_chi_pp_last"]) < PHASE_TOL
    sol.BSE(0)
    sol.calculate_expSqR()
    sol.calculate_expqSR()
    sol.calc_PhiR(0)
    for f in (sol.calc_M_phbar_to_ph, sol.calc_M_pp_to_ph, sol.calc_M_ph_to_pp, sol.calc_M_phbar_to_pp):
        f()
    sol.calculate_PAE()
    for r in "dmst":
        if f"ite0_Phi_{r}" in g:
            assert parity.rel(sol.G(r), g[f"ite0_Phi_{r}"]) < PHASE_TOL
            assert parity.rel(sol.F(r), g[f"ite0_F_{r}"]) < PHASE_TOL
            assert parity.rel(sol.PhiR(r), g[f"ite0_PhiR_{r}"]) < PHASE_TOL
        else:
            assert parity.rel(sol.G(r)[:, :, 0], g[f"ite0_Phi_{r}_q0"]) < PHASE_TOL
            assert parity.rel(sol.F(r)[:, :, -1], g[f"ite0_F_{r}_qlast"]) < PHASE_TOL
    sol.calc_SDE(0)
    assert parity.rel(sol.Sigma, g["ite0_Sigma"]) < PHASE_TOL
    sol.close()
    # the whole loop through the C-ABI loop driver
    sol = Solver(read_prms(str(GOLD / f"prms_{name}")))
    traj = g["traj_Sigma"]
    for ite in range(len(traj)):
        sol.iteration(ite)
        assert parity.rel(sol.Sigma, traj[ite]) < E2E_TOL, ite
        assert abs(sol.mu - float(g["traj_mu"][ite])) <= 1e-14
    for r in "dmst":
        assert parity.rel(sol.F(r)[:, :, 0], g[f"final_F_{r}_q0"]) < E2E_TOL
    sol.close()


def test_bench_workload_one_iteration(gpu_lib):
    """8x8 k, 5 form factors, 32 frequencies (the bench workload): the first
    iteration phase by phase (the oracle takes ~15 s for it)."""
    p = O.Params(beta=5.0, U=2.0, nParticle=1.0, Nx=8, Nf=32, neighbours=2, f_damping=0.5, ite_max=100)
    errs, st, sol = parity.run_side_by_side(p, 1)
    _check(errs)
    sol.close()


def test_end_to_end_ten_iterations(gpu_lib):
    """10 iterations of the 4x4 loop through tups_iteration: Sigma and every
    channel vertex within 1e-10 of the oracle."""
    from tups_b200 import Solver
    p = O.Params(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=16, neighbours=1, f_damping=0.5, ite_max=10)
    st = O.initialize(p)
    sol = Solver(parity.to_solver_params(p))
    for ite in range(10):
        conv_o, info_o = O.iteration(st, ite)
        info_g = sol.iteration(ite)
        assert info_g["converged"] == conv_o
    assert parity.rel(sol.Sigma, st.Sigma) < E2E_TOL
    for r in "dmst":
        assert parity.rel(sol.F(r), st.F[r]) < E2E_TOL
        assert parity.rel(sol.G(r), st.G[r]) < E2E_TOL
    sol.close()


def test_execute_loop_converges_like_oracle(gpu_lib):
    """execute_loop to the reference's convergence test at a strongly damped,
    small, quickly converging point: same iteration count as the oracle."""
    from tups_b200 import Solver
    p = O.Params(beta=1.0, U=0.5, nParticle=1.0, Nx=4, Nf=8, neighbours=1, f_damping=0.5, ite_max=80)
    st = O.initialize(p)
    conv_o, n_o, _ = O.execute_loop(st)
    sol = Solver(parity.to_solver_params(p))
    n_g, conv_g = sol.execute_loop()
    assert (n_g, conv_g) == (n_o, conv_o)
    assert parity.rel(sol.Sigma, st.Sigma) < E2E_TOL
    sol.close()


@pytest.mark.parametrize("case", [
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=16, neighbours=1),
    dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2),
    dict(beta=3.0, U=1.5, nParticle=0.95, Nx=8, Nf=8, neighbours=3, tprime=-0.2),
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=10, neighbours=2, f_range=1),
    dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, Ngrain=3),
], ids=["nl1", "nl5_n09", "nl9_tprime", "frange1", "ngrain3"])
def test_readout_side_by_side(gpu_lib, case):
    """Exact chi0 bubble (4 projections), susceptibilities of all channels,
    IBZ and whole BZ (SRC/parquet_chi.f90:216-430, parquet_sus.f90,
    parquet_plot.f90:14-58)."""
    p = O.Params(f_damping=0.5, ite_max=10, **case)
    errs = parity.readout_side_by_side(p, 2)
    assert errs.pop("mu") == 0.0
    bad = {k: v for k, v in errs.items() if v > PHASE_TOL}
    assert not bad, bad

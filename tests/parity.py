"""Side-by-side driver: the CUDA library vs the CPU oracle, phase by phase.

Used by the gpu-marked parity tests and by ``__graft_entry__.smoke()``.
Both sides start from the same parameters and advance through the phases
of one parquet iteration (SRC/loop.f90:51-222); after each phase the
relevant arrays are compared with a max-norm relative error
max|a - b| / max|b|.
"""
from __future__ import annotations

import numpy as np

from oracle import tups_oracle as O

CH = "dmst"


def rel(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if b.size else 0.0
    return num / den if den > 0 else num


def to_solver_params(p: O.Params):
    from tups_b200 import Params
    kw = {k: getattr(p, k) for k in Params.__dataclass_fields__}
    return Params(**kw)


def iteration_phases(sol, st: O.State, ite: int, errs: dict) -> dict:
    """Run one iteration on both sides and record per-phase errors into errs."""
    p = st.p
    # Green's function
    O.calc_Gkw_Grt(st, ite, False)
    sol.calc_Gkw_Grt(ite, False)
    errs.setdefault("mu", []).append(abs(sol.mu - st.mu))
    errs.setdefault("Gkw", []).append(rel(sol.Gkw, st.Gkw))
    errs.setdefault("Grt", []).append(rel(sol.Grt, st.Grt))
    # chi for a few slots
    for iq in sorted({0, st.Nb // 2, st.Nb - 1}):
        qx, qy, w = (int(v) for v in st.ibz[iq])
        oph, opp = O.calc_chi(st, qx, qy, w)
        gph, gpp = sol.calc_chi(iq + 1)
        errs.setdefault("chi", []).append(max(rel(gph, oph), rel(gpp, opp)))
    # BSE
    O.bse(st, ite)
    sol.BSE(ite)
    errs.setdefault("BSE", []).append(max(rel(sol.G(r), st.G[r]) for r in CH))
    if ite == 0:
        O.calculate_expSqR(st)
        O.calculate_expqSR(st)
        sol.calculate_expSqR()
        sol.calculate_expqSR()
        errs.setdefault("expSqR", []).append(rel(sol.expSqR(), st.expSqR))
        errs.setdefault("expqSR", []).append(rel(sol.expqSR(), st.expqSR))
    O.calc_PhiR(st)
    sol.calc_PhiR(ite)
    errs.setdefault("PhiR", []).append(max(rel(sol.PhiR(r), st.PhiR[r]) for r in CH))
    if ite == 0:
        O.calc_M(st)
        sol.calc_M_phbar_to_ph()
        sol.calc_M_pp_to_ph()
        sol.calc_M_ph_to_pp()
        sol.calc_M_phbar_to_pp()
        names = ["phbar_to_ph", "pp_to_ph", "ph_to_pp", "phbar_to_pp"]
        errs.setdefault("M", []).append(max(rel(sol.M(i), O.M_full(st, n)) for i, n in enumerate(names)))
    O.calculate_PAE(st)
    sol.calculate_PAE()
    errs.setdefault("PAE", []).append(max(rel(sol.F(r), st.F[r]) for r in CH))
    if not p.oneshot or ite == p.ite_max - 1:
        st.arrays["SigmaOld"] = st.Sigma.copy()
        O.calc_SDE(st)
        sol.calc_SDE(ite)
        aux = sol.sde_aux()
        cph, cpp = st.chi_aux
        lc, pc, qc = st.LChi
        errs.setdefault("chi_aux", []).append(max(rel(aux["chi_aux_ph"], cph), rel(aux["chi_aux_pp"], cpp)))
        # LChi enters Sigma only as LChi + PhChi, and in the PA with the U^2
        # term it is (L_d - L_m - 2U) chi = 0 up to rounding: scale its error
        # by |PhChi| instead of by its own (noise-level) size
        lchi_err = float(np.max(np.abs(aux["LChi"] - lc))) / max(float(np.max(np.abs(pc))), 1e-300)
        errs.setdefault("LChi", []).append(max(lchi_err, rel(aux["PhChi"], pc), rel(aux["PPChi"], qc)))
        errs.setdefault("Sigma", []).append(rel(sol.Sigma, st.Sigma))
    conv_o, info_o = O.conv(st)
    info_g = sol.conv()
    errs.setdefault("conv_rel_sig", []).append(
        abs(info_g["rel_sig_max"] - info_o["rel_sig_max"]) / max(info_o["rel_sig_max"], 1e-300))
    if conv_o != info_g["converged"]:
        errs.setdefault("conv_flag_mismatch", []).append(ite)
    if ite % 5 == 0 or ite == p.ite_max - 1 or conv_o:
        O.output_block_mu(st)
        sol.output_block()
    for r in CH:
        st.G[r] = st.F[r] - st.G[r]
    sol.vertex_update()
    errs.setdefault("update", []).append(max(rel(sol.G(r), st.G[r]) for r in CH))
    return info_o


def readout_side_by_side(p: O.Params, full_iterations: int = 2, device: int = 0) -> dict:
    """Run `full_iterations` iterations on both sides, then the next one up
    to the convergence check, then the readout; returns the readout errors."""
    from tups_b200 import Solver
    st = O.initialize(p)
    sol = Solver(to_solver_params(p), device=device)
    for ite in range(full_iterations):
        O.iteration(st, ite)
        sol.iteration(ite)
    ite = full_iterations
    O.calc_Gkw_Grt(st, ite, False)
    sol.calc_Gkw_Grt(ite, False)
    O.bse(st, ite)
    sol.BSE(ite)
    O.calc_PhiR(st)
    sol.calc_PhiR(ite)
    O.calculate_PAE(st)
    sol.calculate_PAE()
    st.arrays["SigmaOld"] = st.Sigma.copy()
    O.calc_SDE(st)
    sol.calc_SDE(ite)
    O.conv(st)
    sol.conv()
    ro = O.readout(st, ite)
    sol.readout(ite)
    errs = {"mu": abs(sol.mu - st.mu)}
    for bz in (False, True):
        c = sol.chi0(bz)
        sfx = "_BZ" if bz else ""
        errs["chi0_ph" + sfx] = rel(c["chi0_ph"], ro["chi0_ph_BZ" if bz else "chi0_ph"])
        errs["chi0_pp" + sfx] = rel(c["chi0_pp"], ro["chi0_pp_BZ" if bz else "chi0_pp"])
        errs["chi0_ph_FF" + sfx] = rel(c["chi0_ph_FF"], ro["chi0_ph_BZ_FF" if bz else "chi0_ph_FF"])
        errs["chi0_pp_FF" + sfx] = rel(c["chi0_pp_FF"], ro["chi0_pp_BZ_FF" if bz else "chi0_pp_FF"])
        for r in CH:
            errs[f"sus_{r}" + sfx] = rel(sol.sus(r, bz), ro[f"sus_{r}" if bz else f"sus_{r}_IBZ"])
    sol.close()
    return errs


def run_side_by_side(p: O.Params, iterations: int, device: int = 0, crossing_products: int = 3):
    """Returns (errors per phase, oracle state, solver)."""
    from tups_b200 import Solver
    st = O.initialize(p)
    sol = Solver(to_solver_params(p), device=device)
    sol.set_crossing_products(crossing_products)
    errs: dict = {}
    errs["init_F"] = [max(rel(sol.F(r), st.F[r]) for r in CH)]
    for ite in range(iterations):
        iteration_phases(sol, st, ite, errs)
    return errs, st, sol

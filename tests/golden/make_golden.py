"""Regenerate the golden fixtures in this directory from the CPU oracle.

    python tests/golden/make_golden.py

Fixtures: per-phase arrays of iteration 0 and the self-energy trajectory for
the 4x4 / 1 form factor / 16 frequency loop (``golden_pa_4x4_nl1.npz``) and a
4x4 / 5 form factor / 8 frequency loop at n = 0.9 (``golden_pa_4x4_nl5.npz``),
plus prms files in the reference's 21-record format.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import tups_oracle as O  # noqa: E402

CASES = {
    "pa_4x4_nl1": O.Params(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=16, neighbours=1, f_damping=0.5, ite_max=10),
    "pa_4x4_nl5": O.Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=4),
}

PRMS_TEMPLATE = """  {beta:.1f}d0                                                !beta
  {U:.1f}d0                                                !U
  {n:.2f}d0                                               !nParticle
  {Nx}                                                    !Nx
  {Nf}                                                   !Nf
  {nb}                                                    !neighbours
  .false.                                               !picklist - decide wether to read picklist
  "inidata/none"                                        !picklist-filename
  1                                                     !Ngrain
  0                                                     !f_range
  {f:.1f}d0                                                !f_damping
  {ite}                                                   !maximum number of iterations
  .false.                                               !DGA
  "inidata/none"                                        !file for Lambdas
  .false.                                               !use selfenergy from DMFT
  "inidata/none"                                        !filename for DMFT Sigma
  .true.                                                !use U2 correction in selfenergy
  .false.                                               !save whole F's
  .false.                                               !oneshot calculation
  .false.                                               !old PAE implementation
  .false.                                               !old SDE implementation
"""


def write_prms(name: str, p: O.Params) -> None:
    (HERE / f"prms_{name}").write_text(PRMS_TEMPLATE.format(
        beta=p.beta, U=p.U, n=p.nParticle, Nx=p.Nx, Nf=p.Nf, nb=p.neighbours, f=p.f_damping, ite=p.ite_max))


def make(name: str, p: O.Params) -> None:
    st = O.initialize(p)
    out = {"FF": st.FF, "FF_inv": st.FF_inv, "signs": st.signs, "reps": st.reps, "lsym": st.lsym,
           "lfac": st.lfac, "ibz": st.ibz}
    small = st.Nz * st.Nz * st.Nb <= 20000
    # iteration 0, phase by phase
    O.calc_Gkw_Grt(st, 0, False)
    out["ite0_mu"] = np.array(st.mu)
    out["ite0_Gkw"] = st.Gkw
    out["ite0_Grt"] = st.Grt
    qx, qy, w = (int(v) for v in st.ibz[st.Nb - 1])
    out["ite0_chi_ph_last"], out["ite0_chi_pp_last"] = O.calc_chi(st, qx, qy, w)
    O.bse(st)
    O.calculate_expSqR(st)
    O.calculate_expqSR(st)
    O.calc_PhiR(st)
    O.calc_M(st)
    O.calculate_PAE(st)
    for r in "dmst":
        if small:
            out[f"ite0_Phi_{r}"] = st.G[r]
            out[f"ite0_F_{r}"] = st.F[r]
            out[f"ite0_PhiR_{r}"] = st.PhiR[r]
        else:
            out[f"ite0_Phi_{r}_q0"] = st.G[r][:, :, 0]
            out[f"ite0_F_{r}_qlast"] = st.F[r][:, :, st.Nb - 1]
    st.arrays["SigmaOld"] = st.Sigma.copy()
    O.calc_SDE(st)
    out["ite0_Sigma"] = st.Sigma
    # full-loop self-energy trajectory
    st = O.initialize(p)
    sig, mus = [], []
    for ite in range(p.ite_max):
        conv, info = O.iteration(st, ite)
        sig.append(st.Sigma.copy())
        mus.append(st.mu)
    out["traj_Sigma"] = np.array(sig)
    out["traj_mu"] = np.array(mus)
    for r in "dmst":
        out[f"final_F_{r}_q0"] = st.F[r][:, :, 0]
    np.savez_compressed(HERE / f"golden_{name}.npz", **out)
    write_prms(name, p)


if __name__ == "__main__":
    for k, v in CASES.items():
        make(k, v)
        print("wrote", k)

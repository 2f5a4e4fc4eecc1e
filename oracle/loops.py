"""Loop-by-loop transliterations of the index-heavy reference routines.

TEST INFRASTRUCTURE ONLY.  These follow the Fortran loop nests statement by
statement (1-based indices kept) and run only on tiny sizes; the tests use
them to check the vectorised oracle in ``tups_oracle``.
"""
from __future__ import annotations

import numpy as np

from .tups_oracle import NS, State, list_symmetries, symmetry_operation


def pick_nu(x: int, Nf: int) -> int:
    """``pickNu`` (parquet_EQContribs.f90:25-38); x in 1..5*Nf."""
    if x <= 2 * Nf:
        return 1
    if 2 * Nf < x < 3 * Nf:
        return x - 2 * Nf
    return Nf


def crossing_call_loops(st: State, call: str, PhiR: np.ndarray, w2: int, fac1: float,
                        fac2: float, F1: np.ndarray, F2: np.ndarray) -> None:
    """One ``calc_*`` call of parquet_EQContribs.f90:44-524, loop for loop.

    ``F1``/``F2`` are the two targets (d,m for *_to_ph, s,t for *_to_pp),
    updated in place.  ``PhiR`` is (Nz*Nz, Nf/2, NR)."""
    Nf, Nl, Nz, NR, Nx = st.Nf, st.Nl, st.Nz, st.NR, st.Nx
    W = PhiR.reshape(Nz, Nz, Nf // 2, NR, order="F")
    mF = lambda nu: -nu + Nf + 1
    FpB = lambda nu, om: nu + om - 1
    BpBmF = lambda o1, o2, nu: o1 + o2 - 1 + (-nu + Nf + 1) - 1
    FmB = lambda nu, om: nu - om + 1
    BmBmF = lambda o1, o2, nu: (o1 - 1) - (nu + o2 - 1) + Nf + 1
    sg = st.signs
    base = call.replace("_TR", "")
    M = st.M_ibz[base]
    for iq in range(1, st.Nb + 1):
        Om = int(st.ibz[iq - 1, 2])
        mq = st.M_q_of_slot[iq - 1]
        for R in range(1, NR + 1):
            for l4 in range(1, Nl + 1):
                for l3 in range(1, Nl + 1):
                    for l2 in range(1, Nl + 1):
                        for l1 in range(1, Nl + 1):
                            m = M[l1 - 1, l2 - 1, l3 - 1, l4 - 1, mq, R - 1]
                            for nu1 in range(1, Nf + 1):
                                if call == "phbar_to_ph":
                                    if FpB(nu1, w2) > Nf:
                                        continue
                                    t = FpB(nu1, w2)
                                    x = W[(l3 - 1) * Nf + nu1 - 1,
                                          (l4 - 1) * Nf + pick_nu(FpB(nu1, Om) + 2 * Nf, Nf) - 1, w2 - 1, R - 1]
                                elif call == "phbar_to_ph_TR":
                                    if FmB(nu1, w2) > Nf or FmB(nu1, w2) < 1:
                                        continue
                                    t = FmB(nu1, w2)
                                    x = sg[l3 - 1] * sg[l4 - 1] * np.conj(
                                        W[(l3 - 1) * Nf + mF(nu1) - 1,
                                          (l4 - 1) * Nf + pick_nu(mF(FpB(nu1, Om)) + 2 * Nf, Nf) - 1, w2 - 1, R - 1])
                                elif call == "pp_to_ph":
                                    v = BmBmF(w2, Om, nu1)
                                    if v > Nf or v < 1:
                                        continue
                                    t = v
                                    x = W[(l3 - 1) * Nf + nu1 - 1, (l4 - 1) * Nf + v - 1, w2 - 1, R - 1]
                                elif call == "pp_to_ph_TR":
                                    v = FpB(nu1, Om + w2 - 1)
                                    if v > Nf or v < 1:
                                        continue
                                    t = mF(v)
                                    x = sg[l3 - 1] * sg[l4 - 1] * np.conj(
                                        W[(l3 - 1) * Nf + mF(nu1) - 1, (l4 - 1) * Nf + v - 1, w2 - 1, R - 1])
                                elif call == "ph_to_pp":
                                    v = BmBmF(Om, w2, nu1)
                                    if v > Nf or v < 1:
                                        continue
                                    t = v
                                    x = W[(l3 - 1) * Nf + nu1 - 1, (l4 - 1) * Nf + v - 1, w2 - 1, R - 1]
                                elif call == "ph_to_pp_TR":
                                    v = BpBmF(Om, w2, nu1)
                                    if v > Nf or v < 1:
                                        continue
                                    t = v
                                    x = sg[l3 - 1] * sg[l4 - 1] * np.conj(
                                        W[(l3 - 1) * Nf + mF(nu1) - 1,
                                          (l4 - 1) * Nf + FmB(nu1, Om + w2 - 1) - 1, w2 - 1, R - 1])
                                elif call == "phbar_to_pp":
                                    if FpB(w2, nu1) > Nf:
                                        continue
                                    t = FpB(nu1, w2)
                                    x = W[(l3 - 1) * Nf + nu1 - 1,
                                          (l4 - 1) * Nf + pick_nu(BmBmF(Om, w2, nu1) + 2 * Nf, Nf) - 1, w2 - 1, R - 1]
                                elif call == "phbar_to_pp_TR":
                                    if FmB(nu1, w2) > Nf or FmB(nu1, w2) < 1:
                                        continue
                                    t = FmB(nu1, w2)
                                    x = sg[l3 - 1] * sg[l4 - 1] * np.conj(
                                        W[(l3 - 1) * Nf + mF(nu1) - 1,
                                          (l4 - 1) * Nf + pick_nu(FmB(nu1, Om + w2 - 1) + 2 * Nf, Nf) - 1, w2 - 1, R - 1])
                                else:
                                    raise KeyError(call)
                                i = (l1 - 1) * Nf + nu1 - 1
                                j = (l2 - 1) * Nf + t - 1
                                F1[i, j, iq - 1] += x * m * fac1 * 1.0 / Nx
                                F2[i, j, iq - 1] += x * m * fac2 * 1.0 / Nx


def sde_sigma_loops(st: State, LChi, PhChi, PPChi) -> np.ndarray:
    """Sigma_V accumulation of parquet_SDE.f90:116-221, loop for loop."""
    p = st.p
    Nx, Ny, Nf, Nl = st.Nx, st.Ny, st.Nf, st.Nl
    Nred = st.Nred
    out = np.zeros(2 * Nred, dtype=np.complex128)

    def get_green(ix, iy, iw):
        fr = 1j * (np.pi / p.beta * (2.0 * (iw - Nf // 2 - 1) + 1.0))
        if iw < 1 or iw > Nf:
            return 1.0 / (fr - st.Ek[ix - 1, iy - 1] + st.mu - st.Sigma_H[ix - 1, iy - 1])
        return st.Gkw[((ix - 1) * Ny + iy - 1) * Nf + iw - 1]

    for k0 in range(1, Nf + 1):
        for kx in range(1, st.Nx_IBZ + 1):
            for ky in range(1, kx + 1):
                mkx, mky, mkw = (-(kx - 1) + Nx) % Nx + 1, (-(ky - 1) + Ny) % Ny + 1, -k0 + Nf + 1
                sig = 0j
                for iq in range(1, st.Nb + 1):
                    qx, qy, w = (int(v) for v in st.ibz[iq - 1])
                    sl = list_symmetries(qx, qy, st.Nx_IBZ)
                    for s in range(1, NS + 1):
                        if not sl[s - 1]:
                            continue
                        sx, sy = symmetry_operation(s, qx, qy, Nx)
                        kq = ((kx - 1 + sx - 1) % Nx + 1, (ky - 1 + sy - 1) % Ny + 1, k0 + w - 1)
                        gkq = get_green(*kq)
                        qmk = ((mkx - 1 + sx - 1) % Nx + 1, (mky - 1 + sy - 1) % Ny + 1, mkw + w - 1)
                        gqmk = get_green(*qmk)
                        kmq = ((-(qmk[0] - 1) + Nx) % Nx + 1, (-(qmk[1] - 1) + Ny) % Ny + 1, -qmk[2] + Nf + 1)
                        gkmq = get_green(*kmq)
                        for l3 in range(1, Nl + 1):
                            i3 = (l3 - 1) * Nf + k0 - 1
                            ff = st.FF_inv[s - 1, kx - 1, ky - 1, l3 - 1]
                            sig += gkq * ff * LChi[i3, iq - 1]
                            sig += gkq * ff * PhChi[i3, iq - 1]
                            sig += gqmk * ff * PPChi[i3, iq - 1]
                            if w == 1:
                                continue
                            i3m = (l3 - 1) * Nf + (-k0 + Nf + 1) - 1
                            sgn = st.signs[l3 - 1]
                            sig += gkmq * ff * sgn * np.conj(LChi[i3m, iq - 1])
                            sig += gkmq * ff * sgn * np.conj(PhChi[i3m, iq - 1])
                            sig += np.conj(gkq) * ff * sgn * np.conj(PPChi[i3m, iq - 1])
                idxk = (((kx - 1) * kx) // 2 + ky - 1) * Nf + k0
                out[idxk - 1] -= p.U / p.beta / p.beta / st.Nc / st.Nc / 2.0 * sig
    return out


def symop_arr_loops(st: State, tosym: np.ndarray, s: int, w_outer: int) -> np.ndarray:
    """``symop_arr`` (parquet_PhiR.f90:311-356) on (Nz*Nz, Nf/2, NIBZ)."""
    Nl, Nf, Nz = st.Nl, st.Nf, st.Nz
    ret = np.zeros_like(tosym)
    for iq in range(st.NIBZ):
        for L2 in range(1, Nl + 1):
            for L1 in range(1, Nl + 1):
                L2s, f2 = int(st.lsym[s - 1, L2 - 1]), st.lfac[s - 1, L2 - 1]
                L1s, f1 = int(st.lsym[s - 1, L1 - 1]), st.lfac[s - 1, L1 - 1]
                for n2 in range(1, Nf + 1):
                    for n1 in range(1, Nf + 1):
                        isym = ((L2s - 1) * Nf + n2 - 1) * Nz + (L1s - 1) * Nf + n1
                        inos = ((L2 - 1) * Nf + n2 - 1) * Nz + (L1 - 1) * Nf + n1
                        ret[inos - 1, w_outer - 1, iq] = f1 * f2 * tosym[isym - 1, w_outer - 1, iq]
    return ret

"""Compiled port of the oracle's crossing and Phi(R) phases (TEST AND
BASELINE INFRASTRUCTURE ONLY: used by ``bench.py``'s CPU baseline and by the
tests that check it against the numpy oracle).

``iteration(st, ite)`` is ``oracle.tups_oracle.iteration`` (loop.f90:51-244)
with ``calc_PhiR`` and ``calculate_PAE`` replaced by the C++/OpenMP loop
nests of ``tups_port.cpp`` (the reference's own form of those phases is
compiled Fortran loops, SRC/parquet_PhiR.f90:196-258 and
SRC/parquet_EQContribs.f90:44-524); the BSE's four ZGEMMs per (q, r) stay
on the host BLAS that numpy links (OpenBLAS), as the reference calls MKL's
ZGEMM (SRC/parquet_BSE.f90:72-124).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from .. import tups_oracle as O

HERE = Path(__file__).resolve().parent
SRC = HERE / "tups_port.cpp"
LIB = HERE / "_build" / "libtups_port.so"
CXXFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17"]

_lib = None


def build(force: bool = False) -> Path:
    """Compile the port with g++ (OpenMP) into oracle/port/_build."""
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", *CXXFLAGS, str(SRC), "-o", str(tmp)], check=True)
    os.replace(tmp, LIB)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(os.fspath(LIB))
        lib.port_threads.argtypes = [C.c_int]
        lib.port_threads.restype = C.c_int
        lib.port_crossing.restype = C.c_int
        lib.port_phir.restype = C.c_int
        _lib = lib
    return _lib


def threads(n: int = 0) -> int:
    """Set (n > 0) and return the OpenMP thread count of the port."""
    return int(load().port_threads(int(n)))


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _parr(arrs) -> C.Array:
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def calc_PhiR(st: O.State) -> None:
    """``calc_PhiR`` (parquet_PhiR.f90:35-258) through ``port_phir``."""
    Nz, Nf, NIBZ, NR = st.Nz, st.Nf, st.NIBZ, st.NR
    cache = st.arrays.setdefault("_port_perm", {})
    if "src" not in cache:
        perms = [O.symop_perm(st, s) for s in range(1, O.NS + 1)]
        cache["src"] = np.ascontiguousarray(np.stack([p[0] for p in perms]), dtype=np.int64)
        cache["fac"] = np.ascontiguousarray(np.stack([p[1] for p in perms]), dtype=np.float64)
    exps = np.asfortranarray(st.expSqR, dtype=np.complex128)
    phiq = [np.asfortranarray(st.G[r]) for r in "dmst"]
    out = {r: np.zeros((Nz * Nz, Nf // 2, NR), dtype=np.complex128, order="F") for r in "dmst"}
    rc = load().port_phir(Nz, Nf, NIBZ, NR, st.Nx, _parr(phiq), _p(cache["src"]), _p(cache["fac"]), _p(exps),
                          _parr([out[r] for r in "dmst"]))
    if rc:
        raise RuntimeError(f"port_phir failed with {rc}")
    st.arrays["PhiR"] = out


def calculate_PAE(st: O.State) -> None:
    """``calculate_PAE`` (parquet_EQOuter.f90:16-118) through ``port_crossing``."""
    Nf = st.Nf
    F = {r: np.asfortranarray(st.G[r].copy(order="F")) for r in "dmst"}
    aux = abs(1.0 / st.FF[0, 0, 0] * 1.0 / st.FF[0, 0, 0])
    q0 = st.ibz[:, 2] - 1
    for r in "dmst":
        F[r][:Nf, :Nf, :] += st.L[r][:, :, q0] * aux
    names = ("phbar_to_ph", "pp_to_ph", "ph_to_pp", "phbar_to_pp")
    Ms = [np.asfortranarray(st.M_ibz[n]) for n in names]
    PhiR = [np.asfortranarray(st.PhiR[r]) for r in "dmst"]
    ibz = np.ascontiguousarray(st.ibz, dtype=np.int64)
    signs = np.ascontiguousarray(st.signs, dtype=np.int64)
    rc = load().port_crossing(st.Nz, Nf, st.Nl, st.Nb, st.NR, st.NIBZ, st.Nx, _p(ibz), _p(signs), _parr(Ms),
                              _parr(PhiR), _parr([F[r] for r in "dmst"]))
    if rc:
        raise RuntimeError(f"port_crossing failed with {rc}")
    st.arrays["F"] = F


def iteration(st: O.State, ite: int) -> tuple[bool, dict]:
    """One pass of ``execute_loop`` (loop.f90:51-244), the oracle's phases
    with the crossing and Phi(R) compiled."""
    p = st.p
    steps = O.calc_Gkw_Grt(st, ite, False)
    O.bse(st, ite)
    if ite == 0:
        O.calculate_expSqR(st)
        O.calculate_expqSR(st)
    calc_PhiR(st)
    if ite == 0:
        O.calc_M(st)
    calculate_PAE(st)
    if not p.oneshot or ite == p.ite_max - 1:
        st.arrays["SigmaOld"] = st.Sigma.copy()
        O.calc_SDE(st)
    converged, info = O.conv(st)
    info["bisection_steps"] = steps
    info["mu"] = st.mu
    if ite % 5 == 0 or ite == p.ite_max - 1 or converged:
        O.output_block_mu(st)
    for r in "dmst":
        st.G[r] = st.F[r] - st.G[r]
    return converged, info

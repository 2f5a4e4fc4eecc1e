"""The reference's program output (SRC/parquet_plot.f90:68-276,
SRC/preprocessing.f90:66-88,161): its file label, and the datasets
``params/``, ``Sigma/``, ``Chi/`` and ``F/`` with the reference's names,
shapes, sign conventions and iteration numbers.

No HDF5 library exists in this environment, so each file is an ``.npz``
archive whose keys are the HDF5 dataset paths and whose arrays are what an
HDF5 reader returns for the reference's datasets: the Fortran dimensions in
reverse (C) order, and complex values as the compound of two float64 fields
``r`` and ``i`` that the reference's HDF5 wrapper writes
(SRC/hdf5_wrapper.f90:285-287).  Copying each key into an HDF5 file gives
the reference's file.
"""
from __future__ import annotations

import os

import numpy as np

COMPLEX = np.dtype([("r", "<f8"), ("i", "<f8")])


def kind_label(p, Nl: int) -> str:
    """``kind_str`` (SRC/preprocessing.f90:66-88): I4.4 fields, beta as I2.2,
    U x 10 and n x 100 truncated as Fortran INT does."""
    f4 = lambda v: f"{int(v):04d}"
    s = (f"NxN{f4(p.Nx * p.Nx)}_Nl{f4(Nl)}_Nf{f4(p.Nf)}_U{f4(int(10 * p.U))}_B{int(p.beta):02d}"
         f"_Gr{f4(p.Ngrain)}_n{f4(int(p.nParticle * 100))}")
    if not p.DGA:
        s += "_pa"
    if p.use_U2:
        s += "_U2"
    if p.oneshot:
        s += "_one"
    s += "_old" if p.old else "_new"
    s += "_SDEold" if p.SDE_old else "_SDEnew"
    return s


def dataset(fortran_array) -> np.ndarray:
    """An array as an HDF5 reader returns the reference's dataset of it:
    dimensions reversed, complex values as the (r, i) compound."""
    a = np.asarray(fortran_array)
    t = a.T
    if np.iscomplexobj(a):
        out = np.empty(t.shape, dtype=COMPLEX)
        out["r"] = t.real
        out["i"] = t.imag
        return out
    return np.ascontiguousarray(t)


def as_fortran(ds: np.ndarray) -> np.ndarray:
    """Inverse of ``dataset``: the Fortran-shaped array."""
    a = ds["r"] + 1j * ds["i"] if ds.dtype == COMPLEX else ds
    return np.asarray(a).T


def _r(a, shape):
    return np.reshape(np.asarray(a), shape, order="F")


class Output:
    """``data/TUPS_<kind>.hdf5`` as ``<directory>/TUPS_<kind>.npz``:
    ``setup_hdf5`` at construction, ``write_sigma`` and ``write_chis`` at the
    output iterations, ``save`` to write the file."""

    def __init__(self, directory, p, Nl: int):
        self.p = p
        self.Nl = Nl
        self.path = os.path.join(str(directory), f"TUPS_{kind_label(p, Nl)}.npz")
        # setup_hdf5 (SRC/parquet_plot.f90:68-94)
        self.data = {"params/beta": np.float64(p.beta), "params/xU": np.float64(p.U),
                     "params/Nx": np.int32(p.Nx), "params/Nf": np.int32(p.Nf), "params/Nl": np.int32(Nl),
                     "params/DGA": np.int32(1 if p.DGA else 0), "params/Ngrain": np.int32(p.Ngrain),
                     "params/f_range": np.int32(p.f_range), "params/nParticle": np.float64(p.nParticle)}

    def write_sigma(self, ite: int, converged: bool, sigma) -> None:
        """``write_sigma`` (SRC/parquet_plot.f90:98-140): Sigma as (Nf, Nx*Ny)."""
        p = self.p
        s = dataset(_r(sigma, (p.Nf, p.Nx * p.Nx)))
        self.data[f"Sigma/sig_{ite:05d}"] = s
        if ite == p.ite_max or converged:
            self.data["Sigma/Final/sig"] = s

    def write_chis(self, ite: int, converged: bool, sus: dict, chi0: dict) -> None:
        """``write_chis`` (SRC/parquet_plot.f90:144-228).  ``sus``: whole-BZ
        ``sus_r`` (Nx*Ny*Nf/2, 4) per channel d, m, s, t; ``chi0``: whole-BZ
        ``chi0_ph``, ``chi0_pp`` (Nx*Ny*Nf/2) and ``chi0_ph_FF``,
        ``chi0_pp_FF`` (Nx*Ny*Nf/2, 4).  Magnetic and bare bubbles are written
        with the reference's minus sign."""
        p = self.p
        nh, nc = p.Nf // 2, p.Nx * p.Nx
        sets = {"chi_d": _r(sus["d"], (nh, nc, 4)), "chi_m": -_r(sus["m"], (nh, nc, 4)),
                "chi_s": _r(sus["s"], (nh, nc, 4)), "chi_t": _r(sus["t"], (nh, nc, 4)),
                "chi_0": -_r(chi0["chi0_ph"], (nh, nc)), "chi_0_pp": -_r(chi0["chi0_pp"], (nh, nc)),
                "chi_0_FF": -_r(chi0["chi0_ph_FF"], (nh, nc, 4)),
                "chi_0_pp_FF": -_r(chi0["chi0_pp_FF"], (nh, nc, 4))}
        final = ite == p.ite_max - 1 or converged
        for name, a in sets.items():
            ds = dataset(a)
            self.data[f"Chi/{name}_{ite:05d}"] = ds
            if final:
                self.data[f"Chi/Final/{name}"] = ds

    def save(self) -> str:
        np.savez(self.path, **self.data)
        return self.path


def write_F(directory, p, Nl: int, Nb: int, F: dict, rank: int = 0) -> str:
    """``write_F`` (SRC/parquet_plot.f90:232-276): the complete vertices of a
    rank as (Nf, Nl, Nf, Nl, Nb) in ``F_<kind>_<rank>.npz``."""
    path = os.path.join(str(directory), f"F_{kind_label(p, Nl)}_{rank:03d}.npz")
    data = {f"F/F_{r}": dataset(_r(F[r], (p.Nf, Nl, p.Nf, Nl, Nb))) for r in "dmst"}
    np.savez(path, **data)
    return path


def run_with_output(sol, directory) -> tuple[int, bool, str]:
    """``execute_loop`` with the reference's output (SRC/loop.f90:51-244 and
    SRC/tups.f90:80-82): Sigma and the susceptibilities at every output
    iteration, the vertices at the end when save_F is set.  ``sol`` is an
    unsharded ``Solver``.  Returns (iterations, converged, main file)."""
    p = sol.params
    out = Output(directory, p, sol.Nl)
    ite, converged = 0, False
    while not converged and ite < p.ite_max:
        info = sol.iteration(ite, readout=True)
        converged = info["converged"]
        if ite % 5 == 0 or ite == p.ite_max - 1 or converged:
            sus = {r: sol.sus(r, bz=True) for r in "dmst"}
            out.write_sigma(ite, converged, sol.Sigma)
            out.write_chis(ite, converged, sus, sol.chi0(bz=True))
        ite += 1
    path = out.save()
    if p.save_F:
        write_F(directory, p, sol.Nl, sol.Nb, {r: sol.F(r) for r in "dmst"}, sol.rank)
    return ite, converged, path

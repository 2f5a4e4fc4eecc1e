"""Batched LU form of the BSE over instances of uneven size.

``make_instances`` builds the standalone batched workload: n_q x n_w
bosonic (q, Omega) instances on an Nx x Nx lattice, each with its own
form-factor count N_ff in {1, 5, 9, 13} drawn by seed and N_nu fermionic
frequencies (n = N_ff * N_nu); chi is the nu-block-diagonal bare bubble of
the t = 1 lattice at half filling (Sigma = 0) projected on the instance's
form factors (parquet_chi.f90:470-521 with G = G0), and Gamma is complex
Gaussian, Hermitian-symmetrised and scaled so that the spectral radius of
Gamma chi is `rho` (estimated by power iteration).

``solve`` runs ``tups_bse_lu_batched``: F = (1 - c Gamma chi)^{-1} Gamma
(or Phi = F - Gamma) for all instances in one persistent launch.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import TupsError

NFF_TO_NEIGHBOURS = {1: 1, 5: 2, 9: 3, 13: 4}


@dataclass
class Instances:
    n: np.ndarray          # (I,) sizes
    nl: np.ndarray         # (I,) form-factor counts
    scale: np.ndarray      # (I,) c
    gamma: list            # I arrays (n, n) complex128, Fortran order
    chi: list              # I arrays (Nl, Nl, Nnu) complex128, Fortran order
    q: np.ndarray          # (I, 3): qx, qy (1-based), Omega (1-based)


def _form_factors(Nx: int, nff: int, nf: int) -> np.ndarray:
    from .parquet import Params, host_tables
    t = host_tables(Params(Nx=Nx, Nf=nf, neighbours=NFF_TO_NEIGHBOURS[nff]))
    assert t["dims"]["Nl"] == nff
    return t["FF"]


def bare_chi_blocks(Nx: int, nf: int, beta: float, qx: int, qy: int, w: int, FF: np.ndarray) -> np.ndarray:
    """nu-diagonal blocks of chi_ph_LL for G = 1/(i nu - e_k) (mu = 0)."""
    k = np.arange(Nx)
    e = -2.0 * np.cos(2.0 * math.pi / Nx * k)[:, None] - 2.0 * np.cos(2.0 * math.pi / Nx * k)[None, :]
    nu = np.arange(1, nf + 1)
    fr = math.pi / beta * (2.0 * (nu - nf // 2 - 1) + 1.0)
    frq = math.pi / beta * (2.0 * ((nu + w - 1) - nf // 2 - 1) + 1.0)
    ekq = np.roll(np.roll(e, -(qx - 1), axis=0), -(qy - 1), axis=1)
    g = 1.0 / (1j * fr[None, None, :] - e[:, :, None])
    gq = 1.0 / (1j * frq[None, None, :] - ekq[:, :, None])
    chi_k = g * gq
    return np.asfortranarray(np.einsum("xyn,xya,xyb->abn", chi_k, FF, FF))


def spectral_radius(M: np.ndarray, seed: int = 0) -> float:
    """Largest |eigenvalue|: LAPACK for small matrices, ARPACK otherwise
    (plain power iteration stalls on these non-normal matrices)."""
    n = M.shape[0]
    if n <= 128:
        return float(np.max(np.abs(np.linalg.eigvals(M))))
    from scipy.sparse.linalg import eigs
    rng = np.random.default_rng(seed)
    v0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    vals = eigs(M, k=1, which="LM", tol=1e-8, ncv=12, v0=v0, return_eigenvectors=False)
    return float(np.max(np.abs(vals)))


def gamma_chi_radius(G: np.ndarray, chi_blocks: np.ndarray, seed: int = 0) -> float:
    """Spectral radius of Gamma chi without forming it: chi acts block-wise."""
    nl, _, nf = chi_blocks.shape
    n = nl * nf
    if n <= 128:
        return spectral_radius(G @ chi_dense(chi_blocks))
    from scipy.sparse.linalg import LinearOperator
    cb = np.ascontiguousarray(np.transpose(chi_blocks, (2, 0, 1)))  # (nu, l1, l2)
    Gc = np.ascontiguousarray(G)

    def mv(v):
        v = np.asarray(v).reshape(nl, nf).T[:, :, None]  # (nu, l, 1)
        w = np.matmul(cb, v)[:, :, 0].T.reshape(n)
        return Gc @ w

    return spectral_radius(LinearOperator((n, n), matvec=mv, dtype=np.complex128), seed=seed)


def chi_dense(chi_blocks: np.ndarray) -> np.ndarray:
    nl, _, nf = chi_blocks.shape
    n = nl * nf
    out = np.zeros((n, n), dtype=np.complex128)
    nu = np.arange(nf)
    for a in range(nl):
        for b in range(nl):
            out[a * nf + nu, b * nf + nu] = chi_blocks[a, b, :]
    return out


def _one_instance(args):
    """Gamma and chi of instance i; its random stream depends on (seed, i) only."""
    i, seed, nl, nf, Nx, beta, rho, qx, qy, w, FF = args
    rng = np.random.default_rng([seed, i])
    n = nl * nf
    cb = bare_chi_blocks(Nx, nf, beta, qx, qy, w, FF)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    G = 0.5 * (A + A.conj().T)
    r = gamma_chi_radius(G, cb, seed=seed + i)
    G = G * (rho / r) if r > 0 else G
    return np.asfortranarray(G), cb


def make_instances(n_q: int = 64, n_w: int = 16, nf: int = 64, Nx: int = 8, beta: float = 10.0, rho: float = 0.9,
                   nff_choices=(1, 5, 9, 13), seed: int = 0, workers: int = 0) -> Instances:
    """The batched workload; `workers` > 0 generates in a spawn process pool
    (start it before any CUDA work in the calling process)."""
    rng = np.random.default_rng(seed)
    nI = n_q * n_w
    nffs = rng.choice(np.array(nff_choices), size=nI)
    FFs = {f: _form_factors(Nx, int(f), nf) for f in set(int(x) for x in nffs)}
    qs = [(qx, qy) for qx in range(1, Nx + 1) for qy in range(1, Nx + 1)][:n_q]
    jobs = []
    for i in range(nI):
        (qx, qy), w = qs[i // n_w], i % n_w + 1
        jobs.append((i, seed, int(nffs[i]), nf, Nx, beta, rho, qx, qy, w, FFs[int(nffs[i])]))
    if workers > 0:
        import multiprocessing as mp
        import os
        from concurrent.futures import ProcessPoolExecutor
        # one BLAS thread per worker: the children inherit these at spawn
        saved = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")}
        for k in saved:
            os.environ[k] = "1"
        try:
            with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
                res = list(ex.map(_one_instance, jobs, chunksize=1))
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
    else:
        res = [_one_instance(j) for j in jobs]
    gam = [r[0] for r in res]
    chis = [r[1] for r in res]
    ns = [int(nffs[i]) * nf for i in range(nI)]
    q = [(j[7], j[8], j[9]) for j in jobs]
    return Instances(n=np.array(ns, dtype=np.int32), nl=nffs.astype(np.int32),
                     scale=np.ones(nI), gamma=gam, chi=chis, q=np.array(q, dtype=np.int32))


def algorithmic_flops(n: np.ndarray) -> float:
    """LU (8/3 n^3) plus the solve for n right-hand sides (8 n^3), complex."""
    n = np.asarray(n, dtype=np.float64)
    return float(np.sum((8.0 / 3.0 + 8.0) * n ** 3))


def pack(inst: Instances):
    g = np.concatenate([np.ravel(a, order="F") for a in inst.gamma])
    c = np.concatenate([np.ravel(a, order="F") for a in inst.chi])
    return g, c


class LuBatch:
    """Device-resident batch: inputs uploaded once, solved by `run`."""

    def __init__(self, inst: Instances, device: int = 0):
        import torch
        self.lib = _lib.load()
        self.inst = inst
        self.dev = torch.device(f"cuda:{device}")
        torch.cuda.set_device(self.dev)
        g, c = pack(inst)
        self.g_host, self.c_host = g, c
        self.dg = torch.from_numpy(g).to(self.dev)
        self.dc = torch.from_numpy(c).to(self.dev)
        self.out = torch.empty_like(self.dg)
        self.work = torch.empty_like(self.dg)
        self.piv = torch.empty(int(inst.n.sum()), dtype=torch.int32, device=self.dev)
        self.n = np.ascontiguousarray(inst.n, dtype=np.int32)
        self.nl = np.ascontiguousarray(inst.nl, dtype=np.int32)
        self.sc = np.ascontiguousarray(inst.scale, dtype=np.float64)
        self.status = np.zeros(len(inst.n), dtype=np.int32)

    def run(self, want_phi: bool = False, check: bool = True) -> None:
        import torch
        stream = torch.cuda.current_stream(self.dev)
        st = self.status.ctypes.data_as(C.POINTER(C.c_int)) if check else None
        rc = self.lib.tups_bse_lu_batched(
            len(self.n), self.n.ctypes.data_as(C.POINTER(C.c_int)), self.nl.ctypes.data_as(C.POINTER(C.c_int)),
            self.sc.ctypes.data_as(C.POINTER(C.c_double)), C.c_void_p(self.dg.data_ptr()),
            C.c_void_p(self.dc.data_ptr()), C.c_void_p(self.out.data_ptr()), C.c_void_p(self.work.data_ptr()),
            C.c_void_p(self.piv.data_ptr()), int(want_phi), st, C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise TupsError(rc, "tups_bse_lu_batched failed")
        if check and np.any(self.status):
            raise TupsError(-4, f"singular pivot in instances {np.nonzero(self.status)[0].tolist()}")

    def run_split(self, slices: int = 5, tol: float = 1e-10, max_refine: int = 6, want_phi: bool = False,
                  check: bool = True) -> dict:
        """The same solve in split precision with FP64 iterative refinement
        (``tups_bse_lu_split_batched``): LU and triangular-solve updates on
        int8 slices (tcgen05), residual Gamma - A X in FP64, corrections
        until max|residual| <= tol max|Gamma| per instance.  Returns the
        corrections applied and the final relative residual per instance."""
        import torch
        nI = len(self.n)
        nptr = self.n.ctypes.data_as(C.POINTER(C.c_int))
        need = int(self.lib.tups_bse_lu_split_workspace(nI, nptr, slices))
        if need == 0:
            raise TupsError(-7, "bad sizes for the split LU workspace")
        if getattr(self, "split_work", None) is None or self.split_work.numel() < need:
            self.split_work = torch.empty(need, dtype=torch.uint8, device=self.dev)
        steps = np.zeros(nI, dtype=np.int32)
        resid = np.zeros(nI, dtype=np.float64)
        stream = torch.cuda.current_stream(self.dev)
        rc = self.lib.tups_bse_lu_split_batched(
            nI, nptr, self.nl.ctypes.data_as(C.POINTER(C.c_int)), self.sc.ctypes.data_as(C.POINTER(C.c_double)),
            C.c_void_p(self.dg.data_ptr()), C.c_void_p(self.dc.data_ptr()), C.c_void_p(self.out.data_ptr()),
            int(want_phi), int(slices), float(tol), int(max_refine), C.c_void_p(self.split_work.data_ptr()),
            C.c_size_t(self.split_work.numel()), steps.ctypes.data_as(C.POINTER(C.c_int)),
            resid.ctypes.data_as(C.POINTER(C.c_double)), self.status.ctypes.data_as(C.POINTER(C.c_int)),
            C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise TupsError(rc, "tups_bse_lu_split_batched failed")
        if check and np.any(self.status):
            raise TupsError(-4, f"singular pivot in instances {np.nonzero(self.status)[0].tolist()}")
        return {"refinements": steps, "residual": resid}

    def results(self) -> list:
        host = self.out.cpu().numpy()
        res, off = [], 0
        for ni in self.inst.n:
            res.append(host[off:off + ni * ni].reshape((ni, ni), order="F"))
            off += ni * ni
        return res


def solve(inst: Instances, device: int = 0, want_phi: bool = False) -> list:
    """F (or Phi) for every instance, computed on the GPU; (n, n) arrays."""
    b = LuBatch(inst, device)
    b.run(want_phi=want_phi)
    return b.results()


def solve_split(inst: Instances, device: int = 0, want_phi: bool = False, slices: int = 5, tol: float = 1e-10,
                max_refine: int = 6):
    """F (or Phi) in split precision with FP64 refinement; returns the
    (n, n) arrays and the per-instance refinement record."""
    b = LuBatch(inst, device)
    info = b.run_split(slices=slices, tol=tol, max_refine=max_refine, want_phi=want_phi)
    return b.results(), info

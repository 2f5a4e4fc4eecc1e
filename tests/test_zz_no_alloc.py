"""tups_bse_noalloc: the BSE update for callers that may not allocate device
memory while they call the library (for instance a host that has handed all
device memory to its own arena, or a loop that must not trigger the
synchronisation a cudaMalloc/cudaFree implies).  It must reproduce the
regular BSE entry point, use only caller-owned buffers plus its static
scratch, and keep doing so on consecutive calls.  This file is collected
last so that a failure here never hides the other tests' results."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12
COEF = {"d": 0.5, "m": 0.5, "s": -0.25, "t": 0.25}


def _blocks(dense: np.ndarray, Nl: int, Nf: int) -> np.ndarray:
    """nu-diagonal blocks (Nl, Nl, Nf) of a dense chi_LL (Nz, Nz)."""
    out = np.empty((Nl, Nl, Nf), dtype=np.complex128, order="F")
    nu = np.arange(Nf)
    for l1 in range(Nl):
        for l2 in range(Nl):
            out[l1, l2, :] = dense[l1 * Nf + nu, l2 * Nf + nu]
    return out


def test_bse_noalloc_matches_bse(gpu_lib):
    import torch

    from tups_b200 import Params, Solver

    p = Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=10)
    sol = Solver(p)
    sol.iteration(0)
    sol.calc_Gkw_Grt(1)
    Nz, Nf, Nl, Nb = sol.Nz, sol.Nf, sol.Nl, sol.Nb
    gam = {r: sol.G(r) for r in "dmst"}
    fv = {r: sol.F(r) for r in "dmst"}
    chi_ph = np.empty((Nl, Nl, Nf, Nb), dtype=np.complex128, order="F")
    chi_pp = np.empty((Nl, Nl, Nf, Nb), dtype=np.complex128, order="F")
    for q in range(Nb):
        ph, pp = sol.calc_chi(q + 1)
        chi_ph[:, :, :, q] = _blocks(ph, Nl, Nf)
        chi_pp[:, :, :, q] = _blocks(pp, Nl, Nf)
    sol.BSE(1)
    phi_ref = {r: sol.G(r) for r in "dmst"}
    sol.close()

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)

    def dev_buf(a: np.ndarray) -> torch.Tensor:
        return torch.from_numpy(np.ravel(a, order="F").copy()).to(dev)

    chi_d = {"ph": dev_buf(chi_ph), "pp": dev_buf(chi_pp)}
    alpha = 1.0 / (p.beta * p.Nx * p.Nx)
    free_after = []
    for call in range(2):
        for r in "dmst":
            g = dev_buf(gam[r])
            f = dev_buf(fv[r])
            chi = chi_d["ph" if r in "dm" else "pp"]
            torch.cuda.synchronize(dev)
            rc = gpu_lib.tups_bse_noalloc(Nb, Nz, Nf, Nl, C.c_void_p(g.data_ptr()), C.c_void_p(f.data_ptr()),
                                          C.c_void_p(chi.data_ptr()), COEF[r] * p.f_damping * alpha, p.f_damping,
                                          C.c_void_p(stream.cuda_stream))
            assert rc == 0
            torch.cuda.synchronize(dev)
            out = g.cpu().numpy().reshape((Nz, Nz, Nb), order="F")
            err = np.abs(out - phi_ref[r]).max() / np.abs(phi_ref[r]).max()
            assert err < TOL, (call, r, err)
            free_after.append(torch.cuda.mem_get_info(dev)[0])
    # after the first call has placed the static scratch, free device memory
    # does not move: the entry point allocates nothing
    assert len(set(free_after[1:])) == 1


def test_bse_noalloc_rejects_oversize(gpu_lib):
    """Nz beyond the static scratch limit is refused before any GPU work."""
    dummy = C.c_void_p(1)
    rc = gpu_lib.tups_bse_noalloc(1, 1040, 80, 13, dummy, dummy, dummy, 1.0, 0.5, None)
    assert rc == -6
    rc = gpu_lib.tups_bse_noalloc(1, 100, 8, 13, dummy, dummy, dummy, 1.0, 0.5, None)
    assert rc == -7


def _reference_update(gam, fv, chi, scale, f_damping):
    """The documented formula, per instance: Phi = scale [(Gamma chi) F +
    F (chi Gamma)] + (1 - f)(F - Gamma), chi rebuilt dense from its blocks."""
    n_inst, Nz = gam.shape[0], gam.shape[1]
    Nl, Nf = chi.shape[1], chi.shape[3]
    dense = np.zeros((n_inst, Nz, Nz), dtype=np.complex128)
    nu = np.arange(Nf)
    for l1 in range(Nl):
        for l2 in range(Nl):
            dense[:, l1 * Nf + nu, l2 * Nf + nu] = chi[:, l1, l2, :]
    gc = np.matmul(gam, dense)
    cg = np.matmul(dense, gam)
    return scale * (np.matmul(gc, fv) + np.matmul(fv, cg)) + (1.0 - f_damping) * (fv - gam)


@pytest.mark.parametrize("shape", [(576, 9, 64, 8), (1024, 16, 64, 3), (2, 1, 2, 70000)],
                         ids=["nz576_3_chunks", "nz1024_chunk_1", "nz2_grid_y_cap"])
def test_bse_noalloc_multiple_chunks(gpu_lib, shape):
    """More instances than one pass through the static scratch holds: Nz = 576
    (3 instances per pass), the Nz = 1024 limit (1 per pass) and Nz = 2, where
    the pass is capped at 65535 instances by the grid; two calls in a row."""
    import torch

    Nz, Nl, Nf, n_inst = shape
    rng = np.random.default_rng(Nz + n_inst)

    def crandn(*s):
        return rng.standard_normal(s) + 1j * rng.standard_normal(s)

    # row-major (inst, col, row) == column-major (row, col) per instance
    gam = crandn(n_inst, Nz, Nz)
    fv = crandn(n_inst, Nz, Nz)
    chi = crandn(n_inst, Nl, Nl, Nf) * 0.1       # (inst, l2, l1, nu) row-major
    scale, f_damping = 0.37, 0.5
    # column-major reference: A_cm = X.T per instance
    chi_cm = np.transpose(chi, (0, 2, 1, 3))       # (inst, l1, l2, nu): chi[l1, l2, nu]
    ref = _reference_update(np.transpose(gam, (0, 2, 1)), np.transpose(fv, (0, 2, 1)), chi_cm, scale, f_damping)
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    # chi blocks in the documented layout l1 + Nl*(l2 + Nl*nu): row-major (inst, nu, l2, l1)
    chi_buf = torch.from_numpy(np.ascontiguousarray(np.transpose(chi_cm, (0, 3, 2, 1)))).to(dev)
    f_buf = torch.from_numpy(fv).to(dev)
    for call in range(2):
        g = torch.from_numpy(gam).to(dev)
        torch.cuda.synchronize(dev)
        rc = gpu_lib.tups_bse_noalloc(n_inst, Nz, Nf, Nl, C.c_void_p(g.data_ptr()), C.c_void_p(f_buf.data_ptr()),
                                      C.c_void_p(chi_buf.data_ptr()), scale, f_damping,
                                      C.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize(dev)
        out = np.transpose(g.cpu().numpy(), (0, 2, 1))
        err = np.abs(out - ref).max() / np.abs(ref).max()
        assert err < TOL, (call, err)

"""Split-precision GEMM (int8 tcgen05) on a B200 against the oracle's
emulation and against FP64."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import split as S
import parity

pytestmark = pytest.mark.gpu

# the GPU sums the same exact int32 diagonals as the oracle and adds them in
# the same FP64 order: only the conversion of the final sums may differ
EMU_TOL = 1e-15


def _zgemm_split(lib, A, B, s):
    import torch
    batch, M, K = A.shape
    N = B.shape[2]
    # column-major per batch = A_b^T row-major
    dA = torch.from_numpy(np.ascontiguousarray(A.transpose(0, 2, 1))).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.transpose(0, 2, 1))).cuda()
    dC = torch.zeros((batch, N, M), dtype=torch.complex128, device="cuda")
    ws = lib.tups_zgemm_split_workspace(batch, M, N, K, s)
    assert ws > 0
    work = torch.empty(ws, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.tups_zgemm_split(batch, M, N, K, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                              C.c_void_p(dC.data_ptr()), s, C.c_void_p(work.data_ptr()), ws, C.c_void_p(stream))
    assert rc == 0, rc
    return dC.cpu().numpy().transpose(0, 2, 1)


@pytest.mark.parametrize("dims", [(2, 128, 80, 64), (3, 200, 150, 300), (1, 40, 8, 7)],
                         ids=["aligned", "ragged", "tiny"])
@pytest.mark.parametrize("s", [2, 5, 8])
def test_zgemm_split_matches_the_emulation(gpu_lib, dims, s):
    batch, M, N, K = dims
    rng = np.random.default_rng(M + N + K + s)
    A = (rng.normal(size=(batch, M, K)) + 1j * rng.normal(size=(batch, M, K))) * np.logspace(-2, 2, K)[None, None, :]
    B = rng.normal(size=(batch, K, N)) + 1j * rng.normal(size=(batch, K, N))
    got = _zgemm_split(gpu_lib, A, B, s)
    for b in range(batch):
        emu = S.ozaki_zgemm(A[b], B[b], s)
        assert parity.rel(got[b], emu) <= EMU_TOL, (b, parity.rel(got[b], emu))
        exact = A[b] @ B[b]
        assert parity.rel(got[b], exact) <= 10.0 ** (1.6 - 2.0 * s) + 1e-14


@pytest.mark.parametrize("dims", [(2, 256, 80, 64), (1, 300, 150, 300)], ids=["pair", "pair_ragged"])
@pytest.mark.parametrize("s", [3, 8])
def test_zgemm_split_cta_pairs_match_the_emulation(gpu_lib, dims, s):
    """The CTA-pair form (M = 256 tiles over two SMs) writes the emulation's
    result like the one-SM form."""
    batch, M, N, K = dims
    rng = np.random.default_rng(7 * M + N + K + s)
    A = (rng.normal(size=(batch, M, K)) + 1j * rng.normal(size=(batch, M, K))) * np.logspace(-2, 2, K)[None, None, :]
    B = rng.normal(size=(batch, K, N)) + 1j * rng.normal(size=(batch, K, N))
    gpu_lib.tups_set_split_cta_pairs(1)
    try:
        got = _zgemm_split(gpu_lib, A, B, s)
    finally:
        gpu_lib.tups_set_split_cta_pairs(0)
    for b in range(batch):
        emu = S.ozaki_zgemm(A[b], B[b], s)
        assert parity.rel(got[b], emu) <= EMU_TOL, (b, parity.rel(got[b], emu))


def test_split_bse_against_fp64(gpu_lib):
    from oracle import tups_oracle as O
    from tups_b200 import Solver
    p = O.Params(beta=3.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, tprime=-0.1, f_damping=0.5,
                 ite_max=20)
    sol = Solver(parity.to_solver_params(p))
    for ite in range(3):
        sol.iteration(ite)
    sol.checkpoint(True)
    sol.calc_Gkw_Grt(3)
    sol.BSE(3)
    ref = [sol.G(r) for r in range(4)]
    for s, tol in ((8, 1e-13), (6, 1e-9), (4, 1e-5)):
        sol.checkpoint(False)
        sol.set_bse_precision(s)
        assert sol.bse_slices == s
        sol.calc_Gkw_Grt(3)
        sol.BSE(3)
        err = max(parity.rel(sol.G(r), ref[r]) for r in range(4))
        assert err <= tol, (s, err)
    sol.close()


# Both loops of a fixed-point comparison stop at max|dSigma| < 1e-12, so that
# the distance of each from the common fixed point (about the last change
# over one minus the contraction rate) stays well below the 1e-10 bound
CONV_ABS = 1e-12
SIGMA_TOL = 1e-10


def test_ladder_loop_reaches_the_fp64_fixed_point(gpu_lib):
    from tups_b200 import Params, Solver
    p = Params(beta=3.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, tprime=-0.1, f_damping=0.5,
               ite_max=10 ** 6, conv_abs=CONV_ABS)
    ref = Solver(p)
    n_ref = 0
    while not ref.iteration(n_ref)["converged"]:
        n_ref += 1
    n_ref += 1
    sig_ref = ref.Sigma
    ref.close()
    sol = Solver(p)
    sol.set_bse_precision(0, ladder=True)
    used = []
    n = 0
    while True:
        used.append(sol.bse_slices)
        ci = sol.iteration(n)
        n += 1
        if ci["converged"]:
            break
        assert n < 3 * n_ref
    # the tuner times FP64 on the first call and tries the split GEMM once
    assert used[0] == 0 and any(u > 0 for u in used)
    assert parity.rel(sol.Sigma, sig_ref) <= SIGMA_TOL
    sol.close()


def test_fixed_slices_loop_reaches_the_fp64_fixed_point(gpu_lib):
    from tups_b200 import Params, Solver
    p = Params(beta=3.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, tprime=-0.1, f_damping=0.5,
               ite_max=10 ** 6, conv_abs=CONV_ABS)
    sols = {}
    for s in (0, 7):
        sol = Solver(p)
        sol.set_bse_precision(s)
        n = 0
        while not sol.iteration(n)["converged"]:
            n += 1
            assert n < 2000
        sols[s] = sol.Sigma
        sol.close()
    # 7 slices: GEMM error ~1e-13 relative; the fixed points agree to 1e-10
    assert parity.rel(sols[7], sols[0]) <= SIGMA_TOL


def test_graph_iterations_equal_plain_ones(gpu_lib):
    from tups_b200 import Params, Solver
    p = Params(beta=3.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, tprime=-0.1, f_damping=0.5,
               ite_max=100)
    out = {}
    for graph in (False, True):
        sol = Solver(p)
        sol.set_graph(graph)
        infos = [sol.iteration(i) for i in range(7)]   # ite 5 applies the output block
        out[graph] = (sol.Sigma, sol.F(0), sol.G(2), sol.mu,
                      [(c["dsigma_inf"],) + tuple(c[f"F_{r}_max"] for r in "dmst") for c in infos],
                      sol.kernel_launches)
        sol.close()
    a, b = out[False], out[True]
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert a[3] == b[3] and a[4] == b[4]
    # graph replays count their kernels; iterations 1-6 replay one, where
    # max|F_r| rides on the vertex update (one launch fewer than k_fmax +
    # k_vertex_update)
    assert b[5] == a[5] - 6


def test_graph_with_ladder_converges(gpu_lib):
    from tups_b200 import Params, Solver
    p = Params(beta=3.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, tprime=-0.1, f_damping=0.5,
               ite_max=10 ** 6, conv_abs=CONV_ABS)
    ref = Solver(p)
    n = 0
    while not ref.iteration(n)["converged"]:
        n += 1
    sig = ref.Sigma
    ref.close()
    sol = Solver(p)
    sol.set_graph(True)
    sol.set_bse_precision(0, ladder=True)
    m = 0
    while not sol.iteration(m)["converged"]:
        m += 1
        assert m < 3 * n + 10
    assert parity.rel(sol.Sigma, sig) <= SIGMA_TOL
    sol.close()

"""Error behaviour of the C ABI on a GPU.  Every failure here is produced on
the host or by a bounded device loop; nothing faults, traps or hangs."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(**kw):
    from tups_b200 import Params
    base = dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=8, neighbours=2, ite_max=5)
    base.update(kw)
    return Params(**base)


def test_call_order_is_checked(gpu_lib):
    from tups_b200 import Solver, TupsError
    sol = Solver(_params())
    with pytest.raises(TupsError, match="STATE"):
        sol.BSE(0)
    sol.calc_Gkw_Grt(0)
    sol.BSE(0)
    with pytest.raises(TupsError, match="STATE"):
        sol.calc_PhiR(0)
    sol.calculate_expSqR()
    sol.calc_PhiR(0)
    with pytest.raises(TupsError, match="STATE"):
        sol.calculate_PAE()
    sol.close()


def test_bisection_cap_reports_error(gpu_lib):
    """U = 0 off half filling: the bracket [mu-U, mu+U] has zero width; the
    device loop stops at its step cap and the call returns MU_NOCONV."""
    from tups_b200 import Solver, TupsError
    sol = Solver(_params(U=0.0, nParticle=0.9))
    with pytest.raises(TupsError, match="MU_NOCONV"):
        sol.calc_Gkw_Grt(0)
    # the context stays usable
    sol.mu = 0.0
    sol.close()


def test_nan_in_sigma_is_detected(gpu_lib):
    from tups_b200 import Solver, TupsError
    sol = Solver(_params())
    s = np.zeros(sol.Nt, dtype=np.complex128)
    s[3] = np.nan
    sol.Sigma = s
    with pytest.raises(TupsError, match="NAN"):
        sol.conv()
    sol.close()


def test_bad_sizes_rejected_before_allocation(gpu_lib):
    from tups_b200 import Solver, TupsError
    with pytest.raises(TupsError):
        Solver(_params(Nx=6, Nf=7))


def test_bad_channel_index(gpu_lib):
    from tups_b200 import Solver, TupsError
    sol = Solver(_params())
    with pytest.raises(TupsError):
        sol._vertex(7, 0)
    with pytest.raises(TupsError):
        sol.calc_chi(0)
    sol.close()


def test_split_gemm_wait_runs_out_and_recovers(gpu_lib):
    """The split GEMM's pipeline waits are bounded: with the stall test the
    MMA warp waits on a barrier nothing signals, its wait runs out after the
    set number of cycles, the kernel drains its in-flight copies, frees its
    tensor memory and returns, and the call reports TUPS_ERR_TIMEOUT.  The
    next call, with the default limit, returns the right product."""
    import ctypes as C
    import torch
    from oracle import split as S
    batch, M, N, K, s = 4, 256, 192, 320, 4
    rng = np.random.default_rng(9)
    A = rng.normal(size=(batch, M, K)) + 1j * rng.normal(size=(batch, M, K))
    B = rng.normal(size=(batch, K, N)) + 1j * rng.normal(size=(batch, K, N))
    dA = torch.from_numpy(np.ascontiguousarray(A.transpose(0, 2, 1))).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B.transpose(0, 2, 1))).cuda()
    dC = torch.zeros((batch, N, M), dtype=torch.complex128, device="cuda")
    ws = gpu_lib.tups_zgemm_split_workspace(batch, M, N, K, s)
    work = torch.empty(ws, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        return gpu_lib.tups_zgemm_split(batch, M, N, K, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                        C.c_void_p(dC.data_ptr()), s, C.c_void_p(work.data_ptr()), ws,
                                        C.c_void_p(stream))
    try:
        assert gpu_lib.tups_set_split_wait(2_000_000, 1) == 0   # ~1 ms, then stall once
        assert call() == -5                                      # TUPS_ERR_TIMEOUT
    finally:
        assert gpu_lib.tups_set_split_wait(0, 0) == 0
    torch.cuda.synchronize()
    assert call() == 0
    got = dC.cpu().numpy().transpose(0, 2, 1)
    for b in range(batch):
        emu = S.ozaki_zgemm(A[b], B[b], s)
        assert np.abs(got[b] - emu).max() <= 1e-15 * np.abs(emu).max()

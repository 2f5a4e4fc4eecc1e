"""LU form of the BSE (F = (1 - c Gamma chi)^{-1} Gamma), batched over
instances of uneven size: CPU checks of the oracle and the workload
generator, GPU parity with LAPACK (scipy zgetrf/zgetrs)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import lu as LU


def test_lu_form_is_the_fixed_point_of_the_damped_update():
    """The reference's damped two-ordering BSE update, iterated with Gamma
    fixed, converges to the LU solution."""
    from tups_b200.bse_batched import make_instances
    inst = make_instances(n_q=2, n_w=1, nf=8, nff_choices=(1, 5), rho=0.6, seed=3)
    for g, c in zip(inst.gamma, inst.chi):
        F_lu = LU.bse_lu(g, c, 1.0)
        F_it = LU.damped_fixed_point(g, c, 1.0, f=0.5)
        assert np.abs(F_lu - F_it).max() <= 1e-12 * np.abs(F_lu).max()


def test_generator_is_seeded_and_scaled():
    from tups_b200.bse_batched import chi_dense, make_instances, spectral_radius
    a = make_instances(n_q=3, n_w=2, nf=8, seed=7)
    b = make_instances(n_q=3, n_w=2, nf=8, seed=7)
    assert np.array_equal(a.nl, b.nl)
    for x, y in zip(a.gamma, b.gamma):
        assert np.array_equal(x, y)
    for g, c in zip(a.gamma, a.chi):
        assert np.allclose(g, g.conj().T)
        assert np.max(np.abs(np.linalg.eigvals(g @ chi_dense(c)))) == pytest.approx(0.9, rel=1e-8)
    assert set(a.n.tolist()) <= {8, 40, 72, 104}


@pytest.mark.gpu
def test_batched_lu_matches_lapack(gpu_lib):
    from tups_b200.bse_batched import make_instances, solve
    inst = make_instances(n_q=6, n_w=4, nf=16, seed=11)  # n in {16, 80, 144, 208}
    assert len(set(inst.n.tolist())) >= 3
    F = solve(inst)
    for i, (g, c) in enumerate(zip(inst.gamma, inst.chi)):
        ref = LU.bse_lu(g, c, 1.0)
        err = np.abs(F[i] - ref).max() / np.abs(ref).max()
        assert err < 1e-12, (i, int(inst.n[i]), err)


@pytest.mark.gpu
def test_batched_lu_phi_and_scale(gpu_lib):
    from tups_b200.bse_batched import make_instances, solve
    inst = make_instances(n_q=2, n_w=3, nf=12, seed=5, rho=0.5)
    inst.scale = np.linspace(0.5, 1.5, len(inst.n))
    Phi = solve(inst, want_phi=True)
    for i, (g, c) in enumerate(zip(inst.gamma, inst.chi)):
        ref = LU.bse_lu(g, c, float(inst.scale[i])) - g
        assert np.abs(Phi[i] - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.gpu
def test_batched_lu_reports_singular_pivot(gpu_lib):
    """Gamma chi with an eigenvalue 1 makes A = I - Gamma chi singular; the
    status array reports the column instead of returning NaNs silently."""
    from tups_b200 import TupsError
    from tups_b200.bse_batched import Instances, solve
    n = 8
    chi = np.zeros((1, 1, n), dtype=np.complex128, order="F")
    chi[0, 0, :] = 1.0
    g = np.asfortranarray(np.eye(n, dtype=np.complex128))  # A = I - I = 0
    inst = Instances(n=np.array([n], dtype=np.int32), nl=np.array([1], dtype=np.int32), scale=np.ones(1),
                     gamma=[g], chi=[chi], q=np.zeros((1, 3), dtype=np.int32))
    with pytest.raises(TupsError, match="singular"):
        solve(inst)


@pytest.mark.gpu
@pytest.mark.parametrize("slices", [4, 5, 7])
def test_split_lu_with_refinement_matches_lapack(gpu_lib, slices):
    """Split-precision LU (int8 trailing and solve updates) refined in FP64
    to the LAPACK answer; sizes up to 2 blocks of 128 plus a ragged tail."""
    from tups_b200.bse_batched import make_instances, solve_split
    inst = make_instances(n_q=4, n_w=4, nf=48, seed=13, nff_choices=(1, 5, 9))  # n in {48, 240, 432}
    assert len(set(inst.n.tolist())) >= 2
    F, info = solve_split(inst, slices=slices, tol=1e-12, max_refine=8)
    assert np.all(info["residual"] <= 1e-12), info
    for i, (g, c) in enumerate(zip(inst.gamma, inst.chi)):
        ref = LU.bse_lu(g, c, 1.0)
        err = np.abs(F[i] - ref).max() / np.abs(ref).max()
        assert err < 1e-12, (i, int(inst.n[i]), slices, err)
    # the int8 factors alone are not FP64-accurate: at least one correction
    assert int(info["refinements"].max()) >= 1


@pytest.mark.gpu
def test_split_lu_phi_scale_and_unrefined_error(gpu_lib):
    """want_phi and per-instance scales; without refinement the error is the
    split GEMM's, after refinement the FP64 LU's."""
    from tups_b200.bse_batched import LuBatch, make_instances
    inst = make_instances(n_q=2, n_w=3, nf=40, seed=5, rho=0.5, nff_choices=(1, 5))
    inst.scale = np.linspace(0.5, 1.5, len(inst.n))
    b = LuBatch(inst)
    refs = [LU.bse_lu(g, c, float(inst.scale[i])) - g for i, (g, c) in enumerate(zip(inst.gamma, inst.chi))]
    errs = {}
    for steps in (0, 8):
        info = b.run_split(slices=3, tol=1e-12, max_refine=steps, want_phi=True)
        out = b.results()
        errs[steps] = max(np.abs(out[i] - refs[i]).max() / np.abs(refs[i]).max() for i in range(len(refs)))
    assert 1e-9 < errs[0] < 1e-2, errs
    assert errs[8] < 1e-12, errs

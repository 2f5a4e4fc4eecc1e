"""The warm start on a B200: MLP kernels vs the float64 oracle, the warm-start
entry point vs the oracle, checkpoint/restore, and the fallback."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import tups_oracle as O
from oracle import warmstart as OW
import parity

pytestmark = pytest.mark.gpu

# FP32 kernels against the float64 oracle: max-norm relative error
MLP_TOL = 1e-4


@pytest.mark.parametrize("shape", [(37, 64, 3, 11, 20), (964, 512, 3, 968, 32)], ids=["small", "config5"])
def test_mlp_forward_and_gradients_match_oracle(gpu_lib, shape):
    from tups_b200.warmstart import MLP
    n_in, hidden, layers, n_out, batch = shape
    net = MLP(n_in, n_out, hidden, layers, max_batch=64, seed=5)
    rng = np.random.default_rng(7)
    p = net.get_params() + rng.normal(0, 0.02, net.n_params).astype(np.float32)
    net.set_params(p)
    x = rng.normal(size=(batch, n_in)).astype(np.float32)
    t = rng.normal(size=(batch, n_out)).astype(np.float32)
    y = net.forward(x)
    y_ref, _ = OW.mlp_forward(p, net.widths, x)
    assert parity.rel(y, y_ref) <= MLP_TOL
    loss, g = net.gradients(x, t)
    loss_ref, g_ref = OW.mlp_loss_grad(p, net.widths, x, t)
    assert abs(loss - loss_ref) <= MLP_TOL * loss_ref
    layout, _ = OW.mlp_layout(net.widths)
    for wo, bo, fin, fout in layout:   # per weight matrix and bias vector
        assert parity.rel(g[wo:bo], g_ref[wo:bo]) <= MLP_TOL
        assert parity.rel(g[bo:bo + fout], g_ref[bo:bo + fout]) <= MLP_TOL
    assert net.kernel_launches > 0
    net.close()


def test_mlp_training_fits_a_smooth_map(gpu_lib):
    from tups_b200.warmstart import MLP
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, size=(160, 6))
    a = rng.normal(size=(6, 4))
    t = np.sin(x @ a) + 0.1 * (x @ a) ** 2
    net = MLP(6, 4, 128, 3, max_batch=256, seed=1)
    loss0, _ = net.gradients(x, t)
    hist = net.train(x, t, batch=32, epochs=400, lr=2e-3, seed=3)
    loss1, _ = net.gradients(x, t)
    assert loss1 < 0.02 * loss0, (loss0, loss1)
    assert hist[-1] < 0.05 * hist[0]
    # determinism: same seed, same parameters
    net2 = MLP(6, 4, 128, 3, max_batch=256, seed=1)
    net2.train(x, t, batch=32, epochs=400, lr=2e-3, seed=3)
    np.testing.assert_allclose(net2.get_params(), net.get_params(), rtol=0, atol=1e-5)
    net.close()
    net2.close()


def _case():
    return O.Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, tprime=-0.1, f_damping=0.5,
                    ite_max=50)


def test_warm_start_matches_oracle(gpu_lib):
    from tups_b200 import Solver
    p = _case()
    st = O.initialize(p)
    O.iteration(st, 0)
    sol = Solver(parity.to_solver_params(p))
    sol.iteration(0)
    rng = np.random.default_rng(4)
    sigma = st.Sigma * (1.0 + 0.05 * rng.normal(size=st.Sigma.size))
    gam = np.array([2.1 + 0.02j, -1.8 - 0.01j, 3.9, 0.3j])
    OW.warm_start(st, sigma, gam)
    sol.warm_start(sigma, gam)
    assert abs(sol.mu - st.mu) <= 1e-12
    assert parity.rel(sol.Sigma, st.Sigma) == 0.0
    for i, r in enumerate("dmst"):
        assert parity.rel(sol.G(i), st.G[r]) == 0.0
        # LU with partial pivoting vs LAPACK's solve: <= 1e-12
        assert parity.rel(sol.F(i), st.F[r]) <= 1e-12, r
    # F is the fixed point of the library's own damped BSE update
    F = [sol.F(i) for i in range(4)]
    G = [sol.G(i) for i in range(4)]
    sol.calc_Gkw_Grt(1)
    sol.BSE(1)
    for i in range(4):
        assert parity.rel(sol.G(i), F[i] - G[i]) <= 1e-12
    # and the loop continues from it on both sides
    sol2 = Solver(parity.to_solver_params(p))
    sol2.iteration(0)
    sol2.warm_start(sigma, gam)
    for ite in range(1, 4):
        O.iteration(st, ite)
        sol2.iteration(ite)
    assert parity.rel(sol2.Sigma, st.Sigma) <= 1e-10
    sol.close()
    sol2.close()


def test_checkpoint_restore_replays_the_same_iterations(gpu_lib):
    from tups_b200 import Solver
    from tups_b200._lib import TupsError
    p = parity.to_solver_params(_case())
    sol = Solver(p)
    with pytest.raises(TupsError):
        sol.checkpoint(False)          # nothing stored yet
    for ite in range(2):
        sol.iteration(ite)
    sol.checkpoint(True)
    a = [sol.iteration(ite)["dsigma_inf"] for ite in range(2, 5)]
    sa, fa = sol.Sigma, sol.F(1)
    sol.checkpoint(False)
    b = [sol.iteration(ite)["dsigma_inf"] for ite in range(2, 5)]
    assert parity.rel(sol.Sigma, sa) <= 1e-14
    assert parity.rel(sol.F(1), fa) <= 1e-14
    np.testing.assert_allclose(a, b, rtol=1e-12)
    sol.close()


def test_run_warm_falls_back_on_a_bad_prediction(gpu_lib):
    from tups_b200 import warmstart as W
    p = parity.to_solver_params(_case())
    p.conv_abs = 1e-10
    cold = W.run_cold(p, max_iter=400)
    assert cold.converged

    def bad(params, sigma2):
        return sigma2 * 40.0, np.array([50.0, -50.0, 80.0, 9.0])

    def exact(params, sigma2):
        return cold.sigma, cold.gamma_l1

    fb = W.run_warm(p, bad, max_iter=400)
    assert fb.fallback and fb.converged
    assert fb.iterations <= cold.iterations + 1
    assert parity.rel(fb.sigma, cold.sigma) <= 1e-8
    # a kept warm start reaches the same fixed point
    kept = W.run_warm(p, exact, max_iter=400, accept=np.inf)
    assert kept.converged and not kept.fallback
    assert parity.rel(kept.sigma, cold.sigma) <= 1e-8


def test_sweep_trains_on_solver_runs_and_reports_the_gain(gpu_lib):
    """The whole learned warm start at a small size: seeded sweep, training by
    the library's kernels, warm vs cold on held-out runs.  Every warm run must
    reach the cold run's fixed point, and the fallback bounds the loss to one
    iteration per run on average."""
    from tups_b200 import Params
    from tups_b200 import warmstart as W
    base = Params(Nx=4, Nf=8, neighbours=1, f_damping=0.5, use_U2=True, ite_max=10 ** 6, conv_abs=1e-10)
    res = W.sweep(base, runs=36, n_train=28, seed=1, max_iter=1000, epochs=400, log=lambda *a: None)
    s = res["summary"]
    print("warm start sweep 4x4/Nl=1/Nf=8:", s)
    assert s["n_train"] >= 20 and s["n_test"] >= 6
    assert s["loss_last"] < 0.2 * s["loss_first"]
    assert s["all_warm_converged"]
    # the reference's mu bisection stops at |n - n0| < 1e-6 (parquet_chi.f90),
    # so two trajectories can settle on self-consistent mu values that differ
    # within that band: their fixed points agree to ~1e-6, not to 1e-10
    assert s["max_final_sigma_rel_diff"] <= 1e-4
    assert s["warm_iterations_mean"] <= s["cold_iterations_mean"] + 1.0

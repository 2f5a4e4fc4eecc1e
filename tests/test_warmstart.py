"""CPU checks of the warm start's host logic and of its oracle."""
from __future__ import annotations

import numpy as np

from oracle import tups_oracle as O
from oracle import warmstart as OW
from tups_b200 import warmstart as W


def test_oracle_mlp_gradient_matches_finite_differences():
    widths = [5, 7, 7, 3]
    p = W.mlp_init_params(widths, seed=1).astype(np.float64)
    p += np.random.default_rng(2).normal(0, 0.1, p.size)   # non-zero biases too
    rng = np.random.default_rng(3)
    x = rng.normal(size=(4, 5))
    t = rng.normal(size=(4, 3))
    loss, g = OW.mlp_loss_grad(p, widths, x, t)
    h = 1e-6
    num = np.empty_like(g)
    for i in range(p.size):
        e = np.zeros_like(p)
        e[i] = h
        num[i] = (OW.mlp_loss_grad(p + e, widths, x, t)[0] - OW.mlp_loss_grad(p - e, widths, x, t)[0]) / (2 * h)
    assert np.max(np.abs(num - g)) <= 1e-8 * max(1.0, np.max(np.abs(g)))
    assert loss > 0


def test_parameter_layout_agrees_with_oracle():
    widths = W.mlp_widths(484, 488)
    assert widths == [484, 512, 512, 512, 488]
    layout, n = OW.mlp_layout(widths)
    assert W.mlp_init_params(widths, 0).size == n
    assert layout[1][0] == 484 * 512 + 512


def test_sigma_wedge_round_trip_on_an_oracle_self_energy():
    # t' != 0 and n != 1 keep the C4v symmetry; two iterations give a
    # k- and nu-dependent Sigma
    p = O.Params(beta=3.0, U=2.0, nParticle=0.9, Nx=8, Nf=8, neighbours=1, tprime=-0.2, ite_max=10)
    st = O.initialize(p)
    for ite in range(2):
        O.iteration(st, ite)
    sig = st.Sigma.copy()
    red = W.reduce_sigma(sig, 8, 8)
    assert red.shape == (15, 8)
    back = W.expand_sigma(red, 8, 8)
    assert np.max(np.abs(back - sig)) <= 1e-13 * np.max(np.abs(sig))
    assert np.max(np.abs(sig.reshape(8, 8, 8).std(axis=(0, 1)))) > 1e-3 * np.max(np.abs(sig))  # k-dependent


def test_features_and_targets_shapes():
    p = W.Params(Nx=8, Nf=32, U=2.0, beta=5.0, nParticle=0.9, tprime=-0.1)
    s2 = np.zeros(8 * 8 * 32, dtype=complex)
    x = W.features(p, s2)
    y = W.targets(p, s2, s2 + 1j, np.arange(4) + 0.5j)
    assert x.shape == (4 + 2 * 15 * 32,) and x[0] == 2.0
    assert y.shape == (2 * 15 * 32 + 8,)
    assert np.all(y[15 * 32:2 * 15 * 32] == 1.0)


def test_oracle_warm_start_is_a_fixed_point_of_the_damped_update():
    p = O.Params(beta=2.0, U=2.0, nParticle=0.95, Nx=4, Nf=8, neighbours=2, tprime=-0.1, ite_max=10)
    st = O.initialize(p)
    O.iteration(st, 0)
    gam = np.array([1.7 + 0.01j, -1.9, 3.5, 0.2])
    OW.warm_start(st, st.Sigma.copy(), gam)
    F = {r: st.F[r].copy() for r in "dmst"}
    G = {r: st.G[r].copy() for r in "dmst"}
    O.bse(st, 1)    # G_r <- Phi_r of the damped update from (F, Gamma)
    for r in "dmst":
        phi = F[r] - G[r]
        assert np.max(np.abs(st.G[r] - phi)) <= 1e-12 * np.max(np.abs(F[r]))

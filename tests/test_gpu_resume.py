"""Resume from a state file (run on a B200): Sigma, mu and the vertices
saved after an iteration and loaded into a new context continue the loop
exactly as the uninterrupted run does."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import tups_oracle as O
import parity

pytestmark = pytest.mark.gpu


def test_resume_from_file_continues_bit_for_bit(gpu_lib, tmp_path):
    from tups_b200 import Solver
    p = parity.to_solver_params(O.Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2,
                                         f_damping=0.5, ite_max=20))
    a = Solver(p)
    for i in range(6):
        a.iteration(i)
    b = Solver(p)
    for i in range(3):
        b.iteration(i)
    b.save_state(tmp_path / "state.npz", 3)
    b.close()
    c = Solver(p)
    ite = c.load_state(tmp_path / "state.npz")
    assert ite == 3
    for i in range(ite, 6):
        c.iteration(i)
    assert np.array_equal(c.Sigma, a.Sigma)
    assert c.mu == a.mu
    for r in "dmst":
        assert np.array_equal(c.F(r), a.F(r)), r
        assert np.array_equal(c.G(r), a.G(r)), r
    a.close()
    c.close()


def test_load_state_rejects_other_sizes(gpu_lib, tmp_path):
    from tups_b200 import Solver
    small = Solver(parity.to_solver_params(O.Params(Nx=4, Nf=8, neighbours=1)))
    small.save_state(tmp_path / "s.npz", 0)
    small.close()
    other = Solver(parity.to_solver_params(O.Params(Nx=4, Nf=8, neighbours=2)))
    with pytest.raises(ValueError):
        other.load_state(tmp_path / "s.npz")
    other.close()

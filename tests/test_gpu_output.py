"""The reference's output written from the CUDA path (run on a B200):
`run_with_output` produces the same datasets as the oracle's loop with its
readout, to the parity bound, under the same keys."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import tups_oracle as O
import parity
from tups_b200.output import Output, as_fortran

pytestmark = pytest.mark.gpu


def test_run_with_output_matches_oracle(gpu_lib, tmp_path):
    from tups_b200 import Solver
    from tups_b200.output import run_with_output
    p = O.Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=3)
    (tmp_path / "gpu").mkdir()
    (tmp_path / "cpu").mkdir()
    sol = Solver(parity.to_solver_params(p))
    ite, conv, path = run_with_output(sol, tmp_path / "gpu")
    sol.close()
    assert ite == 3 and not conv
    st = O.initialize(p)
    out = Output(tmp_path / "cpu", p, st.Nl)
    for i in range(p.ite_max):
        c, info = O.iteration(st, i, with_readout=True)
        if "readout" in info:
            ro = info["readout"]
            out.write_sigma(i, c, st.Sigma)
            out.write_chis(i, c, {r: ro[f"sus_{r}"] for r in "dmst"},
                           {"chi0_ph": ro["chi0_ph_BZ"], "chi0_pp": ro["chi0_pp_BZ"],
                            "chi0_ph_FF": ro["chi0_ph_BZ_FF"], "chi0_pp_FF": ro["chi0_pp_BZ_FF"]})
    g, o = np.load(path), np.load(out.save())
    assert sorted(g.files) == sorted(o.files)
    for k in o.files:
        a, b = as_fortran(g[k]), as_fortran(o[k])
        assert a.shape == b.shape, k
        scale = max(float(np.max(np.abs(b))), 1e-300)
        assert float(np.max(np.abs(a - b))) <= 1e-12 * scale, k

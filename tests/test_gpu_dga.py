"""DGA Lambda input on the CUDA path (run on a B200): the library reads the
reference's Lambda files (SRC/parquet_util.f90:317-346), starts the vertices
from them (SRC/preprocessing.f90:100-116) and every phase that reads Lambda
(parquet equation base pass, SDE Lambda chi) follows the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import tups_oracle as O
import parity
from dga_tables import dga_tables, write_dga_files

pytestmark = pytest.mark.gpu

PHASE_TOL = 1e-12


@pytest.mark.parametrize("case", [
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=16, neighbours=1),
    dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2),
    dict(beta=2.0, U=2.0, nParticle=1.0, Nx=4, Nf=8, neighbours=2, use_U2=False, f_range=1),
], ids=["nl1", "nl5_n09", "noU2_frange1"])
def test_dga_phases_side_by_side(gpu_lib, tmp_path, case):
    stem = str(tmp_path / "Lambda")
    write_dga_files(stem, dga_tables(case["Nf"], case["U"], seed=7))
    p = O.Params(f_damping=0.5, ite_max=10, DGA=True, fname_L=stem, **case)
    errs, st, sol = parity.run_side_by_side(p, 3)
    bad = {k: max(v) for k, v in errs.items() if k not in ("conv_rel_sig", "conv_flag_mismatch")
           and max(v) > PHASE_TOL}
    assert not bad, bad
    assert "conv_flag_mismatch" not in errs
    sol.close()


def test_dga_with_pa_constants_is_bit_identical(gpu_lib, tmp_path):
    """Lambda files holding the PA constants reproduce the PA loop bit for bit."""
    from tups_b200 import Solver
    p = O.Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=10)
    st = O.initialize(p)
    stem = str(tmp_path / "pa")
    write_dga_files(stem, st.tables["L"])
    pd = O.Params(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=10,
                  DGA=True, fname_L=stem)
    a = Solver(parity.to_solver_params(p))
    b = Solver(parity.to_solver_params(pd))
    for r in "dmst":
        assert np.array_equal(a.F(r), b.F(r)), r
    for ite in range(4):
        a.iteration(ite)
        b.iteration(ite)
    assert np.array_equal(a.Sigma, b.Sigma)
    for r in "dmst":
        assert np.array_equal(a.F(r), b.F(r)), r
    a.close()
    b.close()


def test_dga_missing_file_is_an_error(gpu_lib, tmp_path):
    from tups_b200 import Solver, TupsError
    p = O.Params(Nx=4, Nf=8, neighbours=1, DGA=True, fname_L=str(tmp_path / "absent"))
    with pytest.raises(TupsError):
        Solver(parity.to_solver_params(p))

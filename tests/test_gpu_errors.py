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

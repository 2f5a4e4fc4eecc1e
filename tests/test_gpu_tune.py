"""The tile-shape tuner: its choice is never slower than the fixed default in
its own timings, and tuned iterations write the same bits as iterations on
the default tiles (the candidates differ only in how elements are spread
over CTAs and warps, not in any sum's order)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [
    dict(Nx=4, Nf=34, neighbours=1),    # Nl = 1: Nz = 34, flat 8-column crossing tiles
    dict(Nx=4, Nf=10, neighbours=2),    # Nl = 5: Nz = 50
    dict(Nx=8, Nf=6, neighbours=3),     # Nl = 9: Nz = 54, the 81-column tiles
], ids=["nl1", "nl5", "nl9"])
def test_tuned_tiles_equal_default_tiles(gpu_lib, case):
    from tups_b200 import Params, Solver
    from tups_b200.parquet import tuning_table
    p = Params(beta=3.0, U=2.0, nParticle=0.95, f_damping=0.5, ite_max=10, **case)
    out = {}
    for tuned in (False, True):
        sol = Solver(p)
        sol.set_autotune(tuned)
        for ite in range(3):
            sol.iteration(ite)
        out[tuned] = (sol.Sigma, [sol.F(r) for r in "dmst"], [sol.G(r) for r in "dmst"], sol.mu)
        Nz, Nl = sol.Nz, sol.Nl
        sol.close()
    a, b = out[False], out[True]
    assert np.array_equal(a[0], b[0]) and a[3] == b[3]
    for r in range(4):
        assert np.array_equal(a[1][r], b[1][r]) and np.array_equal(a[2][r], b[2][r]), r
    table = tuning_table()
    keys = {ln.split(" | ")[0]: ln for ln in table}
    pae = [k for k in keys if k.startswith((f"k_pae_mma Nl={Nl} Nf={p.Nf} ", f"k_pae_mma(3M) Nl={Nl} Nf={p.Nf} "))]
    bse = f"k_bse_gemm Nz={Nz}"
    assert pae and bse in keys, table
    for k in (pae[0], bse):
        fields = keys[k].split(" | ")
        choice = fields[1].split()[1]
        ms = dict(kv.split("=") for kv in fields[2].split())
        names = list(ms)
        assert all(float(v) > 0 for v in ms.values())
        # the pick is the fastest candidate, so never slower than the default (index 0)
        assert float(ms[choice]) <= float(ms[names[0]])
        assert float(ms[choice]) == min(float(v) for v in ms.values())


@pytest.mark.parametrize("case", [
    dict(Nx=4, Nf=10, neighbours=2),    # Nl = 5
    dict(Nx=8, Nf=6, neighbours=3),     # Nl = 9
], ids=["nl5", "nl9"])
def test_every_crossing_candidate_writes_the_same_bits(gpu_lib, case):
    """Each three-product crossing candidate (names from the tuner's own
    table), fixed by name, against the first: the same F after two full
    iterations and a third crossing."""
    from tups_b200 import Params, Solver
    from tups_b200.parquet import set_tuning, tuning_table
    p = Params(beta=3.0, U=2.0, nParticle=0.95, f_damping=0.5, ite_max=10, **case)

    def crossing(name):
        set_tuning("k_pae_mma(3M) ", name)
        sol = Solver(p)
        for ite in range(2):
            sol.iteration(ite)
        sol.calc_Gkw_Grt(2, False)
        sol.BSE(2)
        sol.calc_PhiR(2)
        sol.calculate_PAE()
        F = [sol.F(r) for r in "dmst"]
        Nl = sol.Nl
        sol.close()
        return F, Nl

    try:
        ref, Nl = crossing(None)     # tuned: fills the table with every candidate
        line = [ln for ln in tuning_table() if ln.startswith(f"k_pae_mma(3M) Nl={Nl} Nf={p.Nf} ")]
        assert line, tuning_table()
        names = [kv.split("=")[0] for kv in line[0].split(" | ")[2].split()]
        assert len(names) >= 4, names
        for name in names:
            F, _ = crossing(name)
            for r in range(4):
                assert np.array_equal(F[r], ref[r]), (name, r)
    finally:
        set_tuning(None, None)


def test_bse_prep_forms_write_the_same_bits(gpu_lib):
    """The BSE prep as two launches or as one (a tuner choice) gives the
    same vertices after two iterations."""
    from tups_b200 import Params, Solver
    from tups_b200.parquet import set_tuning
    p = Params(beta=3.0, U=2.0, nParticle=0.95, f_damping=0.5, ite_max=10, Nx=8, Nf=6, neighbours=3)
    out = {}
    try:
        for form in ("two_launches", "one_launch"):
            set_tuning("k_bse_prep ", form)
            sol = Solver(p)
            for ite in range(2):
                sol.iteration(ite)
            out[form] = (sol.Sigma, [sol.G(r) for r in "dmst"])
            sol.close()
    finally:
        set_tuning(None, None)
    a, b = out["two_launches"], out["one_launch"]
    assert np.array_equal(a[0], b[0])
    for r in range(4):
        assert np.array_equal(a[1][r], b[1][r]), r

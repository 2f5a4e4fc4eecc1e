"""The reference's output layout (SRC/parquet_plot.f90:68-276): file label,
dataset paths, Fortran shapes seen in C order, complex compound (r, i),
the minus signs of chi_m and the bare bubbles, the output iterations and the
Final datasets; driven by the oracle's loop with its readout."""
from __future__ import annotations

import numpy as np

from oracle import tups_oracle as O
from tups_b200.output import COMPLEX, Output, as_fortran, dataset, kind_label, write_F


def _params(**kw):
    base = dict(beta=2.0, U=2.0, nParticle=0.9, Nx=4, Nf=8, neighbours=2, f_damping=0.5, ite_max=3)
    base.update(kw)
    return O.Params(**base)


def test_kind_label():
    p = O.Params(beta=5.0, U=2.0, nParticle=1.0, Nx=8, Nf=32, neighbours=2, use_U2=True)
    assert kind_label(p, 5) == "NxN0064_Nl0005_Nf0032_U0020_B05_Gr0001_n0100_pa_U2_new_SDEnew"
    q = O.Params(beta=10.0, U=3.0, nParticle=0.29, Nx=16, Nf=64, neighbours=3, use_U2=False, DGA=True)
    # INT truncates: 0.29 * 100 = 28.999999999999996 -> 28
    assert kind_label(q, 9) == "NxN0256_Nl0009_Nf0064_U0030_B10_Gr0001_n0028_new_SDEnew"


def test_dataset_round_trip():
    rng = np.random.default_rng(0)
    a = rng.normal(size=(3, 4, 5)) + 1j * rng.normal(size=(3, 4, 5))
    ds = dataset(a)
    assert ds.dtype == COMPLEX and ds.shape == (5, 4, 3)
    assert ds["r"][2, 1, 0] == a[0, 1, 2].real and ds["i"][2, 1, 0] == a[0, 1, 2].imag
    assert np.array_equal(as_fortran(ds), a)
    r = rng.normal(size=(2, 3))
    assert np.array_equal(as_fortran(dataset(r)), r)


def _oracle_run(p, tmp_path):
    st = O.initialize(p)
    out = Output(tmp_path, p, st.Nl)
    ros = {}
    for ite in range(p.ite_max):
        conv, info = O.iteration(st, ite, with_readout=True)
        if "readout" in info:
            ro = info["readout"]
            ros[ite] = ro
            out.write_sigma(ite, conv, st.Sigma)
            out.write_chis(ite, conv, {r: ro[f"sus_{r}"] for r in "dmst"},
                           {"chi0_ph": ro["chi0_ph_BZ"], "chi0_pp": ro["chi0_pp_BZ"],
                            "chi0_ph_FF": ro["chi0_ph_BZ_FF"], "chi0_pp_FF": ro["chi0_pp_BZ_FF"]})
    return st, out, ros


def test_output_file_layout(tmp_path):
    p = _params()
    st, out, ros = _oracle_run(p, tmp_path)
    assert sorted(ros) == [0, 2]  # ite % 5 == 0 and ite == ite_max - 1
    path = out.save()
    assert path.endswith("TUPS_NxN0016_Nl0005_Nf0008_U0020_B02_Gr0001_n0090_pa_U2_new_SDEnew.npz")
    d = np.load(path)
    nh, nc = p.Nf // 2, p.Nx * p.Nx
    assert float(d["params/beta"]) == 2.0 and int(d["params/Nl"]) == 5 and int(d["params/DGA"]) == 0
    names = ["chi_d", "chi_m", "chi_s", "chi_t", "chi_0", "chi_0_pp", "chi_0_FF", "chi_0_pp_FF"]
    for ite in (0, 2):
        assert d[f"Sigma/sig_{ite:05d}"].shape == (nc, p.Nf) and d[f"Sigma/sig_{ite:05d}"].dtype == COMPLEX
        for n in names:
            assert f"Chi/{n}_{ite:05d}" in d.files
    assert "Sigma/Final/sig" not in d.files  # the reference tests ite == ite_max, never reached
    for n in names:
        assert np.array_equal(d[f"Chi/Final/{n}"], d[f"Chi/{n}_00002"])
    ro = ros[2]
    assert d["Chi/chi_d_00002"].shape == (4, nc, nh)
    assert np.array_equal(as_fortran(d["Chi/chi_m_00002"]),
                          -np.reshape(ro["sus_m"], (nh, nc, 4), order="F"))
    assert np.array_equal(as_fortran(d["Chi/chi_0_00002"]),
                          -np.reshape(ro["chi0_ph_BZ"], (nh, nc), order="F"))
    assert np.array_equal(as_fortran(d["Sigma/sig_00002"]), np.reshape(st.Sigma, (p.Nf, nc), order="F"))


def test_readout_leaves_the_trajectory_alone(tmp_path):
    p = _params()
    st_a, _, _ = _oracle_run(p, tmp_path)
    st_b = O.initialize(p)
    for ite in range(p.ite_max):
        O.iteration(st_b, ite)
    assert np.array_equal(st_a.Sigma, st_b.Sigma) and st_a.mu == st_b.mu


def test_write_F_layout(tmp_path):
    p = _params(save_F=True)
    st = O.initialize(p)
    path = write_F(tmp_path, p, st.Nl, st.Nb, st.F)
    d = np.load(path)
    assert path.endswith("_000.npz")
    for r in "dmst":
        a = as_fortran(d[f"F/F_{r}"])
        assert a.shape == (p.Nf, st.Nl, p.Nf, st.Nl, st.Nb)
        assert np.array_equal(np.reshape(a, st.F[r].shape, order="F"), st.F[r])

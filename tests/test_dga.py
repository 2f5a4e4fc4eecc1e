"""DGA Lambda input on the CPU: the oracle's reader of the reference's file
format (SRC/parquet_util.f90:317-346) and the vertex initialisation from it
(SRC/preprocessing.f90:100-116)."""
from __future__ import annotations

import numpy as np

from oracle import tups_oracle as O
from dga_tables import dga_tables, write_dga_files


def test_lambda_file_round_trip(tmp_path):
    L = dga_tables(8, 2.0, seed=3)
    stem = str(tmp_path / "Lambda")
    write_dga_files(stem, L)
    d, m = O.read_lambda_file(stem + "_ph.init", 8)
    s, t = O.read_lambda_file(stem + "_pp.init", 8)
    for r, v in zip("dmst", (d, m, s, t)):
        assert np.array_equal(v, L[r]), r


def test_lambda_file_list_directed_records(tmp_path):
    """A record may span lines, use commas and Fortran d exponents; items left
    on the record's last line are skipped."""
    Nf = 6
    rows = []
    for k1 in range(Nf):
        for k2 in range(Nf):
            for q in range(Nf // 2):
                v = 100 * k1 + 10 * k2 + q
                if (k1 + k2 + q) % 3 == 0:
                    rows.append(f"{k1 + 1}, {k2 + 1}, {q + 1},")
                    rows.append(f"{v}.5d0 -{v}.25D-1")
                    rows.append(f"  {v}.0 {q}.0d+0  99 98")
                else:
                    rows.append(f"{k1 + 1} {k2 + 1} {q + 1} {v}.5 -{v}.25e-1 {v} {q}")
    path = tmp_path / "L_ph.init"
    path.write_text("\n".join(rows) + "\n")
    A, B = O.read_lambda_file(str(path), Nf)
    for k1 in range(Nf):
        for k2 in range(Nf):
            for q in range(Nf // 2):
                v = 100 * k1 + 10 * k2 + q
                assert A[k1, k2, q] == complex(v + 0.5, float(f"-{v}.25e-1"))
                assert B[k1, k2, q] == complex(v, q)


def test_dga_with_pa_constants_is_the_pa_start(tmp_path):
    """Lambda files holding the PA constants give the PA initial state exactly."""
    p = O.Params(beta=2.0, U=2.0, Nx=4, Nf=8, neighbours=2, f_damping=0.5)
    st = O.initialize(p)
    stem = str(tmp_path / "pa")
    write_dga_files(stem, st.tables["L"])
    pd = O.Params(beta=2.0, U=2.0, Nx=4, Nf=8, neighbours=2, f_damping=0.5, DGA=True, fname_L=stem + "   ")
    sd = O.initialize(pd)
    for r in "dmst":
        assert np.array_equal(sd.F[r], st.F[r]), r
        assert np.array_equal(sd.G[r], st.G[r]), r
        assert np.array_equal(sd.tables["L"][r], st.tables["L"][r]), r


def test_dga_vertex_start_follows_the_bosonic_index(tmp_path):
    """F = G = Lambda(:, :, w) * Nc on the (l=1, l=1) block of each slot, zero elsewhere."""
    Nf = 8
    L = dga_tables(Nf, 2.0, seed=1)
    stem = str(tmp_path / "dga")
    write_dga_files(stem, L)
    p = O.Params(beta=2.0, U=2.0, Nx=4, Nf=Nf, neighbours=2, f_damping=0.5, DGA=True, fname_L=stem)
    st = O.initialize(p)
    aux = st.tables["aux"]
    for iq in range(st.Nb):
        w = int(st.ibz[iq, 2])
        for r in "dmst":
            assert np.array_equal(st.F[r][:Nf, :Nf, iq], L[r][:, :, w - 1] * aux)
            assert not st.F[r][Nf:, :, iq].any() and not st.F[r][:, Nf:, iq].any()


def _native_lambda(stem: str, Nf: int):
    import ctypes as C

    from tups_b200 import _lib
    lib = _lib.load()
    out = [np.zeros((Nf, Nf, Nf // 2), dtype=np.complex128, order="F") for _ in range(4)]
    rc = lib.tups_read_lambda(stem.encode(), Nf, *(C.c_void_p(a.ctypes.data) for a in out))
    return rc, dict(zip("dmst", out))


def test_native_reader_equals_oracle(gpu_lib, tmp_path):
    """The library's reader (tups_read_lambda, the one a DGA context uses)
    and the oracle's read the same files to the same bits."""
    Nf = 8
    stem = str(tmp_path / "Lambda")
    write_dga_files(stem, dga_tables(Nf, 2.0, seed=5))
    rc, L = _native_lambda(stem + "  ", Nf)  # blank-padded as a Fortran string
    assert rc == 0
    d, m = O.read_lambda_file(stem + "_ph.init", Nf)
    s, t = O.read_lambda_file(stem + "_pp.init", Nf)
    for r, v in zip("dmst", (d, m, s, t)):
        assert np.array_equal(L[r], v), r


def test_native_reader_list_directed_records(gpu_lib, tmp_path):
    """Records spanning lines, commas, d exponents and trailing items, as the
    Fortran list-directed read takes them, in the library's reader."""
    Nf = 6
    rows = []
    for k1 in range(Nf):
        for k2 in range(Nf):
            for q in range(Nf // 2):
                v = 100 * k1 + 10 * k2 + q
                if (k1 + k2 + q) % 3 == 0:
                    rows += [f"{k1 + 1}, {k2 + 1}, {q + 1},", f"{v}.5d0 -{v}.25D-1", f"  {v}.0 {q}.0d+0  99 98"]
                else:
                    rows.append(f"{k1 + 1} {k2 + 1} {q + 1} {v}.5 -{v}.25e-1 {v} {q}")
    for suffix in ("_ph.init", "_pp.init"):
        (tmp_path / f"L{suffix}").write_text("\n".join(rows) + "\n")
    rc, L = _native_lambda(str(tmp_path / "L"), Nf)
    assert rc == 0
    A, B = O.read_lambda_file(str(tmp_path / "L_ph.init"), Nf)
    assert np.array_equal(L["d"], A) and np.array_equal(L["m"], B)
    assert np.array_equal(L["s"], A) and np.array_equal(L["t"], B)


def test_native_reader_missing_or_short_file(gpu_lib, tmp_path):
    rc, _ = _native_lambda(str(tmp_path / "absent"), 8)
    assert rc != 0
    (tmp_path / "short_ph.init").write_text("1 1 1 1.0 0.0 1.0 0.0\n")
    (tmp_path / "short_pp.init").write_text("1 1 1 1.0 0.0 1.0 0.0\n")
    rc, _ = _native_lambda(str(tmp_path / "short"), 8)
    assert rc != 0

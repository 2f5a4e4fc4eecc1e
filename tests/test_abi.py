"""CPU tests of the C ABI: the library loads, exports every symbol that
include/tups_b200.h declares, and its host-side code (prms parser, index /
symmetry / form-factor tables) agrees with the oracle without a GPU."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import tups_oracle as O

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"


def declared_symbols() -> list[str]:
    text = (ROOT / "include" / "tups_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tups_[a-zA-Z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(gpu_lib):
    names = declared_symbols()
    assert len(names) > 40
    for n in names:
        assert hasattr(gpu_lib, n), n


def test_binding_covers_header(gpu_lib):
    from tups_b200 import exported_symbols
    assert set(declared_symbols()) <= set(exported_symbols())


def test_strerror(gpu_lib):
    assert gpu_lib.tups_strerror(-3) == b"chemical potential bisection did not converge"
    assert gpu_lib.tups_strerror(0) == b"ok"


@pytest.mark.parametrize("name", ["pa_4x4_nl1", "pa_4x4_nl5"])
def test_native_prms_parser(gpu_lib, name):
    from tups_b200 import read_prms
    p = read_prms(str(GOLD / f"prms_{name}"))
    o = O.read_prms(str(GOLD / f"prms_{name}"))
    for k in ("beta", "U", "nParticle", "Nx", "Nf", "neighbours", "Ngrain", "f_range", "f_damping", "ite_max",
              "use_U2", "oneshot", "old", "SDE_old", "DGA", "pick_file"):
        assert getattr(p, k) == getattr(o, k), k


def test_native_prms_parser_rejects_short_file(gpu_lib, tmp_path):
    from tups_b200 import TupsError, read_prms
    f = tmp_path / "prms"
    f.write_text("5.0d0\n2.0d0\n")
    with pytest.raises(TupsError):
        read_prms(str(f))


@pytest.mark.parametrize("nx,nf,nb", [(4, 16, 1), (4, 8, 2), (8, 32, 2), (8, 16, 3), (16, 64, 3), (16, 8, 4)])
def test_host_tables_bit_exact(gpu_lib, nx, nf, nb):
    """Integer tables equal; form factors equal to the last bit (same libm)."""
    from tups_b200 import Params
    from tups_b200.parquet import host_tables
    t = host_tables(Params(Nx=nx, Nf=nf, neighbours=nb))
    st = O.initialize(O.Params(Nx=nx, Nf=nf, neighbours=nb))
    d = t["dims"]
    for k in ("Nl", "Nz", "Nred", "NIBZ", "NR", "Nt"):
        assert d[k] == getattr(st, k), k
    assert np.array_equal(t["signs"], st.signs)
    assert np.array_equal(t["reps"], st.reps)
    assert np.array_equal(t["lsym"], st.lsym)
    assert np.array_equal(t["lfac"], st.lfac)
    assert np.array_equal(t["ibz"], st.ibz)
    assert np.array_equal(t["FF"], st.FF)
    assert np.array_equal(t["FF_inv"], st.FF_inv)


def test_host_tables_reject_bad_sizes(gpu_lib):
    from tups_b200 import Params, TupsError
    from tups_b200.parquet import host_tables
    with pytest.raises(TupsError):
        host_tables(Params(Nx=5, Nf=16))
    with pytest.raises(TupsError):
        host_tables(Params(Nx=4, Nf=15))
    with pytest.raises(TupsError):
        host_tables(Params(Nx=4, Nf=16, old=True))


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++17")])
def test_header_compiles_on_its_own(lang, std):
    """A C or C++ host includes include/tups_b200.h with nothing before it."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") if lang == "c" else shutil.which("g++")
    if cc is None:
        pytest.skip("no host compiler")
    hdr = Path(__file__).resolve().parents[1] / "include" / "tups_b200.h"
    r = subprocess.run([cc, "-fsyntax-only", "-Wall", "-Wextra", "-Werror", std, "-x", lang, str(hdr)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_host_links_and_reads_prms(gpu_lib, tmp_path):
    """A C program linked against libtups_b200.so parses a prms file and gets
    the derived sizes from the host tables, as a compiled host would (no GPU
    needed for these two calls)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no host compiler")
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "host.c"
    src.write_text(
        '#include <stdio.h>\n#include "tups_b200.h"\n'
        "int main(int argc, char** argv) {\n"
        "  tups_params p; tups_dims d;\n"
        "  int rc = tups_read_prms(argv[1], &p);\n"
        "  if (!rc) rc = tups_host_tables(&p, &d, 0, 0, 0, 0, 0, 0, 0);\n"
        "  if (rc) { printf(\"error %d %s\\n\", rc, tups_strerror(rc)); return 1; }\n"
        '  printf("%d %d %d %d %d\\n", d.Nl, d.Nz, d.Nred, d.NIBZ, d.NR);\n'
        "  return 0;\n}\n")
    exe = tmp_path / "host"
    lib_dir = root / "tups_b200"
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", f"-I{root / 'include'}", str(src), f"-L{lib_dir}",
                        "-ltups_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for name in ("pa_4x4_nl1", "pa_4x4_nl5"):
        out = subprocess.run([str(exe), str(GOLD / f"prms_{name}")], capture_output=True, text=True, timeout=60)
        assert out.returncode == 0, out.stdout + out.stderr
        st = O.initialize(O.read_prms(str(GOLD / f"prms_{name}")))
        assert [int(x) for x in out.stdout.split()] == [st.Nl, st.Nz, st.Nred, st.NIBZ, st.NR]

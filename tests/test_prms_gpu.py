"""The optional `<prms>.gpu` file of extension keys beside the reference's
21-record prms (tprime, conv_abs), read alike by the native parser and the
oracle; the reference's prms stays valid as it is."""
from __future__ import annotations

from pathlib import Path

import pytest

from oracle import tups_oracle as O

GOLD = Path(__file__).resolve().parent / "golden"


def _copy_prms(tmp_path, name="prms_pa_4x4_nl5"):
    p = tmp_path / "prms"
    p.write_text((GOLD / name).read_text())
    return p


def test_absent_extensions_are_zero(gpu_lib, tmp_path):
    from tups_b200 import read_prms
    p = _copy_prms(tmp_path)
    assert read_prms(str(p)).tprime == 0.0 and read_prms(str(p)).conv_abs == 0.0
    o = O.read_prms(str(p))
    assert o.tprime == 0.0 and o.conv_abs == 0.0


def test_extensions_read_by_both_parsers(gpu_lib, tmp_path):
    from tups_b200 import read_prms
    p = _copy_prms(tmp_path)
    (tmp_path / "prms.gpu").write_text("! t' hopping\ntprime = -0.2d0\n\n  CONV_ABS 1.0e-10  # dSigma threshold\n")
    n = read_prms(str(p))
    o = O.read_prms(str(p))
    assert n.tprime == -0.2 and n.conv_abs == 1e-10
    assert o.tprime == -0.2 and o.conv_abs == 1e-10
    ref = O.read_prms(str(GOLD / "prms_pa_4x4_nl5"))
    for f in ("beta", "U", "nParticle", "Nx", "Nf", "neighbours", "ite_max", "f_damping"):
        assert getattr(n, f) == getattr(ref, f) == getattr(o, f), f
    # keyword values take precedence over the file
    assert read_prms(str(p), tprime=0.1).tprime == 0.1
    assert O.read_prms(str(p), conv_abs=0.0).conv_abs == 0.0


@pytest.mark.parametrize("text", ["tprim = -0.2\n", "tprime = abc\n", "tprime -0.2 extra\n", "conv_abs\n"])
def test_bad_extension_lines_are_errors(gpu_lib, tmp_path, text):
    from tups_b200 import TupsError, read_prms
    p = _copy_prms(tmp_path)
    (tmp_path / "prms.gpu").write_text(text)
    with pytest.raises(TupsError):
        read_prms(str(p))
    with pytest.raises(ValueError):
        O.read_prms(str(p))

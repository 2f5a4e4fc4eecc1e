"""Numpy FP64 restatement of the TUPS parquet loop (the oracle).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py`` may import this module; the product library
(``tups_b200``) never does.

Parity status: *unpinned*.  The reference (Fortran 90 + MKL + HDF5 + MPI)
ships no golden vectors and cannot be compiled in this image (no Fortran
compiler).  This module restates it function by function; every function
cites the reference file:line it follows.  It is pinned only by the
reference's own inline known-answer checks (``FF_sdwave_check``,
form-factor orthogonality, ``check_chi0``) and by physics invariants (U = 0,
second order, point-group, particle-hole and conjugation symmetry), see
``tests/test_oracle.py``.

Array conventions follow the reference exactly, with 0-based indices:

* vertex arrays ``F_r, G_r``: shape (Nz, Nz, Nb), Fortran order; element
  [(l, nu), (l', nu'), q] sits at row ``l*Nf + nu``;
* ``Sigma``, ``Gkw``: shape (Nt,), index ``(kx*Ny + ky)*Nf + nu``;
* ``Grt``: shape (Nx*Ng, Ny*Ng, Nf);
* ``PhiR_r``: shape (Nz*Nz, Nf/2, NR) (== PhiRWork(Nz, Nz, wperTask, NR));
* ``M_*``: shape (Nl, Nl, Nl, Nl, Nb, NR).

The reference runs with one MPI task here, so ``Nb = Nred``,
``wperTask = Nf/2`` and ``id = 0`` throughout.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

NS = 8  # parquet_ini.f90:23
# parquet_chi.f90:120 compares against the single-precision literal 1e-6.
MU_TOL = float(np.float32(1e-6))
# parquet_ini.f90:31-32: real(1e-8, 8) converts a single-precision literal.
F_SIGMA = float(np.float32(1e-8))
F_VERT = float(np.float32(1e-8))

# character table, parquet_formfactors.f90:572-588; CHAR_TABLE[i, rep] for
# symmetry i (0..7) and representation column rep (0..4)
CHAR_TABLE = np.array([[1, 1, 1, 1, 1, 1, 1, 1],
                       [1, -1, -1, 1, -1, 1, -1, 1],
                       [1, 1, 1, 1, -1, -1, -1, -1],
                       [1, -1, -1, 1, 1, -1, 1, -1],
                       [2, 0, 0, -2, 0, 0, 0, 0]], dtype=np.int64).T


# --------------------------------------------------------------------------
# input: the 21-line prms file, parquet_ini.f90:289-374
# --------------------------------------------------------------------------
@dataclass
class Params:
    beta: float = 2.0
    U: float = 2.0
    nParticle: float = 1.0
    Nx: int = 4
    Nf: int = 16
    neighbours: int = 1
    readinpick: bool = False
    pick_file: str = ""
    Ngrain: int = 1
    f_range: int = 0
    f_damping: float = 0.5
    ite_max: int = 10
    DGA: bool = False
    fname_L: str = ""
    use_sig_dmft: bool = False
    fname_sig_dmft: str = ""
    use_U2: bool = True
    save_F: bool = False
    oneshot: bool = False
    old: bool = False
    SDE_old: bool = False
    # extension (parquet_ini.f90:24 hard-codes tprime = 0 and never reads it):
    # next-nearest-neighbour hopping added as -4 t' cos kx cos ky
    tprime: float = 0.0
    # extension: absolute sup-norm threshold on the self-energy change;
    # 0 disables it and leaves the reference's relative test alone
    conv_abs: float = 0.0


def _fortran_token(line: str) -> str:
    """First list-directed item of a record (quoted string or bare token)."""
    s = line.strip()
    if s[:1] in "\"'":
        q = s[0]
        end = s.find(q, 1)
        return s[1:end] if end > 0 else s[1:]
    return re.split(r"[\s,/]+", s)[0]


def _f_real(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


def _f_logical(tok: str) -> bool:
    t = tok.lstrip(".").upper()
    if t.startswith("T"):
        return True
    if t.startswith("F"):
        return False
    raise ValueError(f"not a Fortran logical: {tok!r}")


def read_prms_extras(path: str) -> dict:
    """The optional ``<prms>.gpu`` file beside the reference's prms (no
    counterpart in the reference): ``key = value`` lines, ``!`` or ``#``
    comments, keys tprime and conv_abs; an unknown key or a bad value raises."""
    out = {"tprime": 0.0, "conv_abs": 0.0}
    if not os.path.exists(path):
        return out
    with open(path) as fh:
        for ln in fh.read().splitlines():
            for c in "!#":
                ln = ln.split(c, 1)[0]
            f = ln.replace("=", " ").split()
            if not f:
                continue
            if len(f) != 2 or f[0].lower() not in out:
                raise ValueError(f"{path}: bad line {ln!r}")
            out[f[0].lower()] = _f_real(f[1])
    return out


def read_prms(path: str, tprime: float | None = None, conv_abs: float | None = None) -> Params:
    """``set_parameters`` (parquet_ini.f90:289-324): one item per record;
    ``<path>.gpu`` (``read_prms_extras``) for t' and conv_abs, which keyword
    values given here override."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines()]
    lines = [ln for ln in lines if ln.strip()]
    if len(lines) < 21:
        raise ValueError(f"prms file {path} has {len(lines)} records, needs 21")
    tok = [_fortran_token(ln) for ln in lines[:21]]
    ext = read_prms_extras(str(path) + ".gpu")
    return Params(beta=_f_real(tok[0]), U=_f_real(tok[1]), nParticle=_f_real(tok[2]),
                  Nx=int(tok[3]), Nf=int(tok[4]), neighbours=int(tok[5]),
                  readinpick=_f_logical(tok[6]), pick_file=tok[7], Ngrain=int(tok[8]),
                  f_range=int(tok[9]), f_damping=_f_real(tok[10]), ite_max=int(tok[11]),
                  DGA=_f_logical(tok[12]), fname_L=tok[13], use_sig_dmft=_f_logical(tok[14]),
                  fname_sig_dmft=tok[15], use_U2=_f_logical(tok[16]), save_F=_f_logical(tok[17]),
                  oneshot=_f_logical(tok[18]), old=_f_logical(tok[19]), SDE_old=_f_logical(tok[20]),
                  tprime=ext["tprime"] if tprime is None else tprime,
                  conv_abs=ext["conv_abs"] if conv_abs is None else conv_abs)


# --------------------------------------------------------------------------
# form factors, parquet_formfactors.f90
# --------------------------------------------------------------------------
def create_list(Nx: int) -> np.ndarray:
    """``create_list``+``sort`` (parquet_formfactors.f90:594-646); stable
    insertion sort of IBZ lattice points by squared length."""
    pts = []
    for i in range(1, Nx // 2 + 2):
        for j in range(1, i + 1):
            pts.append([i - 1, j - 1, (i - 1) ** 2 + (j - 1) ** 2])
    many = len(pts)
    for i in range(1, many + 1):
        for j in range(i, 1, -1):
            if pts[j - 1][2] < pts[j - 2][2]:
                pts[j - 2], pts[j - 1] = pts[j - 1], pts[j - 2]
    return np.array(pts, dtype=np.int64)  # rows = (x, y, r^2)


def init_nl(p: Params, thelist: np.ndarray) -> tuple[int, np.ndarray]:
    """``Init_Formfactor_variables`` (parquet_formfactors.f90:451-537)."""
    Nx, Ny = p.Nx, p.Nx
    npos = Nx * Ny
    if p.readinpick:
        with open(p.pick_file) as fh:
            vals = [_f_logical(_fortran_token(ln)) for ln in fh.read().splitlines() if ln.strip()]
        pick = np.array(vals[:npos], dtype=bool)
        return int(pick.sum()), pick
    Nl = 0
    for i in range(p.neighbours):
        x, y = thelist[i, 0], thelist[i, 1]
        if x == 0 and y == 0:
            Nl += 1
        elif abs(x - Nx / 2.0) < 0.01 and abs(y - Ny / 2.0) < 0.01:
            Nl += 1
        elif abs(x - Nx / 2.0) < 0.01 and y == 0:
            Nl += 2
        elif abs(x - Nx / 2.0) < 0.01:
            Nl += 4
        elif x == y or y == 0:
            Nl += 4
        else:
            Nl += 8
    pick = np.zeros(npos, dtype=bool)
    pick[:Nl] = True
    return Nl, pick


def initialize_bonds(Nx: int, Nl: int, thelist, pick):
    """``initialize_bonds`` (parquet_formfactors.f90:95-360).

    Returns bond0 (Nl, 3) = (bx, by, character column 1..5), signs, reps."""
    Ny = Nx
    bonds = np.zeros((Nl, 3), dtype=np.int64)
    signs = np.ones(Nl, dtype=np.int64)
    reps = np.zeros(Nl, dtype=np.int64)
    chars_41 = [1, 4, 5, 5]
    chars_42 = [1, 3, 5, 5]
    chars_8 = [1, 2, 3, 4, 5, 5, 5, 5]
    st = {"b": 1, "log": 1}

    def put(bx, by, ch, rep, sgn=None):
        b = st["b"]
        bonds[b - 1] = (bx, by, ch)
        reps[b - 1] = rep
        if sgn is not None:
            signs[b - 1] = sgn
        st["b"] = b + 1
        return st["b"] > Nl

    lat = 1
    while True:
        x, y = int(thelist[lat - 1, 0]), int(thelist[lat - 1, 1])
        if x == 0 and y == 0:
            if pick[st["log"] - 1]:
                if put(x, y, 1, 1):
                    break
            st["log"] += 1
            lat += 1
            continue
        elif abs(x - Nx / 2.0) < 0.01 and abs(y - Ny / 2.0) < 0.01:
            if pick[st["log"] - 1]:
                if put(x, y, 1, 1):
                    break
            st["log"] += 1
            lat += 1
            continue
        elif abs(x - Nx / 2.0) < 0.01 and y == 0:
            if pick[st["log"] - 1]:
                if put(x, y, 1, 1):
                    break
            st["log"] += 1
            if pick[st["log"] - 1]:
                if put(x, y, 3, 3):
                    break
            st["log"] += 1
            lat += 1
            continue
        elif x == y:
            done = False
            for i in range(1, 4):
                if pick[st["log"] - 1]:
                    if put(x, y, chars_41[i - 1], chars_41[i - 1], -1 if i == 3 else None):
                        done = True
                        break
                st["log"] += 1
            if done:
                break
            if pick[st["log"] - 1]:
                if put(-y, x, chars_41[3], 6, -1):
                    break
            st["log"] += 1
            lat += 1
            continue
        elif y == 0 or abs(x - Nx / 2.0) < 0.01:
            done = False
            for i in range(1, 4):
                if pick[st["log"] - 1]:
                    if put(x, y, chars_42[i - 1], chars_42[i - 1], -1 if i == 3 else None):
                        done = True
                        break
                st["log"] += 1
            if done:
                break
            # the DO variable is 4 after normal loop completion (chars_42(4) = 5)
            if pick[st["log"] - 1]:
                if put(-y, x, chars_42[3], 6, -1):
                    break
            st["log"] += 1
            lat += 1
            continue
        else:
            done = False
            for i in range(1, 6):
                if pick[st["log"] - 1]:
                    if put(x, y, chars_8[i - 1], chars_8[i - 1], -1 if i == 5 else None):
                        done = True
                        break
                st["log"] += 1
            if done:
                break
            if pick[st["log"] - 1]:
                if put(x, -y, chars_8[5], 6, -1):
                    break
            st["log"] += 1
            if pick[st["log"] - 1]:
                if put(y, x, chars_8[6], 5, -1):
                    break
            st["log"] += 1
            if pick[st["log"] - 1]:
                if put(-y, x, chars_8[7], 6, -1):
                    break
            st["log"] += 1
            lat += 1
            continue
    return bonds, signs, reps


def my_symmetry_operation(i_sym: int, x: int, y: int) -> tuple[int, int]:
    """``my_symmetry_operation`` (parquet_formfactors.f90:367-446), no wrap."""
    return {1: (x, y), 2: (x, -y), 3: (-x, y), 4: (-x, -y), 5: (y, x),
            6: (y, -x), 7: (-y, -x), 8: (-y, x)}[i_sym]


def _wrap_neg(i: int, N: int) -> int:
    """1-based index of -k: mod(-(i-1)+N, N)+1 (parquet_util.f90:928)."""
    return (-(i - 1) + N) % N + 1


def symmetry_operation(i_sym: int, ix: int, iy: int, Nx: int) -> tuple[int, int]:
    """``symmetry_operation`` (parquet_util.f90:896-978) on 1-based (ix, iy)."""
    Ny = Nx
    if i_sym == 1:
        return ix, iy
    if i_sym == 2:
        return ix, _wrap_neg(iy, Ny)
    if i_sym == 3:
        return _wrap_neg(ix, Nx), iy
    if i_sym == 4:
        return _wrap_neg(ix, Nx), _wrap_neg(iy, Ny)
    if i_sym == 5:
        return iy, ix
    if i_sym == 6:
        return iy, _wrap_neg(ix, Nx)
    if i_sym == 7:
        return _wrap_neg(iy, Ny), _wrap_neg(ix, Nx)
    return _wrap_neg(iy, Ny), ix


def symmetry_operation_inv(i_sym: int, ix: int, iy: int, Nx: int) -> tuple[int, int]:
    """``symmetry_operation_inv`` (parquet_util.f90:982-1136) and its copy
    ``my_symmetry_operation_inv`` (parquet_formfactors.f90:651-789): 6 and 8
    are swapped relative to the forward operation."""
    if i_sym == 6:
        return symmetry_operation(8, ix, iy, Nx)
    if i_sym == 8:
        return symmetry_operation(6, ix, iy, Nx)
    return symmetry_operation(i_sym, ix, iy, Nx)


def ff_array(Nx: int, Nl: int, bonds0: np.ndarray) -> np.ndarray:
    """``FF_array`` (parquet_formfactors.f90:11-90): FF(kx, ky, l), real."""
    Ny = Nx
    bx = np.zeros((8, Nl), dtype=np.int64)
    by = np.zeros((8, Nl), dtype=np.int64)
    bw = np.zeros((8, Nl), dtype=np.int64)
    for l in range(Nl):
        x0, y0, ch = bonds0[l]
        for i in range(1, 9):
            bx[i - 1, l], by[i - 1, l] = my_symmetry_operation(i, int(x0), int(y0))
            bw[i - 1, l] = CHAR_TABLE[i - 1, ch - 1]
    ffc = np.zeros((Nx, Ny, Nl), dtype=np.complex128)
    for l in range(Nl):
        for kx in range(1, Nx + 1):
            for ky in range(1, Ny + 1):
                acc = 0j
                for i in range(8):
                    px = 2.0 / Nx * math.pi * (kx - 1)
                    py = 2.0 / Ny * math.pi * (ky - 1)
                    ang = bx[i, l] * px + by[i, l] * py
                    acc = acc + bw[i, l] * complex(math.cos(ang), math.sin(ang))
                ffc[kx - 1, ky - 1, l] = acc
    FF = np.zeros((Nx, Ny, Nl))
    for l in range(Nl):
        norm = 0.0
        for kx in range(Nx):
            for ky in range(Ny):
                a = abs(ffc[kx, ky, l])
                norm += a * a
        inv = 1.0 / math.sqrt(norm)
        FF[:, :, l] = inv * ffc[:, :, l].real + inv * ffc[:, :, l].imag
    return FF


def init_ff_inv(FF: np.ndarray) -> np.ndarray:
    """``init_FF_inv`` (parquet_formfactors.f90:545-569): FF_inv(s, kx, ky, l)."""
    Nx, Ny, Nl = FF.shape
    out = np.zeros((NS, Nx, Ny, Nl))
    for s in range(1, NS + 1):
        for kx in range(1, Nx + 1):
            for ky in range(1, Ny + 1):
                sx, sy = symmetry_operation_inv(s, kx, ky, Nx)
                out[s - 1, kx - 1, ky - 1, :] = FF[sx - 1, sy - 1, :]
    return out


def fill_ff_sdwave(Nx: int) -> np.ndarray:
    """``fill_FF_sdwave`` (parquet_formfactors.f90:792-816)."""
    out = np.zeros((Nx, Nx, 4))
    out[:, :, 0] = 1.0
    for ky in range(1, Nx + 1):
        for kx in range(1, Nx + 1):
            px = 2.0 / Nx * math.pi * (kx - 1)
            py = 2.0 / Nx * math.pi * (ky - 1)
            out[kx - 1, ky - 1, 1] = math.cos(px) - math.cos(py)
            out[kx - 1, ky - 1, 2] = math.sin(px)
            out[kx - 1, ky - 1, 3] = math.sin(px) * math.sin(py)
    return out


def ff_sdwave_check(FF: np.ndarray, Nx: int) -> float:
    """``FF_sdwave_check`` (parquet_check.f90:264-292): returns check_zero."""
    sd = fill_ff_sdwave(Nx)
    Nl = FF.shape[2]
    cz = float(np.sum(np.abs(FF[:, :, 0] - 1.0 / Nx * sd[:, :, 0])))
    if Nl > 1:
        cz += float(np.sum(np.abs(FF[:, :, 2] - 1.0 / Nx * sd[:, :, 1])))
        cz += float(np.sum(np.abs(FF[:, :, 3] - math.sqrt(2.0) / Nx * sd[:, :, 2])))
    return cz


def sym_op_L(is_: int, l_in: int, reps: np.ndarray, char_table=CHAR_TABLE) -> tuple[int, float]:
    """``sym_op_L`` (parquet_util.f90:732-890); 1-based l.  Returns (l_sym, fac)."""
    rep = int(reps[l_in - 1])
    if 1 <= rep <= 4:
        return l_in, float(char_table[is_ - 1, rep - 1])
    if rep == 5:
        if l_in <= 5:
            l_sym = l_in if is_ <= 4 else l_in + 1
            fac = {1: 1, 2: 1, 3: -1, 4: -1, 5: 1, 6: 1, 7: -1, 8: -1}[is_]
            return l_sym, float(fac)
        tab = {1: (1, 0), 2: (-1, 1), 3: (1, 1), 4: (-1, 0),
               5: (1, 0), 6: (1, 1), 7: (-1, 0), 8: (-1, 1)}
        f, d = tab[is_]
        return l_in + d, float(f)
    if rep == 6:
        if l_in <= 5:
            l_sym = l_in if is_ <= 4 else l_in - 1
            fac = {1: 1, 2: -1, 3: 1, 4: -1, 5: 1, 6: -1, 7: -1, 8: 1}[is_]
            return l_sym, float(fac)
        tab = {1: (1, 0), 2: (-1, -1), 3: (1, -1), 4: (-1, 0),
               5: (-1, 0), 6: (-1, -1), 7: (1, 0), 8: (1, -1)}
        f, d = tab[is_]
        return l_in + d, float(f)
    raise ValueError(f"representation {rep} has no l-space symmetry rule")


def list_symmetries(kx: int, ky: int, Nx_IBZ: int) -> list[bool]:
    """``list_symmetries`` (parquet_util.f90:1140-1207); 1-based IBZ point."""
    s = [False] * NS
    if (kx == 1 and ky == 1) or (kx == Nx_IBZ and ky == Nx_IBZ):
        s[0] = True
    elif kx == Nx_IBZ and ky == 1:
        s[0] = s[4] = True
    elif kx == Nx_IBZ and 1 < ky < Nx_IBZ:
        s[0] = s[1] = s[4] = s[7] = True
    elif kx > 1 and ky < Nx_IBZ:
        if ky == 1:
            s[0] = s[2] = s[4] = s[5] = True
        elif ky == kx:
            s[0] = s[1] = s[2] = s[3] = True
        else:
            s = [True] * NS
    return s


# --------------------------------------------------------------------------
# the state of one solver instance (parquet_ini.f90:67-285 module globals)
# --------------------------------------------------------------------------
@dataclass
class State:
    p: Params
    Nx: int = 0
    Ny: int = 0
    Nf: int = 0
    Ng: int = 1
    Nx_IBZ: int = 0
    NIBZ: int = 0
    Nred: int = 0
    Nc: int = 0
    Nl: int = 0
    Nz: int = 0
    Nt: int = 0
    Nb: int = 0
    NR: int = 1
    mu: float = 0.0
    tables: dict = field(default_factory=dict)
    arrays: dict = field(default_factory=dict)

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays", {})
        if name in arrays:
            return arrays[name]
        tables = self.__dict__.get("tables", {})
        if name in tables:
            return tables[name]
        raise AttributeError(name)


def freq(st: State, iw):
    """``get_freq`` (parquet_util.f90:1332-1339), 1-based iw (any integer)."""
    iw = np.asarray(iw)
    return 1j * (math.pi / st.p.beta * (2.0 * (iw - st.Nf // 2 - 1) + 1.0))


def read_lambda_file(path: str, Nf: int) -> tuple[np.ndarray, np.ndarray]:
    """DGA Lambda input (parquet_util.f90:321-343): records in the order k1
    (slowest), k2, q (fastest), each a list-directed read of
    ``i i i re1 im1 re2 im2`` (a record may span lines; items left on its last
    line are skipped).  Returns the two (Nf, Nf, Nf/2) tables."""
    A = np.zeros((Nf, Nf, Nf // 2), dtype=np.complex128)
    B = np.zeros_like(A)
    with open(path) as fh:
        lines = iter(fh.read().splitlines())
        for k1 in range(Nf):
            for k2 in range(Nf):
                for q in range(Nf // 2):
                    tok: list[str] = []
                    while len(tok) < 7:
                        tok += next(lines).replace(",", " ").split()
                    for t in tok[:3]:
                        int(t)  # integer labels, read and dropped as in the reference
                    v = [_f_real(t) for t in tok[3:7]]
                    A[k1, k2, q] = complex(v[0], v[1])
                    B[k1, k2, q] = complex(v[2], v[3])
    return A, B


def write_lambda_file(path: str, A: np.ndarray, B: np.ndarray) -> None:
    """Writes two (Nf, Nf, Nf/2) tables in the record order of
    ``read_lambda_file``, one record per line, 17 significant digits."""
    Nf = A.shape[0]
    with open(path, "w") as fh:
        for k1 in range(Nf):
            for k2 in range(Nf):
                for q in range(Nf // 2):
                    a, b = A[k1, k2, q], B[k1, k2, q]
                    fh.write(f"{k1 + 1} {k2 + 1} {q + 1} {a.real:.17e} {a.imag:.17e} {b.real:.17e} {b.imag:.17e}\n")


def initialize(p: Params, vertices: bool = True) -> State:
    """``set_parameters`` derived sizes (parquet_ini.f90:326-349),
    ``Initialization`` (parquet_util.f90:14-478), ``FF_array`` and the
    vertex initialisation of ``do_preprocessing`` (preprocessing.f90:100-133).

    vertices=False skips the (Nz, Nz, Nb) vertex arrays (61 GB on the 16x16 /
    9 form factor / 64 frequency grid), for the slot-restricted functions
    ``bse_slot``, ``phir_at_w`` and ``crossing_slot``."""
    if p.Nf % 2:
        raise ValueError("Nf must be even")
    if p.old or p.SDE_old:
        raise NotImplementedError("old PAE/SDE paths are outside the hot path")
    st = State(p=p)
    st.Nx = st.Ny = p.Nx
    st.Nf = p.Nf
    st.Ng = p.Ngrain
    st.Nx_IBZ = (p.Nx + 2) // 2
    st.NIBZ = (st.Nx_IBZ * (st.Nx_IBZ + 1)) // 2
    st.Nred = st.NIBZ * p.Nf // 2
    st.Nc = p.Nx * p.Nx
    st.Nt = p.Nx * p.Nx * p.Nf
    st.Nb = st.Nred
    thelist = create_list(p.Nx)
    st.Nl, pick = init_nl(p, thelist)
    st.Nz = st.Nl * st.Nf
    bonds0, signs, reps = initialize_bonds(p.Nx, st.Nl, thelist, pick)
    FF = ff_array(p.Nx, st.Nl, bonds0)
    # NR rule, preprocessing.f90:127-133
    st.NR = {1: 1, 5: 4, 9: 6}.get(st.Nl, 1)
    if st.NR > st.NIBZ:
        raise ValueError("NR exceeds the number of IBZ lattice vectors")
    Nx, Ny, Nf, Ng = st.Nx, st.Ny, st.Nf, st.Ng
    # index_bosonic_IBZ (parquet_util.f90:110-117)
    ibz = np.zeros((st.Nred, 3), dtype=np.int64)
    for kx in range(1, st.Nx_IBZ + 1):
        for ky in range(1, kx + 1):
            for w in range(1, Nf // 2 + 1):
                idx = (((kx - 1) * kx) // 2 + ky - 1) * (Nf // 2) + w
                ibz[idx - 1] = (kx, ky, w)
    symlist = np.zeros((st.NIBZ, NS), dtype=bool)
    qibz = np.zeros((st.NIBZ, 2), dtype=np.int64)
    for iq in range(st.NIBZ):
        kx, ky, _ = ibz[iq * (Nf // 2)]
        qibz[iq] = (kx, ky)
        symlist[iq] = list_symmetries(int(kx), int(ky), st.Nx_IBZ)
    # sym_op_L tables
    lsym = np.zeros((NS, st.Nl), dtype=np.int64)
    lfac = np.zeros((NS, st.Nl))
    for s in range(1, NS + 1):
        for l in range(1, st.Nl + 1):
            ls, f = sym_op_L(s, l, reps)
            lsym[s - 1, l - 1] = ls
            lfac[s - 1, l - 1] = f
    # dispersion (parquet_util.f90:128-164) plus the t' extension
    Ek = np.zeros((Nx, Ny))
    dkx = 2.0 * math.pi / Nx
    dky = 2.0 * math.pi / Ny
    for kx in range(1, Nx + 1):
        px = dkx * (kx - 1)
        for ky in range(1, Ny + 1):
            py = dky * (ky - 1)
            e = 0.0
            if Nx > 1:
                e = e - 2.0 * math.cos(px)
            if Ny > 1:
                e = e - 2.0 * math.cos(py)
            if p.tprime != 0.0:
                e = e - 4.0 * p.tprime * math.cos(px) * math.cos(py)
            Ek[kx - 1, ky - 1] = e
    if st.Nc == 1:
        Ek[:] = 0.0
    Ekg = np.zeros((Ng, Ng, Nx, Ny))
    for iy in range(1, Ny + 1):
        for ix in range(1, Nx + 1):
            for iy2 in range(1, Ng + 1):
                for ix2 in range(1, Ng + 1):
                    px = dkx * (ix - 1) + (ix2 - (Ng + 1) // 2) * dkx / float(Ng)
                    py = dky * (iy - 1) + (iy2 - (Ng + 1) // 2) * dky / float(Ng)
                    e = 0.0 - 2.0 * math.cos(px) - 2.0 * math.cos(py)
                    if p.tprime != 0.0:
                        e = e - 4.0 * p.tprime * math.cos(px) * math.cos(py)
                    Ekg[ix2 - 1, iy2 - 1, ix - 1, iy - 1] = e
    if st.Nc == 1:
        Ekg[:] = 0.0
    st.tables.update(thelist=thelist, pick=pick, bonds0=bonds0, signs=signs, reps=reps,
                     FF=FF, FF_inv=init_ff_inv(FF), ibz=ibz, qibz=qibz, symlist=symlist,
                     lsym=lsym, lfac=lfac, Ek=Ek, Ek_grain=Ekg)
    # self-energy (parquet_util.f90:170-233)
    Sigma = np.zeros(st.Nt, dtype=np.complex128)
    if p.use_sig_dmft:
        with open(p.fname_sig_dmft) as fh:
            rows = [ln.split() for ln in fh.read().splitlines() if ln.strip()]
        sdmft = np.array([complex(0.0, _f_real(r[2])) for r in rows[:Nf]])
        Sigma[:] = np.tile(sdmft, st.Nc)
    # Lambda (parquet_util.f90:302-346)
    U = p.U
    if p.DGA:
        base = p.fname_L.rstrip()
        Ls = {}
        Ls["d"], Ls["m"] = read_lambda_file(base + "_ph.init", Nf)
        Ls["s"], Ls["t"] = read_lambda_file(base + "_pp.init", Nf)
    else:
        Ls = {"d": np.full((Nf, Nf, Nf // 2), U, dtype=np.complex128),
              "m": np.full((Nf, Nf, Nf // 2), -U, dtype=np.complex128),
              "s": np.full((Nf, Nf, Nf // 2), 2.0 * U, dtype=np.complex128),
              "t": np.zeros((Nf, Nf, Nf // 2), dtype=np.complex128)}
    st.tables["L"] = Ls
    # vertex init, preprocessing.f90:100-116
    aux = abs(1.0 / (FF[0, 0, 0] * FF[0, 0, 0]))
    st.tables["aux"] = aux
    F = {}
    G = {}
    q0 = ibz[:, 2] - 1
    for r in "dmst" if vertices else "":
        F[r] = np.zeros((st.Nz, st.Nz, st.Nb), dtype=np.complex128, order="F")
        F[r][:Nf, :Nf, :] = Ls[r][:, :, q0] * aux
        G[r] = F[r].copy(order="F")
    st.arrays.update(Sigma=Sigma, SigmaOld=Sigma.copy(), F=F, G=G,
                     Sigma_H=np.zeros((Nx, Ny), dtype=np.complex128),
                     Gkw=np.zeros(st.Nt, dtype=np.complex128),
                     Grt=np.zeros((Nx * Ng, Ny * Ng, Nf), dtype=np.complex128))
    st.arrays["F_max"] = {r: 0.0 for r in "dmst"}
    st.mu = 0.0
    return st


# --------------------------------------------------------------------------
# MATH_mod.f90
# --------------------------------------------------------------------------
def fftf2d(a: np.ndarray) -> np.ndarray:
    """``fftf2d`` (MATH_mod.f90:215-236): forward 2D DFT (e^{-i}), /n1/n2,
    over the first two axes; dfftpack's zfftf convention (lib/dfftpack/doc:811)."""
    n1, n2 = a.shape[0], a.shape[1]
    return np.fft.fft2(a, axes=(0, 1)) / n1 / n2


def fftb2d(a: np.ndarray) -> np.ndarray:
    """``fftb2d`` (MATH_mod.f90:238-259): backward 2D DFT (e^{+i}),
    unnormalised (lib/dfftpack/doc:858)."""
    n1, n2 = a.shape[0], a.shape[1]
    return np.fft.ifft2(a, axes=(0, 1)) * (n1 * n2)


def fdfit(gt: np.ndarray, dt: float) -> tuple[float, float]:
    """``FDfit`` (MATH_mod.f90:95-107)."""
    L = len(gt)
    fd1 = (-25.0 * gt[0] + 48.0 * gt[1] - 36.0 * gt[2] + 16.0 * gt[3] - 3.0 * gt[4]) / 12.0 / dt
    fd2 = (25.0 * gt[L - 1] - 48.0 * gt[L - 2] + 36.0 * gt[L - 3] - 16.0 * gt[L - 4]
           + 3.0 * gt[L - 5]) / 12.0 / dt
    return fd1, fd2


def nfourier(fermionic: bool, L: int, iwmax: int, fd1: float, fd2: float,
             rin: np.ndarray, beta: float) -> np.ndarray:
    """``nfourier`` (MATH_mod.f90:110-212): cubic-spline tau -> i omega
    transform with clamped end derivatives.  ``rin`` has L+1 points."""
    delta = beta / L
    r = np.asarray(rin, dtype=np.float64)
    q = np.zeros(L + 1)
    u = np.zeros(L + 1)
    xm = np.zeros(L + 1)
    if fd1 > 0.99e30:
        q[0] = 0.0
        u[0] = 0.0
    else:
        q[0] = -0.5
        u[0] = (3.0 / delta) * ((r[1] - r[0]) / delta - fd1)
    for k in range(2, L + 1):
        pp = q[k - 2] / 2.0 + 2.0
        q[k - 1] = -1.0 / 2.0 / pp
        u[k - 1] = 3.0 / delta ** 2 * (r[k] + r[k - 2] - 2.0 * r[k - 1])
        u[k - 1] = (u[k - 1] - u[k - 2] / 2.0) / pp
    if fd2 > 0.99e30:
        q[L] = 0.0
        u[L] = 0.0
    else:
        q[L] = 0.5
        u[L] = (3.0 / delta) * (fd2 - (r[L] - r[L - 1]) / delta)
    xm[L] = (u[L] - q[L] * u[L - 1]) / (q[L] * q[L - 1] + 1.0)
    for k in range(L, 0, -1):
        xm[k - 1] = q[k - 1] * xm[k] + u[k - 1]
    a = r[:L].copy()
    c = xm[:L] / 2.0
    b = (r[1:L + 1] - r[:L]) / delta - (2.0 * xm[:L] + xm[1:L + 1]) * delta / 6.0
    d = (xm[1:L + 1] - xm[:L]) / (6.0 * delta)
    out = np.zeros(iwmax, dtype=np.complex128)
    j = np.arange(1, L + 1)
    for i in range(1, iwmax + 1):
        om = (2.0 * i - 1.0) * math.pi / beta if fermionic else 2.0 * (i - 1) * math.pi / beta
        if abs(om) < 1e-6:
            out[i - 1] = np.sum(a * delta + 0.5 * b * delta * delta + c * delta ** 3 / 3.0
                                + d * delta ** 4 / 4.0)
            continue
        explus = np.exp(1j * om * delta * j)
        ex = np.exp(1j * om * delta * (j - 1))
        t1 = explus * ((-6.0 * d) / om ** 4 + (2.0j * c + 6.0 * delta * 1j * d) / om ** 3
                       + (b + 2.0 * delta * c + 3.0 * delta ** 2 * d) / om ** 2
                       + (-1j * a - delta * 1j * b - delta ** 2 * 1j * c - delta ** 3 * 1j * d) / om)
        t2 = ex * (6.0 * d / om ** 4 - 2.0j * c / om ** 3 - b / om ** 2 + 1j * a / om)
        out[i - 1] = np.sum(t1 + t2)
    return out


# --------------------------------------------------------------------------
# Green's function, parquet_chi.f90:18-210
# --------------------------------------------------------------------------
def _grain_index(k: int, kc: int, N: int, Ng: int) -> int:
    """1-based fine-grid index, parquet_chi.f90:135-139."""
    idx = (k - 1) * Ng + (kc - (Ng + 1) // 2) + 1
    if idx < 1:
        idx += Ng * N
    return idx


def grt_for_mu(st: State, mu: float) -> np.ndarray:
    """G(r, tau) for a given mu: the body of the bisection loop,
    parquet_chi.f90:124-179."""
    p = st.p
    Nx, Ny, Nf, Ng, beta = st.Nx, st.Ny, st.Nf, st.Ng, p.beta
    Sig = st.Sigma.reshape(Nx, Ny, Nf)
    nu = np.arange(1, Nf + 1)
    fr = freq(st, nu)
    tau = beta / (Nf - 1) * (np.arange(1, Nf + 1) - 1)
    # exp(i*(-pi/beta*(2(nu-Nf/2)-1))*tau), parquet_chi.f90:161
    ph = -math.pi / beta * (2.0 * (nu - Nf // 2) - 1.0)
    tw = np.exp(1j * (ph[None, :] * tau[:, None]))  # (tau, nu)
    Grt = np.zeros((Nx * Ng, Ny * Ng, Nf), dtype=np.complex128)
    Ekg = st.Ek_grain
    for ky in range(1, Ny + 1):
        for kx in range(1, Nx + 1):
            for kyc in range(1, Ng + 1):
                for kxc in range(1, Ng + 1):
                    i1 = _grain_index(kx, kxc, Nx, Ng)
                    i2 = _grain_index(ky, kyc, Ny, Ng)
                    e = Ekg[kxc - 1, kyc - 1, kx - 1, ky - 1]
                    gc = 1.0 / (fr + mu - e - Sig[kx - 1, ky - 1, :])
                    d1 = gc - 1.0 / (fr + mu - e)
                    dummy = np.sum((tw * d1[None, :]).real / beta, axis=1)
                    Grt[i1 - 1, i2 - 1, :] = dummy - np.exp((beta - tau) * (e - mu)) / (
                        1.0 + np.exp(beta * (e - mu)))
    return fftf2d(Grt)


def calc_Gkw_Grt(st: State, ite: int, cal_chi: bool, max_steps: int = 1000) -> int:
    """``calc_Gkw_Grt`` without the chi0 readout branch (parquet_chi.f90:18-210).

    Returns the number of bisection steps.  The reference loop has no cap; a
    cap here turns a runaway bisection into an error."""
    p = st.p
    Nx, Ny, Nf = st.Nx, st.Ny, st.Nf
    # Hartree part = Sigma at the last frequency (parquet_chi.f90:105-111)
    Sig = st.Sigma.reshape(Nx, Ny, Nf)
    st.arrays["Sigma_H"] = Sig[:, :, Nf - 1].copy()
    up = st.mu + p.U
    lo = st.mu - p.U
    t1 = 3.0
    steps = 0
    Grt = None
    while abs(t1 - p.nParticle) > MU_TOL:
        if steps >= max_steps:
            raise RuntimeError("chemical potential bisection did not converge")
        st.mu = 0.5 * (up + lo)
        Grt = grt_for_mu(st, st.mu)
        t1 = -2.0 * Grt[0, 0, Nf - 1].real
        steps += 1
        if cal_chi:
            break
        if t1 > p.nParticle:
            up = st.mu
        else:
            lo = st.mu
    if Grt is not None:
        st.arrays["Grt"] = Grt
    # G(k, nu) with the final mu, parquet_chi.f90:203-210
    nu = np.arange(1, Nf + 1)
    fr = freq(st, nu)
    G = 1.0 / (fr[None, None, :] - st.Ek[:, :, None] + st.mu - Sig)
    st.arrays["Gkw"] = G.reshape(-1).copy()
    return steps


def green(st: State, ix, iy, iw):
    """``get_green`` (parquet_util.f90:1278-1299) on arrays of 0-based
    (ix, iy) and 1-based iw."""
    ix = np.asarray(ix)
    iy = np.asarray(iy)
    iw = np.asarray(iw)
    ix, iy, iw = np.broadcast_arrays(ix, iy, iw)
    Nf = st.Nf
    inbox = (iw >= 1) & (iw <= Nf)
    out = np.empty(ix.shape, dtype=np.complex128)
    idx = (ix * st.Ny + iy) * Nf + np.clip(iw, 1, Nf) - 1
    out[inbox] = st.Gkw[idx[inbox]]
    ob = ~inbox
    out[ob] = 1.0 / (freq(st, iw[ob]) - st.Ek[ix[ob], iy[ob]] + st.mu - st.Sigma_H[ix[ob], iy[ob]])
    return out


def green_coarse(st: State, gx, gy, ix, iy, iw):
    """``get_green_coarse`` (parquet_util.f90:1303-1327); 0-based gx, gy, ix,
    iy and 1-based iw."""
    ix, iy, iw, gx, gy = np.broadcast_arrays(np.asarray(ix), np.asarray(iy), np.asarray(iw),
                                             np.asarray(gx), np.asarray(gy))
    Nf = st.Nf
    e = st.Ek_grain[gx, gy, ix, iy]
    inbox = (iw >= 1) & (iw <= Nf)
    sig = np.where(inbox, st.Sigma[(ix * st.Ny + iy) * Nf + np.clip(iw, 1, Nf) - 1],
                   st.Sigma_H[ix, iy])
    return 1.0 / (freq(st, iw) - e + st.mu - sig)


# --------------------------------------------------------------------------
# chi bubble, parquet_chi.f90:438-523
# --------------------------------------------------------------------------
def chi_k(st: State, qx: int, qy: int, w: int) -> tuple[np.ndarray, np.ndarray]:
    """k-space bubbles chi_ph(k, nu), chi_pp(k, nu) for q = (qx, qy, w), 1-based
    (parquet_chi.f90:470-494).  Returns arrays of shape (Nx, Ny, Nf)."""
    Nx, Ny, Nf, Ng = st.Nx, st.Ny, st.Nf, st.Ng
    kx = np.arange(Nx)[:, None, None]
    ky = np.arange(Ny)[None, :, None]
    nu = np.arange(1, Nf + 1)[None, None, :]
    kpqx = (kx + qx - 1) % Nx
    kpqy = (ky + qy - 1) % Ny
    w_kpq = nu + w - 1
    mkx = (-kx + Nx) % Nx
    mky = (-ky + Ny) % Ny
    qmkx = (mkx + qx - 1) % Nx
    qmky = (mky + qy - 1) % Ny
    w_qmk = (-nu + Nf + 1) + w - 1
    cph = np.zeros((Nx, Ny, Nf), dtype=np.complex128)
    cpp = np.zeros((Nx, Ny, Nf), dtype=np.complex128)
    for gx in range(Ng):
        for gy in range(Ng):
            gk = green_coarse(st, gx, gy, kx, ky, nu)
            gkpq = green_coarse(st, gx, gy, kpqx, kpqy, w_kpq)
            cph = cph + gk * gkpq * 1.0 / Ng / Ng
            gqmk = green_coarse(st, Ng - gx - 1, Ng - gy - 1, qmkx, qmky, w_qmk)
            cpp = cpp + gk * gqmk * 1.0 / Ng / Ng
    return cph, cpp


def chi_ll_blocks(st: State, qx: int, qy: int, w: int) -> tuple[np.ndarray, np.ndarray]:
    """The nu-diagonal blocks chi_LL[(l1,nu),(l2,nu)] as (Nf, Nl, Nl) arrays
    (parquet_chi.f90:500-521)."""
    cph, cpp = chi_k(st, qx, qy, w)
    FF = st.FF
    bph = np.einsum("xyn,xya,xyb->nab", cph, FF, FF)
    bpp = np.einsum("xyn,xya,xyb->nab", cpp, FF, FF)
    return bph, bpp


def calc_chi(st: State, qx: int, qy: int, w: int) -> tuple[np.ndarray, np.ndarray]:
    """``calc_chi``: dense (Nz, Nz) chi_ph_LL, chi_pp_LL as the reference stores them."""
    Nl, Nf, Nz = st.Nl, st.Nf, st.Nz
    bph, bpp = chi_ll_blocks(st, qx, qy, w)
    out_ph = np.zeros((Nz, Nz), dtype=np.complex128, order="F")
    out_pp = np.zeros((Nz, Nz), dtype=np.complex128, order="F")
    nu = np.arange(Nf)
    for l1 in range(Nl):
        for l2 in range(Nl):
            out_ph[l1 * Nf + nu, l2 * Nf + nu] = bph[:, l1, l2]
            out_pp[l1 * Nf + nu, l2 * Nf + nu] = bpp[:, l1, l2]
    return out_ph, out_pp


# --------------------------------------------------------------------------
# BSE, parquet_BSE.f90:19-135
# --------------------------------------------------------------------------
BSE_COEF = {"d": 0.5, "m": 0.5, "s": -0.25, "t": 0.25}  # parquet_BSE.f90:73,89,105,120


def bse_slot(st: State, r: str, Gm: np.ndarray, Fm: np.ndarray, chi: np.ndarray) -> np.ndarray:
    """The damped two-ordering update of one (q, channel) instance
    (parquet_BSE.f90:72-128): Phi = c f [(a Gamma chi) F + F (a chi Gamma)]
    + (1 - f)(F - Gamma), a = 1/(beta Nx Ny)."""
    p = st.p
    alpha = 1.0 / (p.beta * st.Nx * st.Ny)
    f = p.f_damping
    c = BSE_COEF[r] * f
    chiG = alpha * (Gm @ chi)
    gam = c * (chiG @ Fm)
    chiG = alpha * (chi @ Gm)
    gam = gam + c * (Fm @ chiG)
    return gam + (1.0 - f) * (Fm - Gm)


def bse(st: State, ite: int = 0) -> None:
    """``BSE(ite)``: the damped two-ordering update; on exit G_r holds Phi_r."""
    for iq in range(st.Nb):
        qx, qy, w = (int(v) for v in st.ibz[iq])
        cph, cpp = calc_chi(st, qx, qy, w)
        for r in "dmst":
            chi = cph if r in "dm" else cpp
            st.G[r][:, :, iq] = bse_slot(st, r, st.G[r][:, :, iq], st.F[r][:, :, iq], chi)


# --------------------------------------------------------------------------
# Phi(q) -> Phi(R), parquet_PhiR.f90
# --------------------------------------------------------------------------
def calculate_expSqR(st: State) -> np.ndarray:
    """``calculate_expSqR`` (parquet_PhiR.f90:360-395): (NIBZ, NR, Ns)."""
    Nf = st.Nf
    out = np.zeros((st.NIBZ, st.NR, NS), dtype=np.complex128)
    for iq in range(st.NIBZ):
        qx, qy, _ = st.ibz[iq * (Nf // 2)]
        sl = list_symmetries(int(qx), int(qy), st.Nx_IBZ)
        for s in range(1, NS + 1):
            if not sl[s - 1]:
                continue
            sx, sy = symmetry_operation(s, int(qx), int(qy), st.Nx)
            for ir in range(st.NR):
                rx, ry, _ = st.ibz[ir * (Nf // 2)]
                qdr = (2.0 * math.pi / st.Nx) * (sx - 1) * (rx - 1) + (2.0 * math.pi / st.Ny) * (sy - 1) * (ry - 1)
                out[iq, ir, s - 1] = complex(math.cos(qdr), math.sin(qdr))
    st.tables["expSqR"] = out
    return out


def calculate_expqSR(st: State) -> np.ndarray:
    """``calculate_expqSR`` (parquet_PhiR.f90:400-435): (Nc, NR, Ns), k index (ky-1)*Nx+kx."""
    Nf = st.Nf
    out = np.zeros((st.Nc, st.NR, NS), dtype=np.complex128)
    for ir in range(st.NR):
        rx, ry, _ = st.ibz[ir * (Nf // 2)]
        sl = list_symmetries(int(rx), int(ry), st.Nx_IBZ)
        for s in range(1, NS + 1):
            if not sl[s - 1]:
                continue
            sx, sy = symmetry_operation(s, int(rx), int(ry), st.Nx)
            for ky in range(1, st.Ny + 1):
                for kx in range(1, st.Nx + 1):
                    ik = (ky - 1) * st.Nx + kx
                    kd = (2.0 * math.pi / st.Nx) * (kx - 1) * (sx - 1) + (2.0 * math.pi / st.Ny) * (ky - 1) * (sy - 1)
                    out[ik - 1, ir, s - 1] = complex(math.cos(kd), -math.sin(kd))
    st.tables["expqSR"] = out
    return out


def symop_perm(st: State, s: int) -> tuple[np.ndarray, np.ndarray]:
    """Flattened form of ``symop_arr`` (parquet_PhiR.f90:311-356) for symmetry s:
    ret[i] = fac[i] * in[src[i]] over the Nz*Nz column-major block."""
    Nl, Nf, Nz = st.Nl, st.Nf, st.Nz
    src = np.zeros(Nz * Nz, dtype=np.int64)
    fac = np.zeros(Nz * Nz)
    nu = np.arange(Nf)
    for L2 in range(1, Nl + 1):
        for L1 in range(1, Nl + 1):
            l2s, f2 = int(st.lsym[s - 1, L2 - 1]), st.lfac[s - 1, L2 - 1]
            l1s, f1 = int(st.lsym[s - 1, L1 - 1]), st.lfac[s - 1, L1 - 1]
            i_sym = ((l2s - 1) * Nf + nu[None, :]) * Nz + (l1s - 1) * Nf + nu[:, None]
            i_nos = ((L2 - 1) * Nf + nu[None, :]) * Nz + (L1 - 1) * Nf + nu[:, None]
            src[i_nos.ravel()] = i_sym.ravel()
            fac[i_nos.ravel()] = f1 * f2
    return src, fac


def phir_at_w(st: State, PhiQ_w: np.ndarray, perms=None) -> np.ndarray:
    """``FTPhis`` (parquet_PhiR.f90:196-258) for one bosonic frequency:
    PhiQ_w (Nz*Nz, NIBZ), Phi_r of the IBZ momenta at that frequency, column-
    major per momentum -> Phi_r(R) (Nz*Nz, NR)."""
    if perms is None:
        perms = [symop_perm(st, s) for s in range(1, NS + 1)]
    exps = st.expSqR
    acc = np.zeros((st.Nz * st.Nz, st.NR), dtype=np.complex128)
    for s in range(NS):
        src, fac = perms[s]
        d1 = fac[:, None] * PhiQ_w[src, :]
        acc = acc + (1.0 / st.Nx) * (d1 @ exps[:, :, s])
    return acc


def calc_PhiR(st: State) -> None:
    """``calc_PhiR`` -> ``communicatePhis`` (a local copy at one task) ->
    ``FTPhis`` (parquet_PhiR.f90:35-258).  Result PhiR[r] (Nz*Nz, Nf/2, NR)."""
    Nz, Nf, NIBZ = st.Nz, st.Nf, st.NIBZ
    perms = [symop_perm(st, s) for s in range(1, NS + 1)]
    PhiR = {}
    for r in "dmst":
        # PhiQ(Nz, Nz, NIBZ*wperTask) == G_r at one task; reshape (Nz*Nz, Nf/2, NIBZ)
        PhiQ = st.G[r].reshape(Nz * Nz, Nf // 2, NIBZ, order="F")
        out = np.zeros((Nz * Nz, Nf // 2, st.NR), dtype=np.complex128)
        for w in range(Nf // 2):
            out[:, w, :] = phir_at_w(st, PhiQ[:, w, :], perms)
        PhiR[r] = out
    st.arrays["PhiR"] = PhiR


# --------------------------------------------------------------------------
# crossing tensors, parquet_EQMatrix.f90 (iteration 0)
# --------------------------------------------------------------------------
def _kflat(st: State):
    """k-grid helpers: FF as (k, l) with k = (kx, ky) ravelled C-order
    (kx slow); expqSR reindexed to the same k order."""
    Nx, Ny = st.Nx, st.Ny
    FFk = st.FF.reshape(Nx * Ny, st.Nl)  # k = kx*Ny + ky
    FFinvk = st.FF_inv.reshape(NS, Nx * Ny, st.Nl)
    kx = np.repeat(np.arange(Nx), Ny)
    ky = np.tile(np.arange(Ny), Nx)
    eidx = ky * Nx + kx  # (ky-1)*Nx + kx, 0-based
    E = st.expqSR[eidx]  # (Nk, NR, Ns)
    return FFk, FFinvk, E, kx, ky


def calc_M(st: State) -> None:
    """All four ``calc_M_*`` (parquet_EQMatrix.f90:21-360) at one task.

    The tensors depend on the momentum of the bosonic slot only; they are
    evaluated per IBZ momentum and broadcast to the Nb slots."""
    Nx, Ny, Nl, NR = st.Nx, st.Ny, st.Nl, st.NR
    FFk, FFinvk, E, kx, ky = _kflat(st)
    Ec = np.conj(E)
    Mphbar_ph = np.zeros((Nl, Nl, Nl, Nl, st.NIBZ, NR), dtype=np.complex128)
    Mpp_ph = np.zeros_like(Mphbar_ph)
    Mph_pp = np.zeros_like(Mphbar_ph)
    Mphbar_pp = np.zeros_like(Mphbar_ph)
    # M2 of calc_M_phbar_to_ph, :45-61
    M2a = np.einsum("krs,kb->brs", E, FFk)
    # M1 of calc_M_pp_to_ph (:141-158) and calc_M_ph_to_pp / phbar_to_pp (:218-235, :292-309)
    M1p = np.einsum("ka,skc,krs->acrs", FFk, FFinvk, E)
    M1m = np.einsum("ka,skc,krs->acrs", FFk, FFinvk, Ec)
    for iq in range(st.NIBZ):
        qx, qy = (int(v) for v in st.qibz[iq])
        kpq = ((kx + qx - 1) % Nx) * Ny + (ky + qy - 1) % Ny
        qmk = ((qx - 1 - kx + Nx) % Nx) * Ny + (qy - 1 - ky + Ny) % Ny
        # M1 of calc_M_phbar_to_ph (:64-89): (l1, l3, l4, R, sym)
        M1a = np.einsum("krs,ka,skc,skd->acdrs", Ec, FFk, FFinvk, FFinvk[:, kpq, :])
        Mphbar_ph[:, :, :, :, iq, :] = np.einsum("acdrs,brs->abcdr", M1a, M2a)
        eq = st.expqSR[(qy - 1) * Nx + qx - 1]  # (NR, Ns)
        Mpp_ph[:, :, :, :, iq, :] = np.einsum("rs,acrs,bdrs->abcdr", eq, M1p, M1p)
        Mph_pp[:, :, :, :, iq, :] = np.einsum("rs,acrs,bdrs->abcdr", eq, M1m, M1m)
        # M2 of calc_M_phbar_to_pp (:312-333): (l2, l4, R, sym)
        M2d = np.einsum("skd,kb,krs->bdrs", FFinvk[:, qmk, :], FFk, E)
        Mphbar_pp[:, :, :, :, iq, :] = np.einsum("acrs,bdrs->abcdr", M1m, M2d)
    qi = np.arange(st.Nb) // (st.Nf // 2)
    st.arrays.pop("_M_matrix", None)
    st.arrays["M_ibz"] = {"phbar_to_ph": Mphbar_ph, "pp_to_ph": Mpp_ph,
                          "ph_to_pp": Mph_pp, "phbar_to_pp": Mphbar_pp}
    st.arrays["M_q_of_slot"] = qi


def M_full(st: State, name: str) -> np.ndarray:
    """A crossing tensor in the reference layout (Nl, Nl, Nl, Nl, Nb, NR)."""
    return st.M_ibz[name][:, :, :, :, st.M_q_of_slot, :]


# --------------------------------------------------------------------------
# parquet equation, parquet_EQOuter.f90 + parquet_EQContribs.f90
# --------------------------------------------------------------------------
def _clamp_nu(x, Nf):
    """``pickNu(x + 2*Nf)`` (parquet_EQContribs.f90:17-39) == clamp(x, 1, Nf)
    for every argument the crossing calls pass."""
    return np.clip(x, 1, Nf)


# each call: (M name, target pair, TR flag); frequency maps below
CALLS = {
    "phbar_to_ph": ("phbar_to_ph", "dm", False), "phbar_to_ph_TR": ("phbar_to_ph", "dm", True),
    "pp_to_ph": ("pp_to_ph", "dm", False), "pp_to_ph_TR": ("pp_to_ph", "dm", True),
    "ph_to_pp": ("ph_to_pp", "st", False), "ph_to_pp_TR": ("ph_to_pp", "st", True),
    "phbar_to_pp": ("phbar_to_pp", "st", False), "phbar_to_pp_TR": ("phbar_to_pp", "st", True),
}

# calculate_PAE dispatch (parquet_EQOuter.f90:84-113): source channel ->
# [(call, fac1, fac2)]; the _TR twins run when w2 > 1 with the same factors
DISPATCH = {
    "d": [("phbar_to_ph", -0.5, -0.5), ("ph_to_pp", 0.5, 0.5), ("phbar_to_pp", 0.5, -0.5)],
    "m": [("phbar_to_ph", -1.5, 0.5), ("ph_to_pp", -1.5, 0.5), ("phbar_to_pp", -1.5, -0.5)],
    "s": [("pp_to_ph", 0.5, -0.5)],
    "t": [("pp_to_ph", 1.5, 0.5)],
}


def crossing_maps(call: str, w2: int, Om: np.ndarray, nu1: np.ndarray, Nf: int):
    """Frequency maps of one crossing call (parquet_EQContribs.f90:44-524,
    helpers :531-585), 1-based.  Om: (Nb,1), nu1: (1,Nf).

    Returns (valid, target nu2, source nu_a (row of Phi_R), source nu_b)."""
    mF = lambda x: -x + Nf + 1
    if call == "phbar_to_ph":
        t = nu1 + w2 - 1
        valid = t <= Nf
        a = nu1
        b = _clamp_nu(nu1 + Om - 1, Nf)
    elif call == "phbar_to_ph_TR":
        t = nu1 - w2 + 1
        valid = (t <= Nf) & (t >= 1)
        a = mF(nu1)
        b = _clamp_nu(mF(nu1 + Om - 1), Nf)
    elif call == "pp_to_ph":
        t = (w2 - 1) - (nu1 + Om - 1) + Nf + 1
        valid = (t <= Nf) & (t >= 1)
        a = nu1
        b = t
    elif call == "pp_to_ph_TR":
        v = nu1 + (Om + w2 - 1) - 1
        valid = (v <= Nf) & (v >= 1)
        t = mF(v)
        a = mF(nu1)
        b = v
    elif call == "ph_to_pp":
        t = (Om - 1) - (nu1 + w2 - 1) + Nf + 1
        valid = (t <= Nf) & (t >= 1)
        a = nu1
        b = t
    elif call == "ph_to_pp_TR":
        t = Om + w2 - 1 + (-nu1 + Nf + 1) - 1
        valid = (t <= Nf) & (t >= 1)
        a = mF(nu1)
        b = nu1 - (Om + w2 - 1) + 1
    elif call == "phbar_to_pp":
        t = nu1 + w2 - 1
        valid = t <= Nf
        a = nu1
        b = _clamp_nu((Om - 1) - (nu1 + w2 - 1) + Nf + 1, Nf)
    elif call == "phbar_to_pp_TR":
        t = nu1 - w2 + 1
        valid = (t <= Nf) & (t >= 1)
        a = mF(nu1)
        b = _clamp_nu(nu1 - (Om + w2 - 1) + 1, Nf)
    else:
        raise KeyError(call)
    t, a, b, valid = np.broadcast_arrays(t, a, b, valid)
    return valid, t, a, b


def crossing_contribution(st: State, call: str, PhiR: np.ndarray, w2: int) -> tuple:
    """One crossing call's contraction, before the fac/Nx scaling.

    Returns (valid (Nb,Nf), nu2 (Nb,Nf), C (Nl, Nl, Nb, Nf)) with
    C[l1, l2, q, nu1] = sum_{R,l3,l4} M[l1,l2,l3,l4,q,R] * X[l3,l4,q,nu1,R]."""
    Nl, Nf, Nz, NR = st.Nl, st.Nf, st.Nz, st.NR
    mname, _, tr = CALLS[call]
    Om = st.ibz[:, 2][:, None].astype(np.int64)
    nu1 = np.arange(1, Nf + 1)[None, :]
    valid, t, a, b = crossing_maps(call, w2, Om, nu1, Nf)
    P = PhiR[:, w2 - 1, :].reshape(Nz, Nz, NR, order="F")
    l = np.arange(Nl)
    ai = np.clip(a, 1, Nf) - 1
    bi = np.clip(b, 1, Nf) - 1
    rows = l[None, :, None, None] * Nf + ai[:, None, None, :]  # (q,l3,1,nu)
    cols = l[None, None, :, None] * Nf + bi[:, None, None, :]  # (q,1,l4,nu)
    X = P[rows, cols, :]  # (q, l3, l4, nu, R)
    if tr:
        sg = st.signs.astype(np.float64)
        X = (sg[:, None] * sg[None, :])[None, :, :, None, None] * np.conj(X)
    X = np.where(valid[:, None, None, :, None], X, 0.0)
    # contraction over (l3, l4, R) as a matmul batched over the slots of each
    # IBZ momentum (the tensors depend on the momentum only)
    nh = Nf // 2
    Xm = X.transpose(0, 1, 2, 4, 3).reshape(st.NIBZ, nh, Nl * Nl * NR, Nf)
    Mm = _M_matrix(st, mname)  # (NIBZ, 1, Nl*Nl, Nl*Nl*NR)
    C = np.matmul(Mm, Xm)  # (NIBZ, nh, Nl*Nl, Nf)
    C = C.reshape(st.Nb, Nl, Nl, Nf).transpose(2, 1, 0, 3)  # (l1, l2, q, nu)
    return valid, t, C


def _M_matrix(st: State, name: str) -> np.ndarray:
    """M_*[l1,l2,l3,l4,Q,R] as (NIBZ, 1, (l2,l1), (l3,l4,R)) for the batched matmul."""
    cache = st.arrays.setdefault("_M_matrix", {})
    if name not in cache:
        M = st.M_ibz[name]  # (l1, l2, l3, l4, Q, R)
        Nl, NR = st.Nl, st.NR
        cache[name] = M.transpose(4, 1, 0, 2, 3, 5).reshape(st.NIBZ, 1, Nl * Nl, Nl * Nl * NR).copy()
    return cache[name]


def calculate_PAE(st: State) -> None:
    """``calculate_PAE`` (parquet_EQOuter.f90:16-118)."""
    Nf, Nl, Nb = st.Nf, st.Nl, st.Nb
    F = {r: st.G[r].copy(order="F") for r in "dmst"}
    aux = abs(1.0 / st.FF[0, 0, 0] * 1.0 / st.FF[0, 0, 0])
    q0 = st.ibz[:, 2] - 1
    for r in "dmst":
        F[r][:Nf, :Nf, :] += st.L[r][:, :, q0] * aux
    inv_nx = 1.0 / st.Nx
    l = np.arange(Nl)
    qq = np.arange(Nb)
    nu1 = np.arange(1, Nf + 1)
    for src in "dmst":
        PhiR = st.PhiR[src]
        for w2 in range(1, Nf // 2 + 1):
            for base, fac1, fac2 in DISPATCH[src]:
                calls = [base] + ([base + "_TR"] if w2 > 1 else [])
                for call in calls:
                    _, pair, _ = CALLS[call]
                    valid, t, C = crossing_contribution(st, call, PhiR, w2)
                    qv, nv = np.nonzero(valid)
                    rows = l[:, None, None] * Nf + (nu1[nv] - 1)[None, None, :]
                    cols = l[None, :, None] * Nf + (t[qv, nv] - 1)[None, None, :]
                    vals = C[:, :, qv, nv]
                    qi = np.broadcast_to(qq[qv][None, None, :], rows.shape)
                    rows, cols = np.broadcast_arrays(rows, cols)
                    F[pair[0]][rows, cols, qi] += vals * fac1 * inv_nx
                    F[pair[1]][rows, cols, qi] += vals * fac2 * inv_nx
    st.arrays["F"] = F


def crossing_slot(st: State, iq: int, Phi: dict, PhiR: dict) -> dict:
    """``calculate_PAE`` (parquet_EQOuter.f90:16-118) restricted to the target
    slot iq (0-based): Phi[r] (Nz, Nz) of that slot, PhiR[r] (Nz*Nz, Nf/2, NR)
    of all slots, the crossing tensors from ``calc_M``.  Returns F[r] (Nz, Nz)
    of the slot, the same sums as ``calculate_PAE`` in the same call order."""
    Nf, Nl, Nz, NR = st.Nf, st.Nl, st.Nz, st.NR
    aux = abs(1.0 / st.FF[0, 0, 0] * 1.0 / st.FF[0, 0, 0])
    Om = int(st.ibz[iq, 2])
    Q = iq // (Nf // 2)
    F = {r: np.array(Phi[r], dtype=np.complex128, order="F") for r in "dmst"}
    for r in "dmst":
        F[r][:Nf, :Nf] += st.L[r][:, :, Om - 1] * aux
    inv_nx = 1.0 / st.Nx
    l = np.arange(Nl)
    nu1 = np.arange(1, Nf + 1)
    sg = st.signs.astype(np.float64)
    Mq = {name: st.M_ibz[name][:, :, :, :, Q, :].reshape(Nl * Nl, Nl * Nl * NR, order="F")
          for name in ("phbar_to_ph", "pp_to_ph", "ph_to_pp", "phbar_to_pp")}
    for src in "dmst":
        for w2 in range(1, Nf // 2 + 1):
            P = PhiR[src][:, w2 - 1, :].reshape(Nz, Nz, NR, order="F")
            for base, fac1, fac2 in DISPATCH[src]:
                calls = [base] + ([base + "_TR"] if w2 > 1 else [])
                for call in calls:
                    mname, pair, tr = CALLS[call]
                    valid, t, a, b = crossing_maps(call, w2, np.array([[Om]]), nu1[None, :], Nf)
                    valid, t, a, b = valid[0], t[0], a[0], b[0]
                    nv = np.nonzero(valid)[0]
                    if nv.size == 0:
                        continue
                    rows = l[:, None, None] * Nf + (np.clip(a[nv], 1, Nf) - 1)[None, None, :]
                    cols = l[None, :, None] * Nf + (np.clip(b[nv], 1, Nf) - 1)[None, None, :]
                    X = P[rows, cols, :]  # (l3, l4, nu, R)
                    if tr:
                        X = (sg[:, None] * sg[None, :])[:, :, None, None] * np.conj(X)
                    Xm = X.transpose(0, 1, 3, 2).reshape(Nl * Nl * NR, nv.size, order="F")
                    C = (Mq[mname] @ Xm).reshape(Nl, Nl, nv.size, order="F")  # (l1, l2, nu)
                    ro = l[:, None, None] * Nf + (nu1[nv] - 1)[None, None, :]
                    co = l[None, :, None] * Nf + (t[nv] - 1)[None, None, :]
                    ro, co = np.broadcast_arrays(ro, co)
                    F[pair[0]][ro, co] += C * fac1 * inv_nx
                    F[pair[1]][ro, co] += C * fac2 * inv_nx
    return F


# --------------------------------------------------------------------------
# Schwinger-Dyson equation, parquet_SDE.f90
# --------------------------------------------------------------------------
def pick_range(st: State) -> np.ndarray:
    """``fillpickNu_range`` (parquet_SDE.f90:649-676), 1-based values for
    nu = 1..(2 f_range + 1) Nf."""
    fr, Nf = st.p.f_range, st.Nf
    nu = np.arange(1, (2 * fr + 1) * Nf + 1)
    return np.where(nu <= fr * Nf, 1, np.where(nu < (fr + 1) * Nf + 1, nu - fr * Nf, Nf))


def calc_chi_aux(st: State) -> tuple[np.ndarray, np.ndarray]:
    """``calc_chi_aux`` (parquet_SDE.f90:344-435): (Nl*(2fr+1)*Nf, Nb) each."""
    Nx, Ny, Nf, Ng, Nl = st.Nx, st.Ny, st.Nf, st.Ng, st.Nl
    fr = st.p.f_range
    nbox = (2 * fr + 1) * Nf
    l40 = np.arange(-fr * Nf + 1, (fr + 1) * Nf + 1)  # 1-based extended frequency
    kx = np.arange(Nx)[:, None, None]
    ky = np.arange(Ny)[None, :, None]
    nu = l40[None, None, :]
    cph = np.zeros((Nl * nbox, st.Nb), dtype=np.complex128)
    cpp = np.zeros((Nl * nbox, st.Nb), dtype=np.complex128)
    FF = st.FF
    for iq in range(st.Nb):
        qx, qy, w = (int(v) for v in st.ibz[iq])
        kpqx = (kx + qx - 1) % Nx
        kpqy = (ky + qy - 1) % Ny
        mkx = (-kx + Nx) % Nx
        mky = (-ky + Ny) % Ny
        qmkx = (mkx + qx - 1) % Nx
        qmky = (mky + qy - 1) % Ny
        gph = np.zeros((Nx, Ny, nbox), dtype=np.complex128)
        gpp = np.zeros((Nx, Ny, nbox), dtype=np.complex128)
        for gx in range(Ng):
            for gy in range(Ng):
                gk = green_coarse(st, gx, gy, kx, ky, nu)
                gkpq = green_coarse(st, gx, gy, kpqx, kpqy, nu + w - 1)
                gph = gph + gk * gkpq / (Ng * Ng)
                gqmk = green_coarse(st, Ng - gx - 1, Ng - gy - 1, qmkx, qmky, (-nu + Nf + 1) + w - 1)
                gpp = gpp + gk * gqmk / (Ng * Ng)
        # sum over k with FF(k, l4); index (l4-1)*(2fr+1)*Nf + fr*Nf + l4_0
        cph[:, iq] = np.einsum("xyn,xyl->ln", gph, FF).reshape(-1)
        cpp[:, iq] = np.einsum("xyn,xyl->ln", gpp, FF).reshape(-1)
    return cph, cpp


def calc_chi_contractions(st: State, cph, cpp):
    """``calc_LChi``, ``calc_PhChi``, ``calc_PPChi`` (parquet_SDE.f90:439-574).

    G_r holds Phi_r here.  Returns LChi, PhChi, PPChi (Nz, Nb)."""
    p = st.p
    Nf, Nl, Nz, Nb = st.Nf, st.Nl, st.Nz, st.Nb
    fr = p.f_range
    nbox = (2 * fr + 1) * Nf
    l40 = np.arange(-fr * Nf + 1, (fr + 1) * Nf + 1)
    inb = (l40 > 0) & (l40 < Nf + 1)
    ff2 = 1.0 / (st.FF[0, 0, 0] * st.FF[0, 0, 0])
    U = p.U
    LChi = np.zeros((Nz, Nb), dtype=np.complex128)
    q0 = st.ibz[:, 2] - 1
    c1 = cph[:nbox, :]  # l4 = 1 block
    # in-box: (L_d - L_m)/FF^2 chi (- 2U/FF^2 chi if use_U2)
    Ld = st.L["d"][:, :, q0]  # (Nf(idxL3), Nf(l4_0), Nb)
    Lm = st.L["m"][:, :, q0]
    cin = c1[inb, :]  # (Nf, Nb)
    acc = np.einsum("ijq,jq->iq", Ld * ff2, cin) - np.einsum("ijq,jq->iq", Lm * ff2, cin)
    if p.use_U2:
        acc = acc - 2.0 * U * ff2 * np.sum(cin, axis=0)[None, :]
    else:
        cout = c1[~inb, :]
        acc = acc + 2.0 * U * ff2 * np.sum(cout, axis=0)[None, :]
    LChi[:Nf, :] = acc
    pk = pick_range(st)  # 1-based
    cols = (np.arange(Nl)[:, None] * Nf + (pk - 1)[None, :]).reshape(-1)  # (Nl*nbox,)
    Phd = st.G["d"][:, cols, :]
    Phm = st.G["m"][:, cols, :]
    Phs = st.G["s"][:, cols, :]
    Pht = st.G["t"][:, cols, :]
    PhChi = np.einsum("ijq,jq->iq", Phd, cph) - np.einsum("ijq,jq->iq", 3.0 * Phm, cph)
    PPChi = np.einsum("ijq,jq->iq", Phs, cpp) + np.einsum("ijq,jq->iq", Pht, cpp)
    return LChi, PhChi, PPChi


def symmetrize_array(st: State, num_freqs: int, arr_in: np.ndarray) -> np.ndarray:
    """``symmetrize_array`` (parquet_util.f90:1215-1272)."""
    Nx, Ny = st.Nx, st.Ny
    out = np.zeros(Nx * Ny * num_freqs, dtype=np.complex128)
    nu = np.arange(num_freqs)
    for qx in range(1, st.Nx_IBZ + 1):
        for qy in range(1, qx + 1):
            idx_q = (((qx - 1) * qx) // 2 + qy - 1) * num_freqs + nu
            sl = list_symmetries(qx, qy, st.Nx_IBZ)
            for s in range(1, NS + 1):
                if not sl[s - 1]:
                    continue
                sx, sy = symmetry_operation(s, qx, qy, Nx)
                idx = ((sx - 1) * Ny + sy - 1) * num_freqs + nu
                out[idx] += arr_in[idx_q]
    return out


def calc_order_2nd(st: State) -> np.ndarray:
    """``calc_order_2nd`` (parquet_SDE.f90:264-338)."""
    p = st.p
    Nx, Ny, Nf, Ng = st.Nx, st.Ny, st.Nf, st.Ng
    Grt = st.Grt
    n1, n2 = Nx * Ng, Ny * Ng
    km1 = np.array([0] + [n1 - k for k in range(1, n1)])
    km2 = np.array([0] + [n2 - k for k in range(1, n2)])
    mirror = Grt[km1[:, None], km2[None, :], :][:, :, ::-1]
    GGG = Grt ** 2 * mirror * p.U * p.U
    GGG = fftb2d(GGG)
    out = np.zeros(Nx * Ny * Nf, dtype=np.complex128)
    dt = p.beta / (Nf - 1)
    for kx in range(1, Nx + 1):
        kxc = (kx - 1) * Ng
        for ky in range(1, Ny + 1):
            kyc = (ky - 1) * Ng
            g = GGG[kxc, kyc, :].real
            fd1, fd2 = fdfit(g, dt)
            ret = nfourier(True, Nf - 1, Nf // 2, fd1, fd2, g, p.beta)
            base = ((kx - 1) * Ny + ky - 1) * Nf
            for nu in range(1, Nf // 2 + 1):
                out[base + nu - 1] += np.conj(ret[Nf // 2 - nu])
                out[base + Nf - nu] += ret[Nf // 2 - nu]
    return out


def sde_sigma_ibz(st: State, LChi, PhChi, PPChi) -> np.ndarray:
    """Sigma_V accumulation loop (parquet_SDE.f90:116-221), vectorised over
    (k_IBZ, nu); returns Sigma_V (NIBZ*Nf,)."""
    p = st.p
    Nx, Ny, Nf, Nl = st.Nx, st.Ny, st.Nf, st.Nl
    # IBZ fermionic points in the order of idxK
    kl = []
    for kx in range(1, st.Nx_IBZ + 1):
        for ky in range(1, kx + 1):
            kl.append((kx, ky))
    kl = np.array(kl, dtype=np.int64)
    nk = len(kl)
    kx = kl[:, 0][:, None]  # 1-based (nk,1)
    ky = kl[:, 1][:, None]
    k0 = np.arange(1, Nf + 1)[None, :]  # (1,Nf)
    sig = np.zeros((nk, Nf), dtype=np.complex128)
    sg = st.signs.astype(np.float64)
    l = np.arange(Nl)
    for iq in range(st.Nb):
        qx, qy, w = (int(v) for v in st.ibz[iq])
        sl = list_symmetries(qx, qy, st.Nx_IBZ)
        for s in range(1, NS + 1):
            if not sl[s - 1]:
                continue
            sx, sy = symmetry_operation(s, qx, qy, Nx)
            # K + Sq
            kqx = (kx - 1 + sx - 1) % Nx
            kqy = (ky - 1 + sy - 1) % Ny
            gkq = green(st, kqx, kqy, k0 + w - 1)
            # -K + Sq
            mkx = (-(kx - 1) + Nx) % Nx
            mky = (-(ky - 1) + Ny) % Ny
            qmkx = (mkx + sx - 1) % Nx
            qmky = (mky + sy - 1) % Ny
            qmkw = (-k0 + Nf + 1) + w - 1
            gqmk = green(st, qmkx, qmky, qmkw)
            kmqx = (-qmkx + Nx) % Nx
            kmqy = (-qmky + Ny) % Ny
            gkmq = green(st, kmqx, kmqy, -qmkw + Nf + 1)
            ffi = st.FF_inv[s - 1, kx[:, 0] - 1, ky[:, 0] - 1, :]  # (nk, Nl)
            idx3 = l[None, :] * Nf + (k0[0] - 1)[:, None]  # (Nf, Nl)
            Lc = LChi[idx3, iq]
            Pc = PhChi[idx3, iq]
            Qc = PPChi[idx3, iq]
            # sum over l3 of FF_inv * chi terms, (nk, Nf)
            sL = np.einsum("kl,nl->kn", ffi, Lc)
            sP = np.einsum("kl,nl->kn", ffi, Pc)
            sQ = np.einsum("kl,nl->kn", ffi, Qc)
            sig += gkq * sL + gkq * sP + gqmk * sQ
            if w == 1:
                continue
            idx3m = l[None, :] * Nf + (Nf - k0[0])[:, None]
            ffs = ffi * sg[None, :]
            tL = np.einsum("kl,nl->kn", ffs, np.conj(LChi[idx3m, iq]))
            tP = np.einsum("kl,nl->kn", ffs, np.conj(PhChi[idx3m, iq]))
            tQ = np.einsum("kl,nl->kn", ffs, np.conj(PPChi[idx3m, iq]))
            sig += gkmq * tL + gkmq * tP + np.conj(gkq) * tQ
    pref = p.U / p.beta / p.beta / st.Nc / st.Nc / 2.0
    return (-pref * sig).reshape(-1)


def calc_SDE(st: State) -> None:
    """``calc_SDE`` (parquet_SDE.f90:27-258)."""
    cph, cpp = calc_chi_aux(st)
    LChi, PhChi, PPChi = calc_chi_contractions(st, cph, cpp)
    st.arrays["chi_aux"] = (cph, cpp)
    st.arrays["LChi"] = (LChi, PhChi, PPChi)
    sv = sde_sigma_ibz(st, LChi, PhChi, PPChi)
    Sigma = symmetrize_array(st, st.Nf, sv)
    if st.p.use_U2:
        Sigma = Sigma + calc_order_2nd(st)
    st.arrays["Sigma"] = Sigma


# --------------------------------------------------------------------------
# convergence and the loop
# --------------------------------------------------------------------------
def conv(st: State) -> tuple[bool, dict]:
    """``conv`` (parquet_check.f90:39-150), plus the optional absolute
    sup-norm test on the self-energy change."""
    S, So = st.Sigma, st.SigmaOld
    with np.errstate(invalid="ignore", divide="ignore"):  # Sigma = 0 (U = 0): NaN, as in the reference
        rel = np.abs(So - S) / np.abs(S)
    rel_sig_max = float(np.max(rel))
    dsig_inf = float(np.max(np.abs(So - S)))
    out = {"rel_sig_max": rel_sig_max, "rel_sig_av": float(abs(np.sum(rel) / rel.size)),
           "dsigma_inf": dsig_inf}
    conv_ok = rel_sig_max < F_SIGMA
    for r in "dmst":
        fmax = float(np.max(np.abs(st.F[r])))
        prev = st.F_max[r]
        err = abs(1.0 - fmax / prev) if prev != 0.0 else math.inf
        out[f"rel_err_{r}"] = err
        out[f"F_{r}_max"] = fmax
        conv_ok = conv_ok and err < F_VERT
        st.F_max[r] = fmax
    if st.p.conv_abs > 0.0:
        conv_ok = dsig_inf < st.p.conv_abs
    st.arrays["SigmaOld"] = S.copy()
    return conv_ok, out


# --------------------------------------------------------------------------
# readout every 5 iterations: exact chi0 bubble and susceptibilities
# (parquet_chi.f90:216-430, parquet_sus.f90:18-643, parquet_plot.f90:14-58)
# --------------------------------------------------------------------------
def grt_pre_fft(st: State) -> np.ndarray:
    """G(k, tau) on the fine grid before the spatial FFT, for the current mu
    and Sigma (parquet_chi.f90:124-174 / :355-390)."""
    Nx, Ny, Nf, Ng, beta, mu = st.Nx, st.Ny, st.Nf, st.Ng, st.p.beta, st.mu
    Sig = st.Sigma.reshape(Nx, Ny, Nf)
    nu = np.arange(1, Nf + 1)
    fr = freq(st, nu)
    tau = beta / (Nf - 1) * (np.arange(1, Nf + 1) - 1)
    ph = -math.pi / beta * (2.0 * (nu - Nf // 2) - 1.0)
    tw = np.exp(1j * (ph[None, :] * tau[:, None]))
    out = np.zeros((Nx * Ng, Ny * Ng, Nf), dtype=np.complex128)
    src = np.zeros((Nx * Ng, Ny * Ng), dtype=np.int64)  # coarse k of each fine point
    for ky in range(1, Ny + 1):
        for kx in range(1, Nx + 1):
            for kyc in range(1, Ng + 1):
                for kxc in range(1, Ng + 1):
                    i1 = _grain_index(kx, kxc, Nx, Ng)
                    i2 = _grain_index(ky, kyc, Ny, Ng)
                    e = st.Ek_grain[kxc - 1, kyc - 1, kx - 1, ky - 1]
                    gc = 1.0 / (fr + mu - e - Sig[kx - 1, ky - 1, :])
                    d1 = gc - 1.0 / (fr + mu - e)
                    dummy = np.sum((tw * d1[None, :]).real / beta, axis=1)
                    out[i1 - 1, i2 - 1, :] = dummy - np.exp((beta - tau) * (e - mu)) / (1.0 + np.exp(beta * (e - mu)))
                    src[i1 - 1, i2 - 1] = (kx - 1) * Ny + (ky - 1)
    return out, src


def _bosonic_ibz(st: State, data: np.ndarray) -> np.ndarray:
    """Spline transform tau -> bosonic frequencies at the IBZ points of a
    fine-grid (n1, n2, Nf) array (parquet_chi.f90:242-257)."""
    Nf, Ng = st.Nf, st.Ng
    out = np.zeros(st.Nred, dtype=np.complex128)
    for i in range(1, st.Nx_IBZ + 1):
        for j in range(1, i + 1):
            g = data[(i - 1) * Ng, (j - 1) * Ng, :].real
            fd1, fd2 = fdfit(g, st.p.beta / float(Nf - 1))
            c = nfourier(False, Nf - 1, Nf // 2, fd1, fd2, g, st.p.beta)
            base = ((i * (i - 1)) // 2 + j - 1) * (Nf // 2)
            out[base:base + Nf // 2] = c
    return out


def _mirror(a: np.ndarray) -> np.ndarray:
    """a(-r, beta - tau): index 1 stays, idx -> n - idx + 2 (1-based), tau reversed."""
    n1, n2 = a.shape[0], a.shape[1]
    m1 = np.array([0] + [n1 - k for k in range(1, n1)])
    m2 = np.array([0] + [n2 - k for k in range(1, n2)])
    return a[m1[:, None], m2[None, :], :][:, :, ::-1]


def calc_chi0_exact(st: State) -> dict:
    """The cal_chi branch of calc_Gkw_Grt (parquet_chi.f90:216-430): Chi0_ph,
    Chi0_pp (Nred) and the s/d-wave projected Chi0_ph_FF, Chi0_pp_FF (Nred, 4).
    Uses the Grt of the preceding calc_Gkw_Grt(.true.) call."""
    Grt = st.Grt
    sd = fill_ff_sdwave(st.Nx)
    out = {"chi0_ph": _bosonic_ibz(st, fftb2d(-Grt * _mirror(Grt))),
           "chi0_pp": _bosonic_ibz(st, fftb2d(-0.5 * Grt ** 2))}
    pre, src = grt_pre_fft(st)
    ph_ff = np.zeros((st.Nred, 4), dtype=np.complex128)
    pp_ff = np.zeros((st.Nred, 4), dtype=np.complex128)
    sdk = sd.reshape(st.Nx * st.Ny, 4)  # k = (kx-1)*Ny + ky-1
    for ff in range(4):
        w = (sdk[src, ff] * sdk[src, ff])[:, :, None]
        FFG = fftf2d(pre * w)
        ph_ff[:, ff] = _bosonic_ibz(st, fftb2d(-Grt * _mirror(FFG)))
        pp_ff[:, ff] = _bosonic_ibz(st, fftb2d(-0.5 * Grt * FFG))
    out["chi0_ph_FF"] = ph_ff
    out["chi0_pp_FF"] = pp_ff
    return out


def calc_GG(st: State, pp: bool) -> np.ndarray:
    """calc_GG_ph / calc_GG_pp (parquet_sus.f90:528-643): (Nl*nbox, Nb, 4)."""
    Nx, Ny, Nf, Ng, Nl = st.Nx, st.Ny, st.Nf, st.Ng, st.Nl
    fr = st.p.f_range
    nbox = (2 * fr + 1) * Nf
    l0 = np.arange(-fr * Nf + 1, (fr + 1) * Nf + 1)
    sd = fill_ff_sdwave(Nx)
    kx = np.arange(Nx)[:, None, None]
    ky = np.arange(Ny)[None, :, None]
    nu = l0[None, None, :]
    out = np.zeros((Nl * nbox, st.Nb, 4), dtype=np.complex128)
    for iq in range(st.Nb):
        qx, qy, w = (int(v) for v in st.ibz[iq])
        g2 = np.zeros((Nx, Ny, nbox), dtype=np.complex128)
        for gx in range(Ng):
            for gy in range(Ng):
                gk = green_coarse(st, gx, gy, kx, ky, nu)
                if not pp:
                    g2 = g2 + gk * green_coarse(st, gx, gy, (kx + qx - 1) % Nx, (ky + qy - 1) % Ny, nu + w - 1) \
                        / Ng / Ng
                else:
                    mkx, mky = (-kx + Nx) % Nx, (-ky + Ny) % Ny
                    g2 = g2 + gk * green_coarse(st, Ng - gx - 1, Ng - gy - 1, (mkx + qx - 1) % Nx,
                                                (mky + qy - 1) % Ny, (-nu + Nf + 1) + w - 1) / Ng / Ng
        for ff in range(4):
            out[:, iq, ff] = np.einsum("xy,xyn,xyl->ln", sd[:, :, ff], g2, st.FF).reshape(-1)
    return out


def calc_sus(st: State) -> dict:
    """calc_sus (parquet_sus.f90:18-522) at one task: sus_r_IBZ (Nred, 4).
    Uses F_r of this iteration and Phi_r (the G arrays before the update)."""
    Nf, Nl, Nx, Ny, beta = st.Nf, st.Nl, st.Nx, st.Ny, st.p.beta
    fr = st.p.f_range
    nbox = (2 * fr + 1) * Nf
    norm = 1.0 / (Nx * Nx * Ny * Ny * beta * beta)
    l0 = np.arange(-fr * Nf + 1, (fr + 1) * Nf + 1)
    inb = (l0 > 0) & (l0 < Nf + 1)
    pk = pick_range(st)
    ff2 = 1.0 / (st.FF[0, 0, 0] * st.FF[0, 0, 0])
    lam = {"d": st.p.U, "m": -st.p.U, "s": 2.0 * st.p.U, "t": 0.0}
    out = {}
    for pp, chans in ((False, "dm"), (True, "st")):
        GG = calc_GG(st, pp)  # (Nl*nbox, Nb, 4)
        Gb = GG.reshape(Nl, nbox, st.Nb, 4)
        vin = Gb[:, inb, :, :].reshape(Nl * Nf, st.Nb, 4)  # in-box, index (l-1)*Nf + l0
        for r in chans:
            s = np.einsum("ijq,iqf,jqf->qf", st.F[r], vin, vin) * norm
            if fr > 0:
                # terms with at least one frequency outside the box
                cols = (np.arange(Nl)[:, None] * Nf + (pk - 1)[None, :]).reshape(-1)
                Phx = st.G[r][cols[:, None], cols[None, :], :]  # (Nl*nbox, Nl*nbox, Nb)
                outside = ~(inb[:, None] & inb[None, :])
                mask = np.tile(outside, (Nl, Nl))
                Gv = GG  # (Nl*nbox, Nb, 4)
                s = s + np.einsum("ijq,iqf,jqf->qf", np.where(mask[:, :, None], Phx, 0.0), Gv, Gv) * norm
                # Lambda term on l1 = l2 = 1
                g1 = Gb[0]  # (nbox, Nb, 4)
                m11 = outside
                s = s + lam[r] * ff2 * np.einsum("ij,iqf,jqf->qf", m11.astype(float), g1, g1) * norm
            out[f"sus_{r}_IBZ"] = s
    return out


def symmetrize_sus(st: State, sus: dict, chi0: dict) -> dict:
    """symmetrize_sus (parquet_plot.f90:14-58): whole-BZ arrays (Nx*Ny*Nf/2[, 4])."""
    nh = st.Nf // 2
    out = {}
    for r in "dmst":
        out[f"sus_{r}"] = np.stack([symmetrize_array(st, nh, sus[f"sus_{r}_IBZ"][:, f]) for f in range(4)], axis=1)
    out["chi0_ph_BZ"] = symmetrize_array(st, nh, chi0["chi0_ph"])
    out["chi0_pp_BZ"] = symmetrize_array(st, nh, chi0["chi0_pp"])
    out["chi0_ph_BZ_FF"] = np.stack([symmetrize_array(st, nh, chi0["chi0_ph_FF"][:, f]) for f in range(4)], axis=1)
    out["chi0_pp_BZ_FF"] = np.stack([symmetrize_array(st, nh, chi0["chi0_pp_FF"][:, f]) for f in range(4)], axis=1)
    return out


def readout(st: State, ite: int) -> dict:
    """The output block of loop.f90:181-213 without HDF5: calc_Gkw_Grt(.true.),
    calc_sus, symmetrize_sus."""
    calc_Gkw_Grt(st, ite, True)
    chi0 = calc_chi0_exact(st)
    sus = calc_sus(st)
    out = dict(chi0)
    out.update(sus)
    out.update(symmetrize_sus(st, sus, chi0))
    return out


def output_block_mu(st: State) -> None:
    """Side effect of the every-5-iterations readout on the trajectory:
    ``calc_Gkw_Grt(.true.)`` (loop.f90:195) resets mu to the midpoint of
    [mu-U, mu+U] (parquet_chi.f90:114-122) and recomputes Sigma_H, Grt and
    Gkw from the new Sigma; the next iteration recomputes those anyway."""
    p = st.p
    st.mu = 0.5 * ((st.mu + p.U) + (st.mu - p.U))


def iteration(st: State, ite: int, with_readout: bool = False) -> tuple[bool, dict]:
    """One pass of ``execute_loop`` (loop.f90:51-244) without the HDF5 output.
    ``with_readout``: at the output iterations run the readout of the output
    block (loop.f90:181-213) where the reference does, after conv and before
    the vertex update, and return it as ``info["readout"]``; its
    calc_Gkw_Grt(.true.) has the same effect on mu as ``output_block_mu``."""
    p = st.p
    steps = calc_Gkw_Grt(st, ite, False)
    bse(st, ite)
    if ite == 0:
        calculate_expSqR(st)
        calculate_expqSR(st)
    calc_PhiR(st)
    if ite == 0:
        calc_M(st)
    calculate_PAE(st)
    if not p.oneshot or ite == p.ite_max - 1:
        st.arrays["SigmaOld"] = st.Sigma.copy()
        calc_SDE(st)
    converged, info = conv(st)
    info["bisection_steps"] = steps
    info["mu"] = st.mu
    if ite % 5 == 0 or ite == p.ite_max - 1 or converged:
        if with_readout:
            info["readout"] = readout(st, ite)
        else:
            output_block_mu(st)
    for r in "dmst":
        st.G[r] = st.F[r] - st.G[r]
    return converged, info


def execute_loop(st: State, ite_max: int | None = None, callback=None):
    """``execute_loop`` (loop.f90:29-249)."""
    ite_max = st.p.ite_max if ite_max is None else ite_max
    converged = False
    ite = 0
    infos = []
    while not converged and ite < ite_max:
        converged, info = iteration(st, ite)
        infos.append(info)
        if callback:
            callback(ite, st, info)
        ite += 1
    return converged, ite, infos

"""Host-side mirror of the reference's Fortran module interface.

``Solver`` holds one device context.  Its methods carry the names of the
reference routines they replace and take the same arguments:

=========================  ==================================================
reference (module :: name)  here
=========================  ==================================================
parquet_ini::set_parameters ``read_prms(path)``
parquet_chi::calc_Gkw_Grt   ``Solver.calc_Gkw_Grt(ite, cal_chi)``
parquet_chi::calc_chi       ``Solver.calc_chi(idx_q)``
Parquet_kernel::BSE         ``Solver.BSE(ite)``
parquet_PhiR::calc_PhiR     ``Solver.calc_PhiR(ite)`` (+ calculate_expSqR/qSR)
parquet_EQMatrix::calc_M_*  ``Solver.calc_M_phbar_to_ph()`` etc.
parquet_EQOuter::calculate_PAE ``Solver.calculate_PAE()``
parquet_SDE::calc_SDE       ``Solver.calc_SDE(ite)``
parquet_check::conv         ``Solver.conv()``
loop::execute_loop          ``Solver.execute_loop()``
=========================  ==================================================

The module-global arrays of ``parquet_ini`` are read and written through
properties (``Sigma``, ``F(channel)``, ``G(channel)``, ``mu`` ...) in the
reference's Fortran layouts.  Every call goes to the CUDA library; a failing
call raises ``TupsError``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib
from ._lib import TupsError, tups_conv_info, tups_dims, tups_params

CHANNELS = "dmst"


@dataclass
class Params:
    """The 21 prms records (SRC/parquet_ini.f90:300-322) plus extensions."""
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
    tprime: float = 0.0
    conv_abs: float = 0.0

    def to_c(self) -> tups_params:
        p = tups_params()
        for f in fields(self):
            v = getattr(self, f.name)
            if isinstance(v, str):
                v = v.encode()[:255]
            elif isinstance(v, bool):
                v = int(v)
            setattr(p, f.name, v)
        return p

    @classmethod
    def from_c(cls, p: tups_params) -> "Params":
        kw = {}
        for f in fields(cls):
            v = getattr(p, f.name)
            if f.type in ("bool", bool):
                v = bool(v)
            elif isinstance(v, bytes):
                v = v.decode()
            kw[f.name] = v
        return cls(**kw)


def _check(lib, ctx, rc: int) -> None:
    if rc != _lib.TUPS_OK:
        msg = lib.tups_last_error(ctx).decode() if ctx else lib.tups_strerror(rc).decode()
        raise TupsError(rc, msg or lib.tups_strerror(rc).decode())


def read_prms(path: str, tprime: float | None = None, conv_abs: float | None = None) -> Params:
    """``set_parameters``: parse a 21-record prms file with the native parser,
    and ``<path>.gpu`` (tprime, conv_abs) when it exists; keyword values given
    here take precedence over that file."""
    lib = _lib.load()
    p = tups_params()
    rc = lib.tups_read_prms(str(path).encode(), C.byref(p))
    if rc != 0:
        raise TupsError(rc, f"cannot read prms file {path} (or its .gpu extensions)")
    out = Params.from_c(p)
    if tprime is not None:
        out.tprime = tprime
    if conv_abs is not None:
        out.conv_abs = conv_abs
    return out


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def host_tables(params: Params) -> dict:
    """Sizes and form-factor/symmetry/index tables built by the native host
    code without touching a GPU (the host part of tups_ctx_create)."""
    lib = _lib.load()
    cp = params.to_c()
    d = tups_dims()
    rc = lib.tups_host_tables(C.byref(cp), C.byref(d), *([None] * 7))
    if rc != 0:
        raise TupsError(rc, "tups_host_tables failed (see stderr)")
    dims = {f[0]: getattr(d, f[0]) for f in d._fields_}
    nl, nx = dims["Nl"], dims["Nx"]
    FF = np.empty((nx, nx, nl), order="F")
    FFi = np.empty((8, nx, nx, nl), order="F")
    signs = np.empty(nl, dtype=np.int32)
    reps = np.empty(nl, dtype=np.int32)
    lsym = np.empty((8, nl), dtype=np.int32, order="F")
    lfac = np.empty((8, nl), order="F")
    ibz = np.empty((3, dims["Nred"]), dtype=np.int32, order="F")
    rc = lib.tups_host_tables(C.byref(cp), C.byref(d), *(_ptr(x) for x in (FF, FFi, signs, reps, lsym, lfac, ibz)))
    if rc != 0:
        raise TupsError(rc, "tups_host_tables failed")
    return {"dims": dims, "FF": FF, "FF_inv": FFi, "signs": signs, "reps": reps, "lsym": lsym, "lfac": lfac,
            "ibz": ibz.T.copy()}


class Solver:
    """One parquet solver instance with device-resident state."""

    def __init__(self, params: Params, device: int = 0, rank: int = 0, ntasks: int = 1, exchange=None):
        """``ntasks > 1``: this solver holds the bosonic slots of rank ``rank``
        (``Nb = Nred / ntasks`` of them, from ``rank * Nb``), and ``exchange``
        (a ``callable(what, device_ptr, count, op) -> None``, e.g.
        ``tups_b200.sharded.TorchExchange``) combines the three buffers that
        need every slot over the ranks."""
        self._lib = _lib.load()
        self.params = params
        self._cp = params.to_c()
        h = C.c_void_p()
        if ntasks > 1:
            if exchange is None:
                raise ValueError("a sharded solver needs an exchange function")
            rc = self._lib.tups_ctx_create_sharded(C.byref(self._cp), device, rank, ntasks, C.byref(h))
        else:
            rc = self._lib.tups_ctx_create(C.byref(self._cp), device, C.byref(h))
        if rc != 0:
            raise TupsError(rc, "tups_ctx_create failed (see stderr)")
        self._ctx = h
        self._xfn = None
        if ntasks > 1:
            def _xch(user, what, data, count, op):
                try:
                    exchange(int(what), int(data), int(count), int(op))
                    return 0
                except Exception as e:  # reported as TUPS_ERR_COMM by the library
                    print(f"tups_b200 exchange {what} failed: {e!r}", flush=True)
                    return 1
            self._xfn = _lib.EXCHANGE_FN(_xch)  # kept alive with the solver
            self._call("tups_set_exchange", C.cast(self._xfn, C.c_void_p), None)
        r, n, s0 = C.c_int(), C.c_int(), C.c_int()
        self._call("tups_get_shard", C.byref(r), C.byref(n), C.byref(s0))
        self.rank, self.ntasks, self.slot0 = r.value, n.value, s0.value
        d = tups_dims()
        self._call("tups_get_dims", C.byref(d))
        self.dims = {f[0]: getattr(d, f[0]) for f in d._fields_}
        for k, v in self.dims.items():
            setattr(self, k, v)

    # -- plumbing --
    def _call(self, name: str, *args) -> None:
        rc = getattr(self._lib, name)(self._ctx, *args)
        _check(self._lib, self._ctx, rc)

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.tups_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.tups_kernel_launches(self._ctx))

    # -- module parquet_chi --
    def calc_Gkw_Grt(self, ite: int, cal_chi: bool = False) -> None:
        self._call("tups_calc_Gkw_Grt", int(ite), int(bool(cal_chi)))

    def calc_chi(self, idx_q: int) -> tuple[np.ndarray, np.ndarray]:
        """Dense (Nz, Nz) chi_ph_LL, chi_pp_LL for the 1-based slot idx_q."""
        ph = np.zeros((self.Nz, self.Nz), dtype=np.complex128, order="F")
        pp = np.zeros((self.Nz, self.Nz), dtype=np.complex128, order="F")
        self._call("tups_calc_chi", int(idx_q), _ptr(ph), _ptr(pp))
        return ph, pp

    # -- module Parquet_kernel --
    def BSE(self, ite: int = 0) -> None:
        self._call("tups_BSE", int(ite))

    # -- module parquet_PhiR --
    def calculate_expSqR(self) -> None:
        self._call("tups_calculate_expSqR")

    def calculate_expqSR(self) -> None:
        self._call("tups_calculate_expqSR")

    def calc_PhiR(self, ite: int = 0) -> None:
        self._call("tups_calc_PhiR", int(ite))

    # -- module parquet_EQMatrix --
    def calc_M_phbar_to_ph(self) -> None:
        self._call("tups_calc_M_phbar_to_ph")

    def calc_M_pp_to_ph(self) -> None:
        self._call("tups_calc_M_pp_to_ph")

    def calc_M_ph_to_pp(self) -> None:
        self._call("tups_calc_M_ph_to_pp")

    def calc_M_phbar_to_pp(self) -> None:
        self._call("tups_calc_M_phbar_to_pp")

    # -- module parquet_EQOuter --
    def calculate_PAE(self) -> None:
        self._call("tups_calculate_PAE")

    # -- module parquet_SDE --
    def calc_SDE(self, ite: int = 0) -> None:
        self._call("tups_calc_SDE", int(ite))

    # -- module parquet_check --
    def conv(self) -> dict:
        ci = tups_conv_info()
        self._call("tups_conv", C.byref(ci))
        return _conv_dict(ci)

    # -- loop.f90 --
    def vertex_update(self) -> None:
        self._call("tups_vertex_update")

    def output_block(self) -> None:
        self._call("tups_output_block")

    def iteration(self, ite: int, readout: bool = False) -> dict:
        """One iteration of execute_loop.  ``readout``: also the output block's
        readout at the output iterations (every 5th, the last, on
        convergence), after conv and before the vertex update as in the
        reference; ``chi0(bz)`` and ``sus(r, bz)`` then hold its results."""
        ci = tups_conv_info()
        self._call("tups_iteration_readout" if readout else "tups_iteration", int(ite), C.byref(ci))
        return _conv_dict(ci)

    def execute_loop(self) -> tuple[int, bool]:
        ite = C.c_int(0)
        conv = C.c_int(0)
        self._call("tups_execute_loop", C.byref(ite), C.byref(conv))
        return ite.value, bool(conv.value)

    def synchronize(self) -> None:
        self._call("tups_synchronize")

    def set_graph(self, enable: bool = True) -> None:
        """Replay iterations (from ite 1 on) from captured CUDA graphs."""
        self._call("tups_set_graph", int(bool(enable)))

    def set_autotune(self, enable: bool = True) -> None:
        """Tile-shape tuner on (default) or off (fixed default tiles)."""
        self._call("tups_set_autotune", int(bool(enable)))

    def set_crossing_products(self, products: int = 3) -> None:
        """Real tensor-core products per complex one in the crossing GEMM: 3 (default) or 4."""
        self._call("tups_set_crossing_products", int(products))

    # -- split-precision BSE --
    def set_bse_precision(self, slices: int = 0, ladder: bool = False) -> None:
        """slices = 0: FP64 tensor cores; 2..8: int8 slices per operand;
        ladder: slices chosen per iteration from the last Sigma change."""
        self._call("tups_set_bse_precision", int(slices), int(bool(ladder)))

    @property
    def bse_slices(self) -> int:
        """Slices the next BSE uses (0 = FP64)."""
        return int(self._lib.tups_get_bse_slices(self._ctx))

    # -- warm start and checkpoint --
    def warm_start(self, sigma: np.ndarray, gamma_l1) -> None:
        """Sigma <- sigma; mu by bisection; Gamma_r <- gamma_l1[r] on the (l=1, l=1)
        nu-block; F_r <- (1 - 2 c_r/(beta Nx Ny) Gamma_r chi_r)^{-1} Gamma_r."""
        sig = np.ascontiguousarray(sigma, dtype=np.complex128).reshape(-1)
        assert sig.size == self.Nt
        gam = np.ascontiguousarray(gamma_l1, dtype=np.complex128).reshape(4)
        self._call("tups_warm_start", _ptr(sig), _ptr(gam))

    def checkpoint(self, save: bool = True) -> None:
        """Store (save) or restore the device-side loop state."""
        self._call("tups_checkpoint", int(bool(save)))

    # -- readout (loop.f90:181-213 without HDF5) --
    def readout(self, ite: int = 0) -> None:
        """calc_Gkw_Grt(.true.) + exact chi0 + calc_sus + symmetrize_sus."""
        self._call("tups_readout", int(ite))

    def chi0(self, bz: bool = False) -> dict:
        n = self.Nc * (self.Nf // 2) if bz else self.Nred
        out = {"chi0_ph": np.empty(n, dtype=np.complex128), "chi0_pp": np.empty(n, dtype=np.complex128),
               "chi0_ph_FF": np.empty((n, 4), dtype=np.complex128, order="F"),
               "chi0_pp_FF": np.empty((n, 4), dtype=np.complex128, order="F")}
        self._call("tups_get_chi0", int(bool(bz)), *(_ptr(out[k]) for k in ("chi0_ph", "chi0_pp", "chi0_ph_FF",
                                                                           "chi0_pp_FF")))
        return out

    def sus(self, channel, bz: bool = False) -> np.ndarray:
        """sus_r_IBZ (Nred, 4) or, with bz, sus_r (Nx*Ny*Nf/2, 4)."""
        ch = CHANNELS.index(channel) if isinstance(channel, str) else int(channel)
        n = self.Nc * (self.Nf // 2) if bz else self.Nred
        a = np.empty((n, 4), dtype=np.complex128, order="F")
        self._call("tups_get_sus", ch, int(bool(bz)), _ptr(a))
        return a

    # -- instrumentation --
    def set_timing(self, enable: bool) -> None:
        self._call("tups_set_timing", int(bool(enable)))

    def phase_times(self) -> dict:
        """Accumulated device milliseconds and launch counts per phase."""
        ms = (C.c_double * len(_lib.PHASES))()
        cnt = (C.c_int * len(_lib.PHASES))()
        self._call("tups_get_phase_times", C.cast(ms, C.c_void_p), C.cast(cnt, C.c_void_p))
        return {p: (ms[i], cnt[i]) for i, p in enumerate(_lib.PHASES)}

    def record_event(self, slot: int) -> None:
        self._call("tups_record_event", int(slot))

    def event_elapsed_ms(self, a: int, b: int) -> float:
        v = C.c_double()
        self._call("tups_event_elapsed", int(a), int(b), C.byref(v))
        return v.value

    def get_sigma_into(self, out: np.ndarray) -> None:
        """D2H of Sigma into a caller-owned (e.g. pinned) complex128 buffer."""
        assert out.dtype == np.complex128 and out.size == self.Nt and out.flags.c_contiguous
        self._call("tups_get_sigma", _ptr(out))

    def set_sigma_from(self, buf: np.ndarray) -> None:
        """H2D of Sigma from a caller-owned (e.g. pinned) complex128 buffer."""
        assert buf.dtype == np.complex128 and buf.size == self.Nt and buf.flags.c_contiguous
        self._call("tups_set_sigma", _ptr(buf))

    # -- state in reference layouts --
    @property
    def Sigma(self) -> np.ndarray:
        a = np.empty(self.Nt, dtype=np.complex128)
        self._call("tups_get_sigma", _ptr(a))
        return a

    @Sigma.setter
    def Sigma(self, v) -> None:
        a = np.ascontiguousarray(v, dtype=np.complex128).reshape(self.Nt)
        self._call("tups_set_sigma", _ptr(a))

    @property
    def SigmaOld(self) -> np.ndarray:
        a = np.empty(self.Nt, dtype=np.complex128)
        self._call("tups_get_sigma_old", _ptr(a))
        return a

    @property
    def Gkw(self) -> np.ndarray:
        a = np.empty(self.Nt, dtype=np.complex128)
        self._call("tups_get_Gkw", _ptr(a))
        return a

    @property
    def Grt(self) -> np.ndarray:
        n1 = self.Nx * self.Ngrain
        a = np.empty((n1, n1, self.Nf), dtype=np.complex128, order="F")
        self._call("tups_get_Grt", _ptr(a))
        return a

    @property
    def mu(self) -> float:
        v = C.c_double()
        self._call("tups_get_mu", C.byref(v))
        return v.value

    @mu.setter
    def mu(self, v: float) -> None:
        self._call("tups_set_mu", C.c_double(v))

    def _vertex(self, channel, which: int) -> np.ndarray:
        ch = CHANNELS.index(channel) if isinstance(channel, str) else int(channel)
        a = np.empty((self.Nz, self.Nz, self.Nb), dtype=np.complex128, order="F")
        self._call("tups_get_vertex", ch, which, _ptr(a))
        return a

    def F(self, channel) -> np.ndarray:
        """Complete vertex F_r, (Nz, Nz, Nb)."""
        return self._vertex(channel, 0)

    def G(self, channel) -> np.ndarray:
        """G_r array: Gamma_r, or Phi_r between BSE and the vertex update."""
        return self._vertex(channel, 1)

    def vertex_slots(self, channel, which: int, slot_begin: int, count: int = 1) -> np.ndarray:
        """F_r (which 0) or G_r (which 1) of `count` consecutive local slots
        from the 0-based `slot_begin`: (Nz, Nz, count)."""
        ch = CHANNELS.index(channel) if isinstance(channel, str) else int(channel)
        a = np.empty((self.Nz, self.Nz, count), dtype=np.complex128, order="F")
        self._call("tups_get_vertex_slots", ch, which, slot_begin, count, _ptr(a))
        return a

    def set_vertex_slots(self, channel, which: int, slot_begin: int, v: np.ndarray) -> None:
        ch = CHANNELS.index(channel) if isinstance(channel, str) else int(channel)
        a = np.asfortranarray(v, dtype=np.complex128)
        if a.ndim == 2:
            a = a[:, :, None]
        self._call("tups_set_vertex_slots", ch, which, slot_begin, a.shape[2], _ptr(a))

    def set_vertex(self, channel, which: int, v: np.ndarray) -> None:
        ch = CHANNELS.index(channel) if isinstance(channel, str) else int(channel)
        a = np.asfortranarray(v, dtype=np.complex128)
        self._call("tups_set_vertex", ch, which, _ptr(a))

    def save_state(self, path, ite: int) -> None:
        """Checkpoint for a resume in another process: Sigma, mu and the
        vertices F_r and G_r (Gamma_r after the vertex update) to an ``.npz``
        file, with ``ite``, the next iteration to run.  Every other piece of
        device state is recomputed by the next iteration (Phi(R), the phase
        tables and the crossing tensors on the first iteration of a new
        context), so a resumed loop repeats the uninterrupted one bit for bit;
        only the first conv after it reports no change of max|F_r| (that
        comparison is host state).  Holds 8 Nz^2 Nb complex values in host
        memory."""
        np.savez(path, ite=ite, Sigma=self.Sigma, mu=self.mu,
                 F=np.stack([self.F(r) for r in CHANNELS]), G=np.stack([self.G(r) for r in CHANNELS]),
                 shape=np.array([self.Nz, self.Nb, self.Nt, self.slot0]))

    def load_state(self, path) -> int:
        """Restore a ``save_state`` file into this context (same parameters and
        slots); returns the iteration to run next."""
        d = np.load(path)
        if tuple(d["shape"]) != (self.Nz, self.Nb, self.Nt, self.slot0):
            raise ValueError(f"{path} holds a state of other sizes {tuple(d['shape'])}")
        self.Sigma = d["Sigma"]
        self.mu = float(d["mu"])
        for i, r in enumerate(CHANNELS):
            self.set_vertex(r, 0, d["F"][i])
            self.set_vertex(r, 1, d["G"][i])
        return int(d["ite"])

    def PhiR(self, channel) -> np.ndarray:
        ch = CHANNELS.index(channel) if isinstance(channel, str) else int(channel)
        a = np.empty((self.Nz * self.Nz, self.Nf // 2, self.NR), dtype=np.complex128, order="F")
        self._call("tups_get_PhiR", ch, _ptr(a))
        return a

    def M(self, which: int) -> np.ndarray:
        nl = self.Nl
        a = np.empty((nl, nl, nl, nl, self.Nb, self.NR), dtype=np.complex128, order="F")
        self._call("tups_get_M", int(which), _ptr(a))
        return a

    def expSqR(self) -> np.ndarray:
        a = np.empty((self.NIBZ, self.NR, 8), dtype=np.complex128, order="F")
        self._call("tups_get_expSqR", _ptr(a))
        return a

    def expqSR(self) -> np.ndarray:
        a = np.empty((self.Nc, self.NR, 8), dtype=np.complex128, order="F")
        self._call("tups_get_expqSR", _ptr(a))
        return a

    def tables(self) -> dict:
        nl, nx = self.Nl, self.Nx
        FF = np.empty((nx, nx, nl), order="F")
        FFi = np.empty((8, nx, nx, nl), order="F")
        signs = np.empty(nl, dtype=np.int32)
        reps = np.empty(nl, dtype=np.int32)
        lsym = np.empty((8, nl), dtype=np.int32, order="F")
        lfac = np.empty((8, nl), order="F")
        ibz = np.empty((3, self.Nred), dtype=np.int32, order="F")
        self._call("tups_get_tables", *(_ptr(x) for x in (FF, FFi, signs, reps, lsym, lfac, ibz)))
        return {"FF": FF, "FF_inv": FFi, "signs": signs, "reps": reps, "lsym": lsym, "lfac": lfac,
                "ibz": ibz.T.copy()}

    def sde_aux(self) -> dict:
        na = (self.Nl * self.nbox, self.Nb)
        nz = (self.Nz, self.Nb)
        out = {k: np.empty(s, dtype=np.complex128, order="F") for k, s in
               (("chi_aux_ph", na), ("chi_aux_pp", na), ("LChi", nz), ("PhChi", nz), ("PPChi", nz))}
        self._call("tups_get_sde_aux", *(_ptr(out[k]) for k in ("chi_aux_ph", "chi_aux_pp", "LChi", "PhChi",
                                                                "PPChi")))
        return out


def _conv_dict(ci: tups_conv_info) -> dict:
    d = {"rel_sig_max": ci.rel_sig_max, "rel_sig_av": ci.rel_sig_av, "dsigma_inf": ci.dsigma_inf,
         "mu": ci.mu, "bisection_steps": ci.bisection_steps, "converged": bool(ci.converged)}
    for i, r in enumerate(CHANNELS):
        d[f"F_{r}_max"] = ci.F_max[i]
        d[f"rel_err_{r}"] = ci.rel_err[i]
    return d


def set_tuning(key_prefix: str | None, name: str | None) -> None:
    """Fix the tuner candidate ``name`` for every key starting with
    ``key_prefix`` in this process (``name=None`` drops the prefix,
    ``key_prefix=None`` drops all); candidates write the same bits."""
    lib = _lib.load()
    rc = lib.tups_set_tuning(None if key_prefix is None else key_prefix.encode(),
                             None if name is None else name.encode())
    if rc != 0:
        raise RuntimeError(f"tups_set_tuning failed: {rc}")


def tuning_table() -> list[str]:
    """The tile-shape tuner's choices in this process, one line per kernel
    and shape: ``key | choice NAME | NAME=ms ...``."""
    lib = _lib.load()
    n = lib.tups_get_tuning(None, 0)
    buf = C.create_string_buffer(max(1, n))
    lib.tups_get_tuning(buf, len(buf))
    return [ln for ln in buf.value.decode().splitlines() if ln]

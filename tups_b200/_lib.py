"""ctypes binding of the C ABI declared in ``include/tups_b200.h``.

The library is loaded from this package directory only.  There is no
fallback: if ``libtups_b200.so`` is missing or fails to load, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtups_b200.so"

TUPS_OK = 0
STATUS = {
    -1: "TUPS_ERR_CUDA", -2: "TUPS_ERR_OOM", -3: "TUPS_ERR_MU_NOCONV", -4: "TUPS_ERR_NAN",
    -5: "TUPS_ERR_TIMEOUT", -6: "TUPS_ERR_BADDIM", -7: "TUPS_ERR_BADARG", -8: "TUPS_ERR_IO",
    -9: "TUPS_ERR_STATE",
}


class TupsError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class tups_params(C.Structure):
    _fields_ = [
        ("beta", C.c_double), ("U", C.c_double), ("nParticle", C.c_double),
        ("Nx", C.c_int), ("Nf", C.c_int), ("neighbours", C.c_int), ("readinpick", C.c_int),
        ("pick_file", C.c_char * 256), ("Ngrain", C.c_int), ("f_range", C.c_int),
        ("f_damping", C.c_double), ("ite_max", C.c_int), ("DGA", C.c_int),
        ("fname_L", C.c_char * 256), ("use_sig_dmft", C.c_int), ("fname_sig_dmft", C.c_char * 256),
        ("use_U2", C.c_int), ("save_F", C.c_int), ("oneshot", C.c_int), ("old", C.c_int),
        ("SDE_old", C.c_int), ("tprime", C.c_double), ("conv_abs", C.c_double),
    ]


class tups_dims(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("Nx", "Ny", "Nf", "Ngrain", "Nx_IBZ", "NIBZ", "Nred", "Nc", "Nl",
                                       "Nz", "Nt", "Nb", "NR", "nbox", "wperTask")]


class tups_conv_info(C.Structure):
    _fields_ = [("rel_sig_max", C.c_double), ("rel_sig_av", C.c_double), ("dsigma_inf", C.c_double),
                ("F_max", C.c_double * 4), ("rel_err", C.c_double * 4), ("mu", C.c_double),
                ("bisection_steps", C.c_int), ("converged", C.c_int)]


# int (*)(void* user, int what, double* data, size_t count, int op): the host
# exchange of a sharded context (tups_set_exchange)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_int)

# (name, argtypes); every function returns int unless listed in _SPECIAL
_PROTOS = {
    "tups_read_prms": [C.c_char_p, C.POINTER(tups_params)],
    "tups_ctx_create": [C.POINTER(tups_params), C.c_int, C.POINTER(C.c_void_p)],
    "tups_ctx_create_sharded": [C.POINTER(tups_params), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "tups_set_exchange": [C.c_void_p, C.c_void_p, C.c_void_p],
    "tups_iteration_readout": [C.c_void_p, C.c_int, C.c_void_p],
    "tups_read_lambda": [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "tups_get_shard": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "tups_ctx_destroy": [C.c_void_p],
    "tups_host_tables": [C.POINTER(tups_params), C.POINTER(tups_dims)] + [C.c_void_p] * 7,
    "tups_get_dims": [C.c_void_p, C.POINTER(tups_dims)],
    "tups_calc_Gkw_Grt": [C.c_void_p, C.c_int, C.c_int],
    "tups_calc_chi": [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
    "tups_BSE": [C.c_void_p, C.c_int],
    "tups_calculate_expSqR": [C.c_void_p],
    "tups_calculate_expqSR": [C.c_void_p],
    "tups_calc_PhiR": [C.c_void_p, C.c_int],
    "tups_calc_M_phbar_to_ph": [C.c_void_p],
    "tups_calc_M_pp_to_ph": [C.c_void_p],
    "tups_calc_M_ph_to_pp": [C.c_void_p],
    "tups_calc_M_phbar_to_pp": [C.c_void_p],
    "tups_calculate_PAE": [C.c_void_p],
    "tups_calc_SDE": [C.c_void_p, C.c_int],
    "tups_conv": [C.c_void_p, C.POINTER(tups_conv_info)],
    "tups_vertex_update": [C.c_void_p],
    "tups_output_block": [C.c_void_p],
    "tups_iteration": [C.c_void_p, C.c_int, C.POINTER(tups_conv_info)],
    "tups_execute_loop": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "tups_warm_start": [C.c_void_p, C.c_void_p, C.c_void_p],
    "tups_checkpoint": [C.c_void_p, C.c_int],
    "tups_readout": [C.c_void_p, C.c_int],
    "tups_get_chi0": [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "tups_get_sus": [C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "tups_get_sigma": [C.c_void_p, C.c_void_p],
    "tups_set_sigma": [C.c_void_p, C.c_void_p],
    "tups_get_sigma_old": [C.c_void_p, C.c_void_p],
    "tups_get_Gkw": [C.c_void_p, C.c_void_p],
    "tups_get_Grt": [C.c_void_p, C.c_void_p],
    "tups_get_mu": [C.c_void_p, C.POINTER(C.c_double)],
    "tups_set_mu": [C.c_void_p, C.c_double],
    "tups_get_vertex": [C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "tups_set_vertex": [C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "tups_get_vertex_slots": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "tups_set_vertex_slots": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p],
    "tups_set_autotune": [C.c_void_p, C.c_int],
    "tups_set_crossing_products": [C.c_void_p, C.c_int],
    "tups_set_split_wait": [C.c_longlong, C.c_int],
    "tups_set_split_tile": [C.c_int],
    "tups_set_split_cta_pairs": [C.c_int],
    "tups_bse_lu_split_batched": [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                  C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.POINTER(C.c_int), C.c_void_p],
    "tups_get_tuning": [C.c_char_p, C.c_size_t],
    "tups_set_tuning": [C.c_char_p, C.c_char_p],
    "tups_get_PhiR": [C.c_void_p, C.c_int, C.c_void_p],
    "tups_get_M": [C.c_void_p, C.c_int, C.c_void_p],
    "tups_get_expSqR": [C.c_void_p, C.c_void_p],
    "tups_get_expqSR": [C.c_void_p, C.c_void_p],
    "tups_get_tables": [C.c_void_p] + [C.c_void_p] * 7,
    "tups_get_sde_aux": [C.c_void_p] + [C.c_void_p] * 5,
    "tups_synchronize": [C.c_void_p],
    "tups_bse_lu_batched": [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                            C.c_void_p],
    "tups_bse_noalloc": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                         C.c_double, C.c_void_p],
    "tups_set_timing": [C.c_void_p, C.c_int],
    "tups_set_bse_precision": [C.c_void_p, C.c_int, C.c_int],
    "tups_set_graph": [C.c_void_p, C.c_int],
    "tups_zgemm_split": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                         C.c_void_p, C.c_size_t, C.c_void_p],
    "tups_mlp_create": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "tups_mlp_destroy": [C.c_void_p],
    "tups_mlp_set_params": [C.c_void_p, C.c_void_p],
    "tups_mlp_get_params": [C.c_void_p, C.c_void_p],
    "tups_mlp_forward": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p],
    "tups_mlp_gradients": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_double)],
    "tups_mlp_train": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                       C.c_ulonglong, C.c_void_p],
    "tups_get_phase_times": [C.c_void_p, C.c_void_p, C.c_void_p],
    "tups_record_event": [C.c_void_p, C.c_int],
    "tups_event_elapsed": [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)],
}

PHASES = ["green", "chi", "bse_prep", "bse_gemm", "phir", "M", "pae", "sde", "conv", "update"]
_SPECIAL = {
    "tups_last_error": ([C.c_void_p], C.c_char_p),
    "tups_strerror": ([C.c_int], C.c_char_p),
    "tups_kernel_launches": ([C.c_void_p], C.c_longlong),
    "tups_mlp_last_error": ([C.c_void_p], C.c_char_p),
    "tups_get_bse_slices": ([C.c_void_p], C.c_int),
    "tups_zgemm_split_workspace": ([C.c_int, C.c_int, C.c_int, C.c_int, C.c_int], C.c_size_t),
    "tups_bse_lu_split_workspace": ([C.c_int, C.POINTER(C.c_int), C.c_int], C.c_size_t),
    "tups_mlp_num_params": ([C.c_void_p], C.c_longlong),
    "tups_mlp_kernel_launches": ([C.c_void_p], C.c_longlong),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (once).  Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m tups_b200.build`")
    lib = C.CDLL(os.fspath(LIB_PATH))
    for name, args in _PROTOS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    for name, (args, res) in _SPECIAL.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return sorted(list(_PROTOS) + list(_SPECIAL))

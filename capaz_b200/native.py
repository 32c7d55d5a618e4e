"""ctypes bindings of libcapaz_b200.so (include/capaz_b200.h).

The library is loaded from capaz_b200/lib/ (built in-tree by
capaz_b200.build).  Loading fails loudly if it is missing: there is no CPU or
pure-Python fallback for any of the entry points.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")
LIBPATH = os.path.join(LIBDIR, "libcapaz_b200.so")

# enum capaz_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED_GRID = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_NO_DEVICE = 5
ERR_NONFINITE = 6
ERR_BAD_STATE = 7
ERR_INI = 8
ERR_UNSUPPORTED = 9

# Largest (ny-2)*max(nz-2,1) that capaz_mass_noalloc accepts.
NOALLOC_MAX_ROWS = 131072
DIAG_SLOTS = 4  # CAPAZ_DIAG_SLOTS

MODEL_DEFAULT = 0
MODEL_BUCKLEY_LEVERETT = 1
MODEL_ENERGY = 2

FORM_FP64 = 0
FORM_FP32C = 1

FLAG_PERCELL_K = 0x1
FLAG_DIAGNOSTICS = 0x2
FLAG_SOURCE_WINDOW = 0x4
FLAG_NO_TMA = 0x8
FLAG_TEST_WAIT_TIMEOUT = 0x10
FLAG_POW_PRODUCTS = 0x20

ADJ_INIT_FROM_M = 0x1

FIELDS = {
    "P_w": 0, "S_n": 1, "S_w": 2, "m": 3, "K": 4, "P_n": 5, "P_g": 6, "S_g": 7,
    "ro_w": 8, "ro_n": 9, "ro_g": 10, "Xi_w": 11, "Xi_n": 12, "Xi_g": 13,
    "ux_w": 14, "uy_w": 15, "uz_w": 16, "ux_n": 17, "uy_n": 18, "uz_n": 19,
    "ux_g": 20, "uy_g": 21, "uz_g": 22, "roS_w": 23, "roS_n": 24, "roS_g": 25,
    "roS_w_old": 26, "roS_n_old": 27, "roS_g_old": 28,
    "T": 29, "H_w": 30, "H_n": 31, "H_g": 32, "H_r": 33, "E": 34, "E_new": 35,
}
FIELD_COUNT = 36
ENERGY_FIELDS = ("T", "H_w", "H_n", "H_g", "H_r", "E", "E_new")


class Params(C.Structure):
    """capaz_params (include/capaz_b200.h)."""

    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("phases", C.c_int32),
        ("form", C.c_int32), ("newton_iterations", C.c_int32), ("source", C.c_int32),
        ("flags", C.c_uint32),
        ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double), ("dt", C.c_double),
        ("beta_w", C.c_double), ("beta_n", C.c_double), ("beta_g", C.c_double),
        ("ro0_w", C.c_double), ("ro0_n", C.c_double), ("ro0_g", C.c_double),
        ("mu_w", C.c_double), ("mu_n", C.c_double), ("mu_g", C.c_double),
        ("g_const", C.c_double), ("P_atm", C.c_double), ("lambda_", C.c_double),
        ("S_wr", C.c_double), ("S_nr", C.c_double), ("S_gr", C.c_double), ("P_d", C.c_double),
        ("S_n_gr", C.c_double), ("S_w_gr", C.c_double), ("S_w_init", C.c_double),
        ("S_n_init", C.c_double), ("porosity", C.c_double), ("K0", C.c_double),
        ("timeX", C.c_double), ("P_top_offset", C.c_double), ("S_n_background", C.c_double),
        ("z_offset", C.c_int32), ("nz_global", C.c_int32),
        ("model", C.c_int32), ("pad_", C.c_int32), ("Q", C.c_double), ("background_Pw", C.c_double),
        ("background_Sn", C.c_double), ("injwell_Pw", C.c_double), ("outwell_Pw", C.c_double),
        ("reserved", C.c_double * 1),
    ]

    def copy(self) -> "Params":
        q = Params()
        C.memmove(C.byref(q), C.byref(self), C.sizeof(Params))
        return q

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k not in ("reserved", "pad_")}

    @property
    def ncell(self) -> int:
        return self.nx * self.ny * self.nz


class Diag(C.Structure):
    """capaz_diag (include/capaz_b200.h)."""

    _fields_ = [("mass", C.c_double * 3), ("max_residual", C.c_double), ("nonfinite_cells", C.c_double)]


# Every entry point declared in include/capaz_b200.h, with its prototype.
_VP = C.c_void_p
PROTOTYPES = {
    "capaz_abi_version": (C.c_int, []),
    "capaz_params_size": (C.c_size_t, []),
    "capaz_diag_size": (C.c_size_t, []),
    "capaz_params_default": (C.c_int, [C.POINTER(Params)]),
    "capaz_params_from_ini": (C.c_int, [C.c_char_p, C.POINTER(Params)]),
    "capaz_params_validate": (C.c_int, [C.POINTER(Params)]),
    "capaz_create": (_VP, [C.POINTER(Params), C.c_int, C.POINTER(C.c_int)]),
    "capaz_destroy": (C.c_int, [_VP]),
    "capaz_get_params": (C.c_int, [_VP, C.POINTER(Params)]),
    "capaz_last_error": (C.c_char_p, [_VP]),
    "capaz_set_field": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "capaz_get_field": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "capaz_set_field_device": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "capaz_get_field_device": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "capaz_init_state": (C.c_int, [_VP, _VP]),
    "capaz_reference_init": (C.c_int, [C.POINTER(Params), _VP, C.c_int, _VP, _VP, _VP, _VP, _VP]),
    "capaz_get_derived": (C.c_int, [_VP, C.c_int, C.c_int, _VP, C.c_int, _VP]),
    "capaz_step": (C.c_int, [_VP, C.c_int, _VP]),
    "capaz_read_diag": (C.c_int, [_VP, C.POINTER(Diag), _VP]),
    "capaz_post_diag": (C.c_int, [_VP, C.c_int, _VP]),
    "capaz_step_post_diag": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "capaz_wait_diag": (C.c_int, [_VP, C.c_int, C.POINTER(Diag)]),
    "capaz_set_dt": (C.c_int, [_VP, C.c_double]),
    "capaz_set_sweep_tile": (C.c_int, [_VP, C.c_int]),
    "capaz_launch_count": (C.c_int64, [_VP]),
    "capaz_batch_create": (_VP, [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "capaz_batch_destroy": (C.c_int, [_VP]),
    "capaz_batch_instance": (_VP, [_VP, C.c_int]),
    "capaz_batch_step": (C.c_int, [_VP, C.c_int, _VP]),
    "capaz_batch_autotune": (C.c_int, [_VP, _VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "capaz_batch_launch_count": (C.c_int64, [_VP]),
    "capaz_batch_get_tuning": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "capaz_batch_set_tuning": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int]),
    "capaz_sync": (C.c_int, [_VP]),
    "capaz_get_plane": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    "capaz_set_plane": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    "capaz_get_plane_raw": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    "capaz_set_plane_raw": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    "capaz_get_reference": (C.c_int, [_VP, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "capaz_set_reference": (C.c_int, [_VP, C.POINTER(C.c_double), C.c_double]),
    "capaz_step_split": (C.c_int, [_VP, _VP, _VP]),
    "capaz_read_permeability_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _VP]),
    "capaz_load_permeability": (C.c_int, [_VP, C.c_char_p]),
    "capaz_generate_media": (C.c_int, [_VP, C.c_ulonglong, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_int]),
    "capaz_write_plot": (C.c_int, [_VP, C.c_char_p, C.c_double]),
    "capaz_save": (C.c_int, [_VP, C.c_char_p, C.c_int]),
    "capaz_restore": (C.c_int, [_VP, C.c_char_p, C.POINTER(C.c_int)]),
    "capaz_adjoint_create": (_VP, [_VP, C.c_int, C.c_int, _VP, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "capaz_adjoint_destroy": (C.c_int, [_VP]),
    "capaz_adjoint_set_observations": (C.c_int, [_VP, _VP, C.c_int, _VP]),
    "capaz_forward_checkpointed": (C.c_int, [_VP, C.POINTER(C.c_double), _VP]),
    "capaz_backward": (C.c_int, [_VP, _VP, _VP, C.c_int, _VP]),
    "capaz_mass_noalloc": (C.c_int, [C.POINTER(Params), _VP, _VP, _VP, _VP, _VP]),
}

_lib = None


def load() -> C.CDLL:
    """Loads libcapaz_b200.so, raising if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(
            f"{LIBPATH} is missing: build it with `python -m capaz_b200.build` "
            "(there is no fallback implementation)")
    lib = C.CDLL(LIBPATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.capaz_params_size() != C.sizeof(Params) or lib.capaz_diag_size() != C.sizeof(Diag):
        raise RuntimeError("capaz_params/capaz_diag layout mismatch between Python and the library")
    _lib = lib
    return lib


class CapazError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"capaz error {code}: {msg}")
        self.code = code


def check(code: int, ctx=None) -> None:
    if code != OK:
        lib = load()
        msg = lib.capaz_last_error(ctx)
        raise CapazError(code, msg.decode() if msg else "")

"""ctypes binding of libpfc_b200.so (the C ABI declared in include/pfc_b200.h).

The shared library is built in-tree (``make -C mcstar-libs_b200``) into
``mcstar_b200/lib/libpfc_b200.so``.  There is no fallback: if the library is missing
or cannot be loaded, every entry point raises, so no CPU or library path can stand in
for the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpfc_b200.so")

PFC_OK, PFC_ERR_INVALID, PFC_ERR_UNSUPPORTED, PFC_ERR_CUDA, PFC_ERR_NOMEM, PFC_ERR_CAPACITY, PFC_ERR_NONFINITE = range(7)
PFC_F32, PFC_F64 = 0, 1
PFC_BOND_NCOL = 14

# Every symbol include/pfc_b200.h declares (checked by the CPU test suite).
EXPORTED = (
    "pfc_create", "pfc_destroy", "pfc_set_stream", "pfc_last_error", "pfc_status_string",
    "pfc_state_bytes", "pfc_workspace_bytes", "pfc_fft_r2c", "pfc_fft_c2r", "pfc_update_eom",
    "pfc_update_eom_with_fen", "pfc_psi3_split", "pfc_norm", "pfc_calc_fen", "pfc_noise_fill_kspace",
    "pfc_noise_fill", "pfc_findpeaks", "pfc_bond_order", "pfc_step", "pfc_free_energy",
    "pfc_profile_enable", "pfc_profile_read", "pfc_findpeaks_static", "pfc_ensemble_create",
    "pfc_ensemble_run", "pfc_ensemble_destroy", "pfc_ensemble_last_error", "pfc_adjoint_workspace_bytes",
    "pfc_sf_loss", "pfc_adjoint_step", "pfc_init_eom_op", "pfc_update_eom_exp", "pfc_update_eom_exp_with_fen",
    "pfc_update_el", "pfc_init_el_op", "pfc_update_el_exp", "pfc_update_eom_py", "pfc_update_eom_hpfcnoise",
    "pfc_gaussian_init", "pfc_kmult_real", "pfc_kmult_imag", "pfc_square", "pfc_write_lowpass_2d",
    "pfc_amplitude_lowpass", "pfc_bond_reserve", "pfc_default_options", "pfc_create_with", "pfc_get_options",
    "pfc_tune", "pfc_step_prop", "pfc_step_host", "pfc_findpeaks_async", "pfc_findpeaks_wait", "pfc_slab_zinv", "pfc_slab_xy", "pfc_slab_zpass",
)

# pfc_propagator
PROPAGATORS = {"conserved": 0, "conserved_exp": 1, "relax": 2, "relax_exp": 3, "conserved_poly": 4,
               "conserved_hpfc": 5}


class PfcError(RuntimeError):
    """A non-zero pfc_status; ``status`` holds the code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class PfcDesc(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("dtype", ctypes.c_int)]


class PfcStepParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("eps", ctypes.c_double), ("mu", ctypes.c_double), ("C", ctypes.c_double),
                ("namp", ctypes.c_double), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("lz", ctypes.c_double), ("seed", ctypes.c_uint64), ("counter", ctypes.c_uint64)]


class PfcOptions(ctypes.Structure):
    _fields_ = [("z_carry", ctypes.c_int), ("x_kernel", ctypes.c_int), ("tiled", ctypes.c_int),
                ("radix_order", ctypes.c_int), ("tile_shift", ctypes.c_int * 4), ("y_kernel", ctypes.c_int)]

    def to_dict(self):
        return {"z_carry": self.z_carry, "x_kernel": self.x_kernel, "tiled": self.tiled,
                "radix_order": self.radix_order, "tile_shift": list(self.tile_shift), "y_kernel": self.y_kernel}

    @classmethod
    def from_dict(cls, d):
        o = cls()
        lib().pfc_default_options(ctypes.byref(o))
        for k in ("z_carry", "x_kernel", "tiled", "radix_order", "y_kernel"):
            if k in d:
                setattr(o, k, int(d[k]))
        if "tile_shift" in d:
            for i, v in enumerate(d["tile_shift"]):
                o.tile_shift[i] = int(v)
        return o


PROFILE_FAMILIES = 5  # PFC_PROFILE_FAMILIES


class PfcProfile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_longlong), ("calls", ctypes.c_longlong * PROFILE_FAMILIES),
                ("ms", ctypes.c_double * PROFILE_FAMILIES), ("xy_variant", ctypes.c_int), ("xy_mode", ctypes.c_int),
                ("z_mode", ctypes.c_int), ("z_variant", ctypes.c_int), ("y_variant", ctypes.c_int)]


_lib = None
_lock = threading.Lock()

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_U64 = ctypes.c_uint64
_SIGS = {
    "pfc_create": ([ctypes.POINTER(PfcDesc), ctypes.POINTER(_P)], _I),
    "pfc_default_options": ([ctypes.POINTER(PfcOptions)], _I),
    "pfc_create_with": ([ctypes.POINTER(PfcDesc), ctypes.POINTER(PfcOptions), ctypes.POINTER(_P)], _I),
    "pfc_get_options": ([_P, ctypes.POINTER(PfcOptions)], _I),
    "pfc_tune": ([ctypes.POINTER(PfcDesc), ctypes.c_char_p, ctypes.POINTER(PfcOptions), ctypes.POINTER(_D)], _I),
    "pfc_destroy": ([_P], _I),
    "pfc_set_stream": ([_P, _P], _I),
    "pfc_last_error": ([_P], ctypes.c_char_p),
    "pfc_status_string": ([_I], ctypes.c_char_p),
    "pfc_state_bytes": ([_P], ctypes.c_size_t),
    "pfc_workspace_bytes": ([_P], ctypes.c_size_t),
    "pfc_fft_r2c": ([_P, _P, _P], _I),
    "pfc_fft_c2r": ([_P, _P, _P], _I),
    "pfc_update_eom": ([_P, _P, _P, _P, _D, _D, _D, _D, _D, _D], _I),
    "pfc_update_eom_with_fen": ([_P, _P, _P, _P, _D, _D, _D, _D, _D, _D], _I),
    "pfc_psi3_split": ([_P, _P, _P, _D, _I], _I),
    "pfc_norm": ([_P, _P], _I),
    "pfc_calc_fen": ([_P, _P, _P, _D, _D, _D, ctypes.POINTER(_D)], _I),
    "pfc_noise_fill_kspace": ([_P, _P, _U64, _U64], _I),
    "pfc_noise_fill": ([_P, _P, _D, _U64, _U64], _I),
    "pfc_findpeaks": ([_P, _P, _D, _P, _I, ctypes.POINTER(_I)], _I),
    "pfc_bond_order": ([_P, _P, _I, _D, _D, _D, _D, _D, _D, _P, _I, ctypes.POINTER(_I)], _I),
    "pfc_bond_reserve": ([_P, _I, ctypes.c_longlong], _I),
    "pfc_step": ([_P, _P, _I, ctypes.POINTER(PfcStepParams)], _I),
    "pfc_step_prop": ([_P, _P, _I, ctypes.POINTER(PfcStepParams), _I, ctypes.POINTER(_D)], _I),
    "pfc_step_host": ([_P, _P, _P, _P, _I, ctypes.POINTER(PfcStepParams)], _I),
    "pfc_findpeaks_async": ([_P, _P, _D, _P, _I, ctypes.POINTER(_I)], _I),
    "pfc_findpeaks_wait": ([_P, ctypes.POINTER(_I)], _I),
    "pfc_slab_zinv": ([_P, _P, _P, _I], _I),
    "pfc_slab_xy": ([_P, _P, _P, _D, _D], _I),
    "pfc_slab_zpass": ([_P, _P, _P, ctypes.POINTER(PfcStepParams), _I, _I, _I], _I),
    "pfc_free_energy": ([_P, _P, _D, _D, _D, _D, _D, _D, _D, ctypes.POINTER(_D)], _I),
    "pfc_profile_enable": ([_P, _I], _I),
    "pfc_profile_read": ([_P, ctypes.POINTER(PfcProfile)], _I),
    "pfc_findpeaks_static": ([_P, _I, _I, _I, _I, _D, _P, _I, ctypes.POINTER(_I), _P], _I),
    "pfc_ensemble_create": ([_I, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(PfcStepParams), _I,
                             ctypes.POINTER(_P)], _I),
    "pfc_ensemble_run": ([_P, _I, _P], _I),
    "pfc_ensemble_destroy": ([_P], _I),
    "pfc_ensemble_last_error": ([_P], ctypes.c_char_p),
    "pfc_adjoint_workspace_bytes": ([_P], ctypes.c_size_t),
    "pfc_sf_loss": ([_P, _P, _P, _P, ctypes.POINTER(_D)], _I),
    "pfc_adjoint_step": ([_P, _P, _P, _P, ctypes.POINTER(PfcStepParams), _P, ctypes.POINTER(_D)], _I),
    "pfc_init_eom_op": ([_P, _P, _D, _D, _D, _D, _D], _I),
    "pfc_update_eom_exp": ([_P, _P, _P, _P, _P, _D, _D, _D, _D, _D], _I),
    "pfc_update_eom_exp_with_fen": ([_P, _P, _P, _P, _P, _D, _D, _D, _D, _D], _I),
    "pfc_update_el": ([_P, _P, _P, _D, _D, _D, _D, _D, ctypes.POINTER(_D)], _I),
    "pfc_init_el_op": ([_P, _P, _D, _D, _D, _D, _D], _I),
    "pfc_update_el_exp": ([_P, _P, _P, _P, ctypes.POINTER(_D)], _I),
    "pfc_update_eom_py": ([_P, _P, _P, _P, _D, _D, _D, _D, _D, _D], _I),
    "pfc_update_eom_hpfcnoise": ([_P, _P, _P, _P, _P, _P, _D, _D, _D, _D, _D, _D], _I),
    "pfc_gaussian_init": ([_P, _P, _D, _D, _D, _D, _D, _D, _D], _I),
    "pfc_kmult_real": ([_P, _P, _P], _I),
    "pfc_kmult_imag": ([_P, _P, _P], _I),
    "pfc_square": ([_P, _P], _I),
    "pfc_write_lowpass_2d": ([_P, _P, _P, _D, _D, ctypes.c_char_p], _I),
    "pfc_amplitude_lowpass": ([_P, _P, _P, _P, _D, _D, ctypes.c_char_p], _I),
}


def lib():
    """The loaded library (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise OSError(f"libpfc_b200.so not built: {LIB_PATH} is missing "
                                  f"(run `make -C mcstar-libs_b200` or __graft_entry__.build())")
                L = ctypes.CDLL(LIB_PATH)
                for name, (argt, rest) in _SIGS.items():
                    fn = getattr(L, name)
                    fn.argtypes = argt
                    fn.restype = rest
                _lib = L
    return _lib


def check(status, ctx=None, what=""):
    if status != PFC_OK:
        msg = lib().pfc_status_string(status).decode()
        if ctx:
            detail = lib().pfc_last_error(ctx).decode()
            if detail:
                msg = f"{msg}: {detail}"
        raise PfcError(status, f"{what}: {msg}" if what else msg)
    return status

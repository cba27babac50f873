"""ctypes binding of libephmc_cuda.so (the C ABI declared in include/ephmc.h).

The shared library is built in-tree by ``electron-phonon-hmc_b200/build.py``.
There is no CPU fallback: loading fails loudly when the library is missing,
and every call raises ``EphmcError`` on a non-OK status.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libephmc_cuda.so")

FORCE_REFERENCE = 0
FORCE_ADJOINT = 1
FORCE_MIXED = 2
MODES = {"reference": FORCE_REFERENCE, "adjoint": FORCE_ADJOINT, "mixed": FORCE_MIXED}

OK = 0
ERR_UNSUPPORTED = 7
WARN_NEGATIVE_DET = 0x1

_D, _U, _P, _I = C.c_double, C.c_uint, C.c_void_p, C.c_int


class EphmcError(RuntimeError):
    def __init__(self, status, what, message=""):
        self.status = status
        super().__init__(f"{what}: status {status} ({message})")


class Flags(C.Structure):
    """organic_flags (simulation/organic_flags.h:4-14), same layout."""
    _fields_ = [("schur_form_inv", C.c_int), ("zero_filling", C.c_int), ("static_disorder", C.c_int),
                ("single_particle", C.c_int), ("constant_force", C.c_int), ("no_fourier_acc", C.c_int),
                ("classical_fourier_acc", C.c_int), ("cfa_steps", C.c_uint), ("cfa_mass", C.c_double)]


_lib = None


def load_library(path: str | None = None, build_if_missing: bool = True):
    """Load (building if needed) libephmc_cuda.so and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path) and build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_ephmc_build", os.path.join(PKG_ROOT, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing; run electron-phonon-hmc_b200/build.py")
    lib = C.CDLL(path)

    def sig(name, res, args):
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args

    sig("ephmc_last_status", _I, [])
    sig("ephmc_last_warnings", _U, [])
    sig("ephmc_status_string", C.c_char_p, [_I])
    sig("ephmc_last_error_message", C.c_char_p, [])
    sig("ephmc_version", C.c_char_p, [])
    sig("ephmc_ctx_create", _I, [C.POINTER(_P), _U, _U, _U, _P, _P, _D, _D, _U, _P, _I])
    sig("ephmc_ctx_create_nnt", _I, [C.POINTER(_P), _P, _U, _U, _P, _P, _D, _D, _U, _P, _I])
    sig("ephmc_ctx_destroy", _I, [_P])
    sig("ephmc_ctx_set_params", _I, [_P, _P, _P, _D, _D, _U])
    sig("ephmc_ctx_set_flags", _I, [_P, _P])
    sig("ephmc_ctx_set_checkpoint", _I, [_P, _U])
    sig("ephmc_ctx_set_segment", _I, [_P, _U])
    sig("ephmc_ctx_set_stabilize", _I, [_P, _I])
    sig("ephmc_ctx_memory", _I, [_P, C.POINTER(C.c_size_t)])
    sig("ephmc_ctx_autotune", _I, [_P, _P, _I, C.POINTER(C.c_float), C.POINTER(C.c_float)])
    sig("ephmc_ctx_tuning", _I, [_P, C.POINTER(C.c_int)])
    sig("ephmc_ctx_lattice", _I, [_P, _P])
    sig("ephmc_ctx_set_stream", _I, [_P, _P])
    sig("ephmc_eval", _I, [_P, _P, _P, C.POINTER(_D), _I])
    sig("ephmc_construct_M_hat", _I, [_P, _P, _P])
    sig("ephmc_batch_eval", _I, [C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_D), _U, _I])
    sig("ephmc_leapfrog", _I, [_P, _P, _P, _U, _D, _I, C.POINTER(_U)])
    sig("ephmc_leapfrog_graph", _I, [_P, _P, _P, _U, _D, _I, C.POINTER(_U)])
    sig("ephmc_logdet_inverse", _I, [_P, _P, _P, C.POINTER(_D), C.POINTER(_I)])
    sig("ephmc_ctx_get_inverse", _I, [_P, _P])
    sig("ephmc_ctx_last_timings", _I, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)])
    sig("ephmc_fa_evolve", _I, [_P, _P, _P, _D])
    sig("ephmc_fa_approx_step", _I, [_P, _P, _P, _D])
    sig("ephmc_fa_scale_momenta", _I, [_P, _P])
    sig("ephmc_fa_scale_free_bosons", _I, [_P, _P])
    sig("ephmc_fa_energy", _I, [_P, _P, C.POINTER(_D)])
    sig("ephmc_hamilton", _I, [_P, _P, _D, _D, C.POINTER(_D)])
    sig("ephmc_tl_create", _I, [C.POINTER(_P), _U, _U, _U, _P, _P, _D, _P, _U, _I])
    sig("ephmc_tl_destroy", _I, [_P])
    sig("ephmc_tl_set_stream", _I, [_P, _P])
    sig("ephmc_tl_default_width", _I, [_P, C.POINTER(_D)])
    sig("ephmc_tl_run", _I, [_P, _P, _U, _D, _P, _P])
    sig("ephmc_tl_last_timings", _I, [_P, C.POINTER(C.c_float)])
    sig("ephmc_conv_sigma_w", _I, [_P, _U, _D, _P, _U, _P])
    sig("ephmc_conv_sigma_t", _I, [_P, _U, _D, _P, _U, _U, _U, _P])
    sig("ephmc_alloc", _P, [C.c_size_t])
    sig("ephmc_free", None, [_P])
    sig("ephmc_device_synchronize", _I, [])
    sig("ephmc_launch_count", C.c_ulonglong, [])
    sig("ephmc_measure_fma_peak", _I, [_I, C.POINTER(C.c_float)])
    _lib = lib
    return lib


def check(status: int, what: str):
    if status != OK:
        lib = load_library()
        msg = lib.ephmc_last_error_message()
        raise EphmcError(status, what, msg.decode() if msg else "")


def ptr(a):
    """Raw pointer of a numpy array (host) or a torch tensor (device or host)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported buffer type {type(a)}")

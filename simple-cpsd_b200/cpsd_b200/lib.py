"""ctypes binding of include/cpsd_b200.h (the in-tree libcpsd_b200.so).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

CPSD_OK = 0
CPSD_ERR_CUDA = 1
CPSD_ERR_ARG = 2
CPSD_ERR_GRID = 3
CPSD_ERR_BANDS = 4
CPSD_ERR_EMPTY_MASK = 5
CPSD_ERR_UNMASKED_PSI = 6
CPSD_ERR_MOVE = 7
CPSD_ERR_TIMEOUT = 8
CPSD_ERR_SCRATCH = 9
CPSD_WARN_LAGRANGE = 10
CPSD_ERR_EIG = 11
CPSD_ERR_IO = 12

CPSD_PREC_FP64 = 0
CPSD_PREC_MIXED = 1

CPSD_GEMM_FP64 = 0
CPSD_GEMM_TF32X3 = 1
CPSD_GEMM_TF32X3_OVERLAPS = 3

# every symbol include/cpsd_b200.h declares
EXPORTS = [
    "cpsd_gpu_strerror", "cpsd", "cpsd_gpu_cpsd", "cr_fft3b_", "rc_fft3f_", "cpsd_gpu_fft_status",
    "cpsd_gpu_create", "cpsd_gpu_set_scalars", "cpsd_gpu_set_tables", "cpsd_gpu_set_state",
    "cpsd_gpu_run", "cpsd_gpu_get_state", "cpsd_gpu_npw", "cpsd_gpu_launches_per_step",
    "cpsd_gpu_geometry",
    "cpsd_gpu_lagrange_failures", "cpsd_gpu_counters", "cpsd_gpu_use_graphs",
    "cpsd_gpu_set_precision",
    "cpsd_gpu_dropin_context", "cpsd_gpu_phase_timing", "cpsd_gpu_phase_times",
    "cpsd_gpu_phase_name", "cpsd_gpu_stream", "cpsd_gpu_destroy", "cpsd_gpu_batch_create",
    "cpsd_gpu_batch_run", "cpsd_gpu_batch_counters", "cpsd_gpu_batch_stream", "cpsd_gpu_batch_destroy",
    "cpsd_mlp_nparams", "cpsd_mlp_create", "cpsd_mlp_forward", "cpsd_mlp_gradient", "cpsd_mlp_train",
    "cpsd_mlp_get_params", "cpsd_mlp_set_params", "cpsd_mlp_destroy", "cpsd_gpu_set_preconditioner",
    "cpsd_gpu_set_preconditioner_range", "cpsd_gpu_save_orbitals", "cpsd_gpu_restore_orbitals",
    "cpsd_gpu_get_packed", "cpsd_gpu_set_packed", "cpsd_gpu_get_sphere", "cpsd_gpu_set_gemm",
    "cpsd_overlap_tn", "cpsd_overlap_tn_noalloc", "cpsd_gpu_epilogue", "cpsd_write_elcout",
    "cpsd_write_ionout", "cpsd_gpu_kbpp", "cpsd_makepsi",
    "cpsd_gpu_get_tuning", "cpsd_gpu_set_tuning", "cpsd_gpu_tuning_limits", "cpsd_gpu_autotune",
    "cpsd_gpu_set_band_range", "cpsd_gpu_step_phase", "cpsd_gpu_bp_buffers", "cpsd_gpu_bp_finish",
    "cpsd_gpu_run_guarded",
]


class Params(ctypes.Structure):
    _fields_ = [
        ("nfft", _I), ("ispin", _I), ("ne", _I * 2), ("nion", _I), ("nkatm", _I), ("nsh", _I),
        ("precision", _I), ("device", _I), ("unitg", _D * 9), ("omega", _D), ("dt", _D),
        ("fmass", _D), ("cewald", _D), ("rcut", _D),
    ]


class Tuning(ctypes.Structure):
    """cpsd_gpu_tuning of include/cpsd_b200.h."""
    _fields_ = [("plane_occupancy", _I * 4), ("tn_ctas_per_sm", _I), ("density_chunks", _I),
                ("lagrange_solver", _I)]

    def as_dict(self) -> dict:
        return {"plane_occupancy": list(self.plane_occupancy), "tn_ctas_per_sm": self.tn_ctas_per_sm,
                "density_chunks": self.density_chunks, "lagrange_solver": self.lagrange_solver}


class CpsdError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__("%s: status %d (%s)" % (what, status, strerror(status)))


_lib = None


def load(path: str = LIB) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            "%s is missing: build it with `python -m cpsd_b200.build` "
            "(there is no CPU fallback)" % path)
    lib = ctypes.CDLL(path)
    lib.cpsd_gpu_strerror.restype = ctypes.c_char_p
    lib.cpsd_gpu_strerror.argtypes = [_I]
    lib.cpsd_gpu_create.argtypes = [ctypes.POINTER(Params), _P, ctypes.POINTER(_P)]
    lib.cpsd_gpu_set_scalars.argtypes = [_P, _P, _D, _D, _D, _D, _D]
    lib.cpsd_gpu_set_tables.argtypes = [_P] + [_P] * 12
    lib.cpsd_gpu_set_state.argtypes = [_P, _P, _P]
    lib.cpsd_gpu_run.argtypes = [_P, _I, _I, _P, _P, _P, _P]
    lib.cpsd_gpu_get_state.argtypes = [_P] + [_P] * 9
    lib.cpsd_gpu_epilogue.argtypes = [_P, _P, _P, _P]
    lib.cpsd_gpu_kbpp.argtypes = [_D, _I, _I, _D, _P, _P, _P, _I, _P, _P, _P, _P]
    lib.cpsd_makepsi.argtypes = [_I, _I, _P, _P, _P]
    lib.cpsd_write_elcout.argtypes = [ctypes.c_char_p, _I, _I, _D, _I, _P, _P]
    lib.cpsd_write_ionout.argtypes = [ctypes.c_char_p, _I, ctypes.POINTER(ctypes.c_char_p), _P, _I, _P, _P]
    lib.cpsd_gpu_npw.argtypes = [_P]
    lib.cpsd_gpu_launches_per_step.argtypes = [_P]
    lib.cpsd_gpu_geometry.argtypes = [_P, _P]
    lib.cpsd_gpu_lagrange_failures.argtypes = [_P]
    lib.cpsd_gpu_counters.argtypes = [_P, _P]
    lib.cpsd_gpu_counters.restype = None
    lib.cpsd_gpu_use_graphs.argtypes = [_P, _I]
    lib.cpsd_gpu_set_precision.argtypes = [_P, _I]
    lib.cpsd_gpu_dropin_context.restype = _P
    lib.cpsd_gpu_phase_timing.argtypes = [_P, _I]
    lib.cpsd_gpu_phase_times.argtypes = [_P, _P, _I]
    lib.cpsd_gpu_phase_name.argtypes = [_I]
    lib.cpsd_gpu_phase_name.restype = ctypes.c_char_p
    lib.cpsd_gpu_stream.argtypes = [_P]
    lib.cpsd_gpu_stream.restype = _P
    lib.cpsd_gpu_batch_create.argtypes = [_P, _I, ctypes.POINTER(_P)]
    lib.cpsd_gpu_batch_run.argtypes = [_P, _I, _P, _P, _P]
    lib.cpsd_gpu_batch_counters.argtypes = [_P, _P]
    lib.cpsd_gpu_batch_counters.restype = None
    lib.cpsd_gpu_batch_stream.argtypes = [_P]
    lib.cpsd_gpu_batch_stream.restype = _P
    lib.cpsd_gpu_batch_destroy.argtypes = [_P]
    lib.cpsd_gpu_batch_destroy.restype = None
    lib.cpsd_mlp_create.argtypes = [ctypes.c_ulonglong, ctypes.POINTER(_P)]
    lib.cpsd_mlp_forward.argtypes = [_P, _P, _I, _P]
    lib.cpsd_mlp_gradient.argtypes = [_P, _P, _P, _I, _P, _P]
    lib.cpsd_mlp_train.argtypes = [_P, _P, _P, _I, _I, _I, ctypes.c_float, _P]
    lib.cpsd_mlp_get_params.argtypes = [_P, _P]
    lib.cpsd_mlp_set_params.argtypes = [_P, _P]
    lib.cpsd_mlp_destroy.argtypes = [_P]
    lib.cpsd_mlp_destroy.restype = None
    lib.cpsd_gpu_set_preconditioner.argtypes = [_P, _P]
    lib.cpsd_gpu_set_preconditioner_range.argtypes = [_P, _D, _D]
    lib.cpsd_gpu_save_orbitals.argtypes = [_P]
    lib.cpsd_gpu_restore_orbitals.argtypes = [_P]
    lib.cpsd_gpu_get_packed.argtypes = [_P, _P, _P, _P]
    lib.cpsd_gpu_set_packed.argtypes = [_P, _P]
    lib.cpsd_gpu_get_sphere.argtypes = [_P, _P, _P, _P]
    lib.cpsd_gpu_set_gemm.argtypes = [_P, _I]
    lib.cpsd_gpu_get_tuning.argtypes = [_P, ctypes.POINTER(Tuning)]
    lib.cpsd_gpu_set_tuning.argtypes = [_P, ctypes.POINTER(Tuning)]
    lib.cpsd_gpu_tuning_limits.argtypes = [_P, ctypes.POINTER(Tuning)]
    lib.cpsd_gpu_run_guarded.argtypes = [_P, _I, _I, _P, _P, _P, _P, _P]
    lib.cpsd_gpu_set_band_range.argtypes = [_P, _I, _I]
    lib.cpsd_gpu_step_phase.argtypes = [_P, _I]
    lib.cpsd_gpu_bp_buffers.argtypes = [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                                        ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_long)]
    lib.cpsd_gpu_bp_finish.argtypes = [_P, _I, _P, _P, _P]
    lib.cpsd_gpu_autotune.argtypes = [_P, _I, _I, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    _L = ctypes.c_long
    lib.cpsd_overlap_tn.argtypes = [_I, _I, _I, _I, _P, _L, _P, _L, _P, _P, _L, _P]
    lib.cpsd_overlap_tn_noalloc.argtypes = [_I, _I, _I, _I, _P, _L, _P, _L, _P, _P, _L, _P]
    lib.cpsd_gpu_destroy.argtypes = [_P]
    lib.cpsd_gpu_destroy.restype = None
    lib.cpsd_gpu_fft_status.restype = _I
    lib.cr_fft3b_.restype = None
    lib.rc_fft3f_.restype = None
    lib.cpsd.restype = None
    lib.cpsd_gpu_cpsd.restype = _I
    _lib = lib
    return lib


def strerror(status: int) -> str:
    try:
        return load().cpsd_gpu_strerror(int(status)).decode()
    except FileNotFoundError:
        return "library not built"

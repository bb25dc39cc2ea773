"""ctypes binding of the C ABI in include/vpfft_capi.h.

The shared library vpfft_b200/lib/libvpfft_b200.so is built in-tree by
``python -m vpfft_b200.build``.  Loading fails loudly when it is missing:
there is no CPU fallback for any solve.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libvpfft_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "vpfft_capi.h")

NSYS = 12

# vpfft_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED_SIZE = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_NO_DEVICE = 5
ERR_MAX_RSS_TINY = 6
ERR_NONFINITE = 7
ERR_NOT_INITIALIZED = 8
ERR_IO = 9
ERR_CANCELLED = 10
ERR_BUSY = 12
# bits of Stats.status_bits / BatchResult.status_bits (include/vpfft_capi.h)
STATUS_MAX_RSS_TINY = 0x1
STATUS_NONFINITE = 0x2
STATUS_DEVICE_TIMEOUT = 0x4
STATUS_LOOP_NOT_CONVERGED = 0x100
STATUS_NR_CAPPED = 0x200

PREC_FP64 = 0
PREC_MIXED = 1

FIELD_STRESS = 0
FIELD_LAGRANGE = 1
FIELD_ORIENTATION = 2
FIELD_CRSS = 3
FIELD_ACCUMULATED_SHEAR = 4
FIELD_POLARIZATION = 5
FIELD_STRAIN_RATE_VARIATION = 6
FIELD_STRAIN_RATE = 7
FIELD_SCHMID = 8
FIELD_WIDTH = {0: 5, 1: 5, 2: 9, 3: 12, 4: 1, 5: 5, 6: 5, 7: 5, 8: 60}

NUM_PHASES = 7
NOALLOC_MAX_POINTS = 4096

PRINT_STRAIN = 0
PRINT_STRESS = 1
PRINT_LAGRANGE = 2
PRINT_POLARIZATION = 3


class Material(C.Structure):
    _fields_ = [
        ("gamma_dot_base", C.c_double * NSYS),
        ("rate_sensitivity", C.c_int32 * NSYS),
        ("crss", C.c_double * NSYS),
        ("tau0", C.c_double * NSYS),
        ("tau1", C.c_double * NSYS),
        ("theta0", C.c_double * NSYS),
        ("theta1", C.c_double * NSYS),
        ("hardening", C.c_double * (NSYS * NSYS)),
    ]


class SolverOptions(C.Structure):
    _fields_ = [
        ("init_nr_epsilon", C.c_double),
        ("init_nr_max_iter", C.c_int32),
        ("nr_epsilon", C.c_double),
        ("nr_max_resolved", C.c_double),
        ("nr_max_iter", C.c_int32),
        ("green_operator", C.c_int32),
        ("mixed_certify_step", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("stress_error", C.c_double),
        ("strain_rate_error", C.c_double),
        ("avg_strain_rate", C.c_double * 5),
        ("nr_not_converged", C.c_int64),
        ("status_bits", C.c_int32),
        ("pad_", C.c_int32),
        ("seconds_init", C.c_double),
        ("seconds_loop", C.c_double),
        ("seconds_post", C.c_double),
        ("L0", C.c_double * 25),
        ("nr_fp64_steps", C.c_int64),
    ]


class Config(C.Structure):
    _fields_ = [
        ("num_x", C.c_int32), ("num_y", C.c_int32), ("num_z", C.c_int32),
        ("input_strain_rate", C.c_double * 9),
        ("max_nr_iter", C.c_int32),
        ("nr_tolerance", C.c_double),
        ("time_step", C.c_double),
        ("num_time_iter", C.c_int32),
        ("init_method", C.c_int32),
        ("input_microstructure", C.c_char * 1024),
        ("material", Material),
        ("voxel_length", C.c_double * 3),
        ("convergence_epsilon", C.c_double),
        ("max_iter", C.c_int32),
        ("precision", C.c_int32),
    ]


class BatchOptions(C.Structure):
    _fields_ = [
        ("max_slots", C.c_int32),
        ("iterations_per_tick", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("use_graphs", C.c_int32),
        ("fft_tiles", C.c_int32),
    ]


class TileTuning(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("fft_tiles", C.c_int32),
        ("families", C.c_int32),
        ("source", C.c_int32),
        ("ms_per_chain", C.c_double * 3),
    ]


class BatchResult(C.Structure):
    _fields_ = [
        ("request_id", C.c_int64),
        ("status", C.c_int32),
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("status_bits", C.c_int32),
        ("avg_stress", C.c_double * 5),
        ("stress_error", C.c_double),
        ("strain_rate_error", C.c_double),
        ("nr_not_converged", C.c_int64),
        ("seconds_queued", C.c_double),
        ("seconds_total", C.c_double),
    ]


class BatchInfo(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "queued", "active", "completed", "ticks", "graph_replays", "kernel_launches",
        "arena_bytes_in_use", "arena_bytes", "admissions_deferred_for_memory")]


STEP_CALLBACK = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                            C.c_void_p)

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_G = C.c_void_p

_PROTOS = {
    "vpfft_version": (C.c_char_p, []),
    "vpfft_status_string": (C.c_char_p, [C.c_int]),
    "vpfft_device_count": (C.c_int, []),
    "vpfft_material_default": (None, [C.POINTER(Material)]),
    "vpfft_solver_options_default": (None, [C.POINTER(SolverOptions)]),
    "vpfft_grid_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(Material),
                                    C.POINTER(SolverOptions), C.c_int, C.POINTER(_G)]),
    "vpfft_grid_destroy": (C.c_int, [_G]),
    "vpfft_grid_dims": (C.c_int, [_G, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "vpfft_grid_set_fields": (C.c_int, [_G, _D, _D]),
    "vpfft_grid_set_fields_device": (C.c_int, [_G, C.c_void_p, C.c_void_p]),
    "vpfft_grid_set_voxel_length": (C.c_int, [_G, C.c_double, C.c_double, C.c_double]),
    "vpfft_grid_get_voxel_length": (C.c_int, [_G, _D]),
    "vpfft_grid_set_crss": (C.c_int, [_G, _D]),
    "vpfft_grid_get_field": (C.c_int, [_G, C.c_int, _D]),
    "vpfft_grid_set_field": (C.c_int, [_G, C.c_int, _D]),
    "vpfft_grid_snapshot_size": (C.c_int, [_G, C.POINTER(C.c_size_t)]),
    "vpfft_grid_snapshot": (C.c_int, [_G, C.c_void_p, C.c_size_t]),
    "vpfft_grid_restore": (C.c_int, [_G, C.c_void_p, C.c_size_t]),
    "vpfft_run_single_strain_step": (C.c_int, [_G, _D, C.c_int, C.c_double, C.c_double, _D,
                                               C.POINTER(Stats)]),
    "vpfft_run": (C.c_int, [_G, _D, C.c_int, C.c_int, C.c_double, C.c_double, C.c_char_p,
                            STEP_CALLBACK, C.c_void_p]),
    "vpfft_initialize_computation": (C.c_int, [_G, _D]),
    "vpfft_build_reference_medium": (C.c_int, [_G, _D]),
    "vpfft_fixed_point": (C.c_int, [_G, _D, C.c_int, C.c_double, _D, C.POINTER(Stats)]),
    "vpfft_post_increment": (C.c_int, [_G, _D, C.c_double]),
    "vpfft_grid_synchronize": (C.c_int, [_G]),
    "vpfft_grid_stream": (C.c_void_p, [_G]),
    "vpfft_grid_launch_count": (C.c_int64, [_G]),
    "vpfft_last_error": (C.c_char_p, [_G]),
    "vpfft_grid_set_profiling": (C.c_int, [_G, C.c_int]),
    "vpfft_grid_phase_times": (C.c_int, [_G, _D, C.POINTER(C.c_int64)]),
    "vpfft_phase_name": (C.c_char_p, [C.c_int]),
    "vpfft_solve_constitutive": (C.c_int, [C.c_int, _D, _D, _D, C.POINTER(Material), _D,
                                           C.c_double, C.c_double, C.c_int, _D]),
    "vpfft_solve_constrained_constitutive": (C.c_int, [C.c_int, _D, _D, _D, C.POINTER(Material),
                                                       _D, _D, _D, _D, C.c_double, C.c_double,
                                                       C.c_int, _D, _D]),
    "vpfft_solve_constrained_constitutive_noalloc": (
        C.c_int, [C.c_int, _D, _D, _D, C.POINTER(Material), _D, _D, _D, _D, C.c_double,
                  C.c_double, C.c_int, _D, _D, C.POINTER(C.c_int64)]),
    "vpfft_apply_constitutive": (C.c_int, [C.c_int, _D, _D, _D, C.POINTER(Material), _D]),
    "vpfft_solve_sachs": (C.c_int, [C.c_int, _D, _D, _D, _D]),
    "vpfft_schmid_tensors": (C.c_int, [C.c_int, _D, _D]),
    "vpfft_green_apply": (C.c_int, [C.c_int, _I32, C.c_int, C.c_int, C.c_int, _D, _D, _D, _D,
                                    C.c_int]),
    "vpfft_fft3d_r2c": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _D, _D, C.c_int]),
    "vpfft_set_tma_passes": (C.c_int, [C.c_int]),
    "vpfft_grid_green_operator": (C.c_int, [_G, C.POINTER(C.c_int), _D, _D]),
    "vpfft_fft3d_c2r": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _D, _D, C.c_int]),
    "vpfft_fixture_polycrystal": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, _D,
                                            _I32]),
    "vpfft_edot_from_matrix": (None, [_D, _D]),
    "vpfft_matrix_from_edot": (None, [_D, _D]),
    "vpfft_batch_options_default": (None, [C.POINTER(BatchOptions)]),
    "vpfft_batch_create": (C.c_int, [C.c_int, C.POINTER(Material), C.POINTER(SolverOptions),
                                     C.POINTER(BatchOptions), C.POINTER(_G)]),
    "vpfft_batch_destroy": (C.c_int, [_G]),
    "vpfft_batch_submit": (C.c_int, [_G, _G, _D, C.c_int, C.c_double, C.c_double,
                                     C.POINTER(C.c_int64)]),
    "vpfft_batch_step": (C.c_int, [_G, C.POINTER(C.c_int)]),
    "vpfft_batch_run": (C.c_int, [_G]),
    "vpfft_batch_poll": (C.c_int, [_G, C.POINTER(BatchResult), C.c_int, C.POINTER(C.c_int)]),
    "vpfft_batch_cancel": (C.c_int, [_G, C.c_int64]),
    "vpfft_batch_get_info": (C.c_int, [_G, C.POINTER(BatchInfo)]),
    "vpfft_batch_get_tunings": (C.c_int, [_G, C.POINTER(TileTuning), C.c_int,
                                          C.POINTER(C.c_int)]),
    "vpfft_batch_last_error": (C.c_char_p, [_G]),
    "vpfft_print_field": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, _D, _D]),
    "vpfft_grid_print": (C.c_int, [_G, C.c_int, C.c_char_p]),
    "vpfft_write_random_material": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _D, _D]),
    "vpfft_read_random_material": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _D, _D]),
    "vpfft_read_euler_texture": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _D]),
    "vpfft_euler_matrix": (C.c_int, [C.c_double, C.c_double, C.c_double, _D]),
    "vpfft_fixture_two_grain": (C.c_int, [C.c_int, C.c_int, C.c_int, _D]),
    "vpfft_config_read": (C.c_int, [C.c_char_p, C.POINTER(Config), C.c_char_p, C.c_size_t]),
}

_lib = None


def declared_symbols(header: str = HEADER) -> list[str]:
    """Names of the functions declared in include/vpfft_capi.h."""
    txt = open(header).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b(vpfft_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(n for n in names if not n.endswith("_t")))


def load(path: str = LIB_PATH):
    """Load the native library (build it first with python -m vpfft_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"vpfft_b200 native library not found at {path}; build it with "
            "`python -m vpfft_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class VpfftError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"vpfft status {status}: {msg}")
        self.status = status


def check(status: int, grid=None) -> None:
    if status != OK:
        lib = load()
        detail = lib.vpfft_last_error(grid).decode(errors="replace")
        base = lib.vpfft_status_string(status).decode()
        raise VpfftError(status, f"{base}: {detail}" if detail else base)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I32)


def f64(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def material(gamma_dot_base=15.5, rate_sensitivity=10, crss=11.0, tau0=11.0, tau1=11.0,
             theta0=430.0, theta1=110.0, hardening=1.0) -> Material:
    """A Material with scalars broadcast to the 12 systems (defaults are the
    reference's hard-coded values, MaterialGrid.cpp:322-336, 390)."""
    m = Material()
    for name, val in (("gamma_dot_base", gamma_dot_base), ("crss", crss), ("tau0", tau0),
                      ("tau1", tau1), ("theta0", theta0), ("theta1", theta1)):
        arr = np.broadcast_to(np.asarray(val, np.float64), (NSYS,))
        getattr(m, name)[:] = list(arr)
    m.rate_sensitivity[:] = list(np.broadcast_to(np.asarray(rate_sensitivity, np.int32), (NSYS,)))
    m.hardening[:] = list(np.broadcast_to(np.asarray(hardening, np.float64), (NSYS, NSYS)).ravel())
    return m


def solver_options(green_operator: int = 0, mixed_certify_step: float | None = None
                   ) -> SolverOptions:
    """The default solver constants (the reference's, vpfft_solver_options_default)
    with the x pass's Green operator (0 chosen per grid size, 1 computed, 2 stored)
    and, for mixed precision, the bound below which the FP64 residual certifies
    the FP32 predictor's stress (None: the default, 1e-5; 0: the FP64 Newton step
    is always taken)."""
    o = SolverOptions()
    load().vpfft_solver_options_default(C.byref(o))
    o.green_operator = int(green_operator)
    if mixed_certify_step is not None:
        o.mixed_certify_step = float(mixed_certify_step)
    return o


def device_count() -> int:
    return int(load().vpfft_device_count())

"""ctypes binding of libcc_b200.so (the C ABI declared in include/cc_step.h,
include/cc_ic.h, include/cc_batch.h and include/cc_adjoint.h).  Loading fails loudly: there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcc_b200.so"

CC_OK = 0
CC_ERR_ARG = -1
CC_ERR_CUDA = -2
CC_ERR_STATE = -3
CC_ERR_NONFINITE = -4
CC_ERR_NOT_CONVERGED = -5
CC_ERR_UNSUPPORTED = -6
CC_ERR_TOO_LARGE = -7
CC_ERR_IO = -8
CC_NOALLOC_MAX_CELLS = 1 << 18
CC_NOALLOC_MAX_SIDE = 4096

CC_FP64 = 0
CC_FP32 = 1
CC_POISSON_SOR = 0
CC_POISSON_FFT = 1
CC_POISSON_DIRECT = 2
CC_POISSON_SOR_LEX = 5
CC_GRAVITY_ENCLOSED = 3
CC_GRAVITY_SHELLS = 4
CC_BATCH_MAX_DIRECT_SIDE = 2048
CC_STAGE_TILE = 0
CC_STAGE_MARCH = 1


class CcMhd2dParams(C.Structure):
    _fields_ = [
        ("gamma", C.c_double), ("cfl", C.c_double),
        ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
        ("Nx", C.c_int32), ("Ny", C.c_int32),
        ("t_end", C.c_double), ("dt_store", C.c_double),
        ("floor_rho", C.c_double), ("floor_P", C.c_double),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32),
        ("eta", C.c_double),
        ("gravity_on", C.c_int32),
        ("G", C.c_double), ("softening", C.c_double),
        ("sor_iters", C.c_int32), ("sor_omega", C.c_double),
        ("sor_tol", C.c_double),
        ("poisson_kind", C.c_int32), ("precision", C.c_int32), ("compensated", C.c_int32),
    ]


class CcMhd3dParams(C.Structure):
    _fields_ = [
        ("gamma1", C.c_double), ("gamma2", C.c_double), ("K1", C.c_double), ("rho_nuc", C.c_double),
        ("gamma_th", C.c_double), ("rho_bounce", C.c_double), ("gamma_bounce", C.c_double),
        ("Kbounce", C.c_double), ("gamma_init", C.c_double), ("cfl", C.c_double),
        ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
        ("z0", C.c_double), ("z1", C.c_double),
        ("Nx", C.c_int32), ("Ny", C.c_int32), ("Nz", C.c_int32), ("precision", C.c_int32),
        ("t_end", C.c_double), ("dt_store", C.c_double),
        ("floor_rho", C.c_double), ("floor_P", C.c_double),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("periodic_z", C.c_int32), ("reserved", C.c_int32),
        ("eta", C.c_double),
    ]


class CcEuler2dParams(C.Structure):
    _fields_ = [
        ("gamma", C.c_double), ("cfl", C.c_double),
        ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
        ("Nx", C.c_int32), ("Ny", C.c_int32),
        ("t_end", C.c_double), ("dt_store", C.c_double),
        ("floor_rho", C.c_double), ("floor_P", C.c_double),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32),
        ("gravity_on", C.c_int32), ("sor_max_iter", C.c_int32),
        ("G", C.c_double), ("softening", C.c_double),
        ("sor_tol", C.c_double), ("sor_omega", C.c_double),
        ("poisson_kind", C.c_int32), ("precision", C.c_int32),
        ("Nr_bins", C.c_int32), ("reserved", C.c_int32),
        ("xc", C.c_double), ("yc", C.c_double),
    ]


class CcNs2dParams(C.Structure):
    _fields_ = [
        ("gamma", C.c_double), ("cfl", C.c_double),
        ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
        ("Nx", C.c_int32), ("Ny", C.c_int32),
        ("t_end", C.c_double), ("dt_store", C.c_double),
        ("seed", C.c_uint32), ("viscosity_on", C.c_int32),
        ("floor_rho", C.c_double), ("floor_P", C.c_double),
        ("mu", C.c_double), ("cfl_visc", C.c_double),
        ("gravity_on", C.c_int32), ("precision", C.c_int32),
        ("G", C.c_double),
    ]


class CcDiag(C.Structure):
    _fields_ = [
        ("mass", C.c_double), ("mom_x", C.c_double), ("mom_y", C.c_double), ("mom_z", C.c_double),
        ("energy", C.c_double), ("max_divB", C.c_double), ("t", C.c_double), ("dt_last", C.c_double),
        ("steps", C.c_int64), ("poisson_iters", C.c_int32), ("nonfinite", C.c_int32),
        ("poisson_residual", C.c_double),
    ]


class CcPerf(C.Structure):
    _fields_ = [
        ("kernel_launches", C.c_int64), ("stage_launches", C.c_int64), ("stage_ms", C.c_double),
        ("poisson_solves", C.c_int64), ("steps", C.c_int64),
    ]


class CcIc3Knobs(C.Structure):
    _fields_ = [
        ("rho_bg", C.c_double), ("rho_core", C.c_double), ("r_core", C.c_double), ("r_edge", C.c_double),
        ("P0", C.c_double), ("vin", C.c_double), ("rot_omega", C.c_double),
        ("B0x", C.c_double), ("B0z", C.c_double), ("Bshear", C.c_double),
    ]


class CcIcKnobs(C.Structure):
    _fields_ = [
        ("rho_bg", C.c_double), ("rho_core", C.c_double), ("r_core", C.c_double), ("r_edge", C.c_double),
        ("P0", C.c_double), ("vin", C.c_double), ("rot_omega", C.c_double),
        ("B0x", C.c_double), ("Bshear", C.c_double), ("gamma_eff", C.c_double),
    ]


_DP = C.POINTER(C.c_double)
_H = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/*.h
class CcBatchInfo(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("precision", C.c_int32), ("cells", C.c_int64),
        ("shape", C.c_int32), ("n_shapes", C.c_int32), ("tile_x", C.c_int32), ("tile_y", C.c_int32),
        ("stage_tiles", C.c_int32), ("stage_ctas", C.c_int32), ("reduce_tiles", C.c_int32),
        ("poisson_tiles", C.c_int32), ("device_bytes", C.c_int64), ("poisson_tile", C.c_int32),
        ("reserved", C.c_int32),
    ]


SIGNATURES = {
    "cc_mhd2d_params_default": (None, [C.POINTER(CcMhd2dParams)]),
    "cc_mhd2d_create": (C.c_int, [C.POINTER(CcMhd2dParams), C.POINTER(_H)]),
    "cc_destroy": (C.c_int, [_H]),
    "cc_last_error": (C.c_char_p, [_H]),
    "cc_set_stream": (C.c_int, [_H, C.c_void_p]),
    "cc_synchronize": (C.c_int, [_H]),
    "cc_set_profiling": (C.c_int, [_H, C.c_int]),
    "cc_get_perf": (C.c_int, [_H, C.POINTER(CcPerf)]),
    "cc_reset_perf": (C.c_int, [_H]),
    "cc_mhd2d_upload": (C.c_int, [_H] + [_DP] * 8),
    "cc_mhd2d_download": (C.c_int, [_H] + [_DP] * 8),
    "cc_mhd2d_compute_gravity": (C.c_int, [_H, _DP, _DP]),
    "cc_mhd2d_compute_dt": (C.c_int, [_H, _DP]),
    "cc_mhd2d_rk2_step": (C.c_int, [_H, _DP, _DP, C.c_double]),
    "cc_mhd2d_advance": (C.c_int, [_H, C.c_int, _DP]),
    "cc_mhd2d_set_stage_kernel": (C.c_int, [_H, C.c_int, C.c_int]),
    "cc_mhd2d_diagnostics": (C.c_int, [_H, C.POINTER(CcDiag)]),
    "cc_mhd2d_derived": (C.c_int, [_H, C.POINTER(C.POINTER(C.c_double))]),
    "cc_mhd2d_checkpoint_save": (C.c_int, [_H, C.c_char_p]),
    "cc_mhd2d_checkpoint_load": (C.c_int, [_H, C.c_char_p]),
    "cc_mhd2d_gravity_fft_noalloc": (C.c_int, [C.POINTER(CcMhd2dParams), C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p]),
    "cc_mhd3d_params_default": (None, [C.POINTER(CcMhd3dParams)]),
    "cc_mhd3d_create": (C.c_int, [C.POINTER(CcMhd3dParams), C.POINTER(_H)]),
    "cc_mhd3d_upload": (C.c_int, [_H] + [_DP] * 8),
    "cc_mhd3d_download": (C.c_int, [_H] + [_DP] * 8),
    "cc_mhd3d_compute_dt": (C.c_int, [_H, _DP]),
    "cc_mhd3d_rk2_step": (C.c_int, [_H, C.c_double]),
    "cc_mhd3d_advance": (C.c_int, [_H, C.c_int, _DP]),
    "cc_mhd3d_diagnostics": (C.c_int, [_H, C.POINTER(CcDiag)]),
    "cc_mhd3d_derived": (C.c_int, [_H, C.POINTER(C.POINTER(C.c_double))]),
    "cc_euler2d_params_default": (None, [C.POINTER(CcEuler2dParams)]),
    "cc_euler2d_create": (C.c_int, [C.POINTER(CcEuler2dParams), C.POINTER(_H)]),
    "cc_euler2d_upload": (C.c_int, [_H] + [_DP] * 4),
    "cc_euler2d_download": (C.c_int, [_H] + [_DP] * 4),
    "cc_euler2d_compute_dt": (C.c_int, [_H, _DP]),
    "cc_euler2d_compute_gravity": (C.c_int, [_H, _DP, _DP]),
    "cc_euler2d_rk2_step": (C.c_int, [_H, C.c_double]),
    "cc_euler2d_advance": (C.c_int, [_H, C.c_int, _DP]),
    "cc_euler2d_diagnostics": (C.c_int, [_H, C.POINTER(CcDiag)]),
    "cc_euler2d_derived": (C.c_int, [_H, C.POINTER(C.POINTER(C.c_double))]),
    "cc_euler2d_checkpoint_save": (C.c_int, [_H, C.c_char_p]),
    "cc_euler2d_checkpoint_load": (C.c_int, [_H, C.c_char_p]),
    "cc_ns2d_checkpoint_save": (C.c_int, [_H, C.c_char_p]),
    "cc_ns2d_checkpoint_load": (C.c_int, [_H, C.c_char_p]),
    "cc_mhd3d_checkpoint_save": (C.c_int, [_H, C.c_char_p]),
    "cc_mhd3d_checkpoint_load": (C.c_int, [_H, C.c_char_p]),
    "cc_ns2d_params_default": (None, [C.POINTER(CcNs2dParams)]),
    "cc_ns2d_create": (C.c_int, [C.POINTER(CcNs2dParams), C.POINTER(_H)]),
    "cc_ns2d_upload": (C.c_int, [_H] + [_DP] * 4),
    "cc_ns2d_download": (C.c_int, [_H] + [_DP] * 4),
    "cc_ns2d_compute_dt": (C.c_int, [_H, _DP]),
    "cc_ns2d_compute_gravity": (C.c_int, [_H, _DP, _DP, _DP]),
    "cc_ns2d_compute_rhs": (C.c_int, [_H, C.POINTER(_DP)]),
    "cc_ns2d_rk2_step": (C.c_int, [_H, C.c_double]),
    "cc_ns2d_advance": (C.c_int, [_H, C.c_int, _DP]),
    "cc_ns2d_diagnostics": (C.c_int, [_H, C.POINTER(CcDiag)]),
    "cc_ns2d_derived": (C.c_int, [_H, C.POINTER(_DP)]),
    "cc_ic_ns2d_collapse": (C.c_int, [C.POINTER(CcNs2dParams), C.POINTER(_DP)]),
    "cc_mhd2d_ic_knobs_default": (None, [C.POINTER(CcIcKnobs)]),
    "cc_ic_mhd2d_reference": (C.c_int, [C.POINTER(CcMhd2dParams), C.POINTER(CcIcKnobs), C.POINTER(_DP)]),
    "cc_mhd3d_ic_knobs_default": (None, [C.POINTER(CcIc3Knobs)]),
    "cc_ic_mhd3d_reference": (C.c_int, [C.POINTER(CcMhd3dParams), C.POINTER(CcIc3Knobs), C.POINTER(_DP)]),
    "cc_ic_mhd2d_collapse": (C.c_int, [C.POINTER(CcMhd2dParams), C.c_double, C.c_double, C.c_double, C.c_uint32,
                                       C.c_double, C.c_double, C.c_double, C.POINTER(_DP)]),
    "cc_ic_mhd2d_orszag_tang": (C.c_int, [C.POINTER(CcMhd2dParams), C.c_double, C.c_double, C.POINTER(_DP)]),
    "cc_ic_euler2d_random_blob": (C.c_int, [C.POINTER(CcEuler2dParams), C.POINTER(_DP)]),
    "cc_batch_create": (C.c_int, [C.POINTER(CcMhd2dParams), C.c_int, C.POINTER(_H)]),
    "cc_batch_upload": (C.c_int, [_H, C.c_int, C.POINTER(_DP)]),
    "cc_batch_download": (C.c_int, [_H, C.c_int, C.POINTER(_DP)]),
    "cc_batch_compute_dt": (C.c_int, [_H, _DP]),
    "cc_batch_advance": (C.c_int, [_H, C.c_int, _DP]),
    "cc_batch_diagnostics": (C.c_int, [_H, C.c_int, C.POINTER(CcDiag)]),
    "cc_batch_times": (C.c_int, [_H, _DP]),
    "cc_batch_autotune": (C.c_int, [_H, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "cc_batch_set_shape": (C.c_int, [_H, C.c_int]),
    "cc_batch_get_info": (C.c_int, [_H, C.POINTER(CcBatchInfo)]),
    "cc_adjoint_create": (C.c_int, [C.POINTER(CcMhd2dParams), C.c_int, C.c_int, C.POINTER(_H)]),
    "cc_adjoint_upload": (C.c_int, [_H, C.POINTER(_DP)]),
    "cc_adjoint_forward": (C.c_int, [_H, C.c_int, C.c_double, C.c_int, _DP]),
    "cc_adjoint_download": (C.c_int, [_H, C.POINTER(_DP)]),
    "cc_adjoint_get_dts": (C.c_int, [_H, _DP, C.c_int]),
    "cc_adjoint_set_dts": (C.c_int, [_H, _DP, C.c_int]),
    "cc_adjoint_vjp": (C.c_int, [_H, C.POINTER(_DP), C.POINTER(_DP), _DP]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libcc_b200.so (built by core_collapse_b200.build).  Raises if absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m core_collapse_b200.build` (no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib

"""ctypes layer over libwarpsph_b200.so (declared in include/warpsph_b200.h).

Loads the in-tree shared library and exposes each C entry point with argument
types.  There is no fallback: if the library is missing, or a call is made on
tensors that are not CUDA float32, a RuntimeError is raised.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libwarpsph_b200.so"

SPH_OK = 0
SPH_ERR_BAD_ARG = -1
STATUS_LIST_OVERFLOW = 0x1
STATUS_NONFINITE = 0x2
STATUS_NOT_CONVERGED = 0x4
STATUS_TIMEOUT = 0x8
STATUS_LIST_STALE = 0x10

SUPPORT_GATHER = 0
SUPPORT_SCATTER = 1
SUPPORT_SYMMETRIC = 2
SUPPORT_SUPERSYMMETRIC = 3
SUPPORT_KERNELMEANSYMMETRIC = 4


class SphParams(C.Structure):
    """Mirror of the C struct SphParams (include/warpsph_b200.h)."""

    _fields_ = [
        ("domain_min", C.c_double * 3),
        ("domain_max", C.c_double * 3),
        ("verlet_scale", C.c_double),
        ("C_l", C.c_double), ("C_q", C.c_double), ("Cu_l", C.c_double), ("Cu_q", C.c_double), ("K", C.c_double),
        ("eta_crit", C.c_double), ("eta_fold", C.c_double),
        ("gamma", C.c_double),
        ("alpha_min", C.c_double), ("alpha_max", C.c_double), ("beta_xi", C.c_double),
        ("target_neighbors", C.c_double),
        ("cfl", C.c_double), ("min_dt", C.c_double), ("max_dt", C.c_double), ("dt_growth", C.c_double),
        ("c_s", C.c_double),
        ("beta_c", C.c_double), ("beta_d", C.c_double),
        ("reserved_d", C.c_double * 5),
        ("dim", C.c_int32),
        ("kernel", C.c_int32),
        ("periodic", C.c_int32 * 3),
        ("viscosity_term", C.c_int32),
        ("monaghan_switch", C.c_int32), ("correct_xi", C.c_int32), ("scale_beta", C.c_int32),
        ("enable_crk_limiter", C.c_int32), ("enable_vanleer_limiter", C.c_int32),
        ("force_vanleer_off", C.c_int32), ("force_vanleer_on", C.c_int32),
        ("energy_scheme", C.c_int32),
        ("limit_xi", C.c_int32),
        ("kahan", C.c_int32),
        ("list_stride", C.c_int32),
        ("conductivity_term", C.c_int32),
        ("correct_velocity_gradient", C.c_int32),
        ("reserved_i", C.c_int32 * 5),
    ]


class SphJacobiConfig(C.Structure):
    """Mirror of the C struct SphJacobiConfig (include/warpsph_b200.h)."""

    _fields_ = [
        ("rest_density", C.c_double),
        ("tolerance", C.c_double),
        ("relaxation", C.c_double),
        ("min_iterations", C.c_int32),
        ("max_iterations", C.c_int32),
        ("init_mode", C.c_int32),
        ("barrier_timeout_us", C.c_int32),
        ("reserved_i", C.c_int32 * 2),
    ]


class SphWcParams(C.Structure):
    """Mirror of the C struct SphWcParams (include/warpsph_b200.h)."""

    _fields_ = [
        ("rest_density", C.c_double), ("sound_speed", C.c_double), ("polytropic_exponent", C.c_double), ("kappa", C.c_double),
        ("density_delta", C.c_double), ("viscosity_nu", C.c_double), ("inviscid_alpha", C.c_double),
        ("inviscid", C.c_int32), ("density_scheme", C.c_int32), ("pressure_term", C.c_int32), ("eos", C.c_int32),
        ("reserved_i", C.c_int32 * 4),
    ]


_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32

# name -> argtypes (restype is int unless listed in _RESTYPE)
_PROTOS = {
    "sph_version": [],
    "sph_last_error_string": [],
    "sph_launch_count": [],
    "sph_launch_count_conditional": [],
    "sph_kernel_constants": [_I32, _I32, _P, _P],
    "sph_neighbors_workspace_size": [_P, _I64, _I64, _P],
    "sph_neighbors_build": [_P, _I64, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _P,
                            _P, _P, _P, _P],
    "sph_neighbors_refresh": [_P, _I64] + [_P] * 13,
    "sph_neighbors_refresh_volume": [_P, _I64] + [_P] * 14,
    "sph_neighbors_update": [_P, _I64, _P, _P, _P, _P, _P, _I64, _I64] + [_P] * 8 + [_I64] + [_P] * 5,
    "sph_neighbors_rewrite": [_P, _I64] + [_P] * 13,
    "sph_rk_combine_fields": [_P, _I32, _P, _P, _P, _P, _I32, _P, _P, _P, _P],
    "sph_crk_factors_eos": [_P, _I64] + [_P] * 17,
    "sph_neighbors_expand": [_I64, _P, _P, _P, _I64, _P, _P, _P],
    "sph_density_gather": [_P, _I64, _I32, _P, _P, _P, _P, _P, _P, _P, _P],
    "sph_adaptive_h_iter": [_P, _I64, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "sph_minmax": [_I64, _P, _P, _P],
    "sph_owen_iter": [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _I32, C.c_double, _P, _P, _P, _P, _P, _P],
    "sph_crk_volume": [_P, _I64, _P, _P, _P, _P, _P, _P, _P],
    "sph_crk_factors": [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "sph_eos_ideal_gas": [_P, _I64, _P, _P, _P, _P, _P, _P],
    "sph_grad_v": [_P, _I64] + [_P] * 19,
    "sph_switch_cullen": [_P, _I64] + [_P] * 18,
    "sph_switch_balsara": [_P, _I64, _P, _P, _P, _P],
    "sph_switch_hopkins_terms": [_P, _I64] + [_P] * 14,
    "sph_switch_hopkins_update": [_P, _I64] + [_P] * 14,
    "sph_crk_accel_dudt": [_P, _I64] + [_P] * 23,
    "sph_crk_record_floats": [_I32],
    "sph_crk_accel_dudt_packed": [_P, _I64] + [_P] * 24,
    "sph_crk_accel": [_P, _I64] + [_P] * 21,
    "sph_crk_dudt": [_P, _I64] + [_P] * 18,
    "sph_compsph_prep": [_P, _I64] + [_P] * 12,
    "sph_grad_h_omega": [_P, _I64] + [_P] * 9,
    "sph_compsph_accel_dudt": [_P, _I64] + [_P] * 19,
    "sph_compsph_record_floats": [_I32],
    "sph_compsph_accel_dudt_packed": [_P, _I64] + [_P] * 20,
    "sph_compsph_accel": [_P, _I64] + [_P] * 17,
    "sph_compsph_dudt": [_P, _I64] + [_P] * 14,
    "sph_monaghan_rhs": [_P, _I64] + [_P] * 22,
    "sph_compsph_balance": [_P, _I64] + [_P] * 16,
    "sph_compsph_balance_noalloc": [_P, _I64] + [_P] * 14,
    "sph_cfl_dt": [_P, _I64, _P, _P, _P, _P, _P, _P],
    "sph_rk_combine": [_P, _I64, _P, _I32, _P, _P, _P, _I32, _P, _P],
    "sph_finalize_compatible_energy": [_P, _I64, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "sph_conservation_sums": [_P, _I64, _P, _P, _P, _P, _P],
    "sph_dfsph_alpha": [_P, _I64] + [_P] * 9,
    "sph_incompressible_divergence": [_P, _I64, C.c_double] + [_P] * 12,
    "sph_pressure_accel_iisph": [_P, _I64] + [_P] * 10,
    "sph_pressure_shift_iisph": [_P, _I64] + [_P] * 10,
    "sph_dfsph_workspace_size": [_I64, _I32],
    "sph_dfsph_features": [_P, _P, _I32, _I64] + [_P] * 12 + [_I64] + [_P] * 3,
    "sph_mlp_param_count": [],
    "sph_mdbc_density": [_P, _I64] + [_P] * 10 + [C.c_double, C.c_double] + [_P] * 4,
    "sph_mdbc_nopen_shift": [_P, _I64] + [_P] * 11,
    "sph_deltasph_rhs": [_P, _P, _I64] + [_P] * 13,
    "sph_wc_eos": [_P, _I64, _P, _P, _P],
    "sph_ensemble_neighbors_workspace_size": [_I64, _I64],
    "sph_ensemble_neighbors_build": [_P, _I64, _I32, _P, _P, _P, _I64, _P, _P, _P, _I64, _P, _P, _P, _I64, _P, _P, _P],
    "sph_ensemble_step_workspace_size": [_I64, _I32],
    "sph_ensemble_step": [_P, _P, _I64] + [_P] * 12 + [_I64, _I32, _I32, _P, _P, _P],
    "sph_mlp_forward": [_P, _I64, _P, _P, _P, _P],
    "sph_mlp_forward_tc": [_P, _I64, _P, _P, _P, _P, _P],
    "sph_wc_visc_continuity": [_P, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "sph_surface_color_field": [_P, _I64] + [_P] * 9,
    "sph_surface_detect_color_field": [_P, _I64] + [_P] * 8 + [C.c_float, C.c_float] + [_P] * 4,
    "sph_surface_dilate": [_P, _I64] + [_P] * 8,
    "sph_surface_barecasco": [_P, _I64] + [_P] * 5 + [C.c_float] + [_P] * 4,
    "sph_surface_maronne": [_P, _I64] + [_P] * 9,
    "sph_surface_detect_color_gradient": [_P, _I64] + [_P] * 8 + [C.c_float] + [_P] * 3,
    "sph_surface_renormalization": [_P, _I64] + [_P] * 10,
    "sph_surface_renormalized_normals": [_P, _I64, _I32] + [_P] * 12,
    "sph_delta_shift": [_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_float, _P, _P, _P],
    "sph_mlp_grad": [_P, _I64, _P, _P, _P, _P, _P],
    "sph_mlp_grad_tc": [_P, _I64, _P, _P, _P, _P, _P, _P],
    "sph_mlp_adam": [_P, _P, _P, _P, _I64, C.c_float, C.c_float, C.c_float, C.c_float, _I64, _P],
    "sph_dfsph_div_solve": [_P, _P, _I64] + [_P] * 12 + [_I64] + [_P] * 6,
    "sph_dfsph_density_solve": [_P, _P, _I64] + [_P] * 12 + [_I64] + [_P] * 6,
}
_RESTYPE = {"sph_version": C.c_char_p, "sph_last_error_string": C.c_char_p, "sph_launch_count": C.c_int64, "sph_launch_count_conditional": C.c_int64,
            "sph_dfsph_workspace_size": C.c_int64,
            "sph_mlp_param_count": C.c_int64, "sph_ensemble_neighbors_workspace_size": C.c_int64,
            "sph_ensemble_step_workspace_size": C.c_int64}

_lib = None


def lib() -> C.CDLL:
    """Loads libwarpsph_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("WARPSPH_B200_LIB", LIB_PATH))
    if not path.exists():
        raise RuntimeError(
            f"libwarpsph_b200.so not found at {path}; build it with `python -m warpsph_b200.build` "
            "(there is no CPU fallback)")
    L = C.CDLL(str(path))
    for name, args in _PROTOS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, C.c_int)
        setattr(L, name, _Strict(fn, name, len(args)))
    _lib = L
    return L


class _Strict:
    """A C entry point that refuses a call with the wrong number of arguments (ctypes
    passes surplus arguments on silently, which would shift every argument after a
    forgotten or extra one)."""

    __slots__ = ("fn", "name", "nargs")

    def __init__(self, fn, name: str, nargs: int):
        self.fn, self.name, self.nargs = fn, name, nargs

    def __call__(self, *args):
        if len(args) != self.nargs:
            raise TypeError(f"{self.name} takes {self.nargs} arguments ({len(args)} given)")
        return self.fn(*args)


def declared_functions() -> list[str]:
    return list(_PROTOS)


def last_error() -> str:
    return lib().sph_last_error_string().decode()


def check(rc: int, what: str) -> None:
    if rc != SPH_OK:
        raise RuntimeError(f"{what} failed ({rc}): {last_error()}")


def ptr(t) -> int | None:
    """Device pointer of a contiguous CUDA tensor (None for None); anything else raises."""
    if t is None:
        return None
    if isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous():
        return t.data_ptr()
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"expected a torch.Tensor, got {type(t)}")
    if not t.is_cuda:
        raise RuntimeError("warpsph_b200 operates on CUDA tensors only (no CPU fallback)")
    raise RuntimeError("warpsph_b200 requires contiguous tensors")


def fptr(t) -> int | None:
    if t is not None and t.dtype != torch.float32:
        raise RuntimeError(f"expected float32 tensor, got {t.dtype}")
    return ptr(t)


def iptr(t) -> int | None:
    if t is not None and t.dtype != torch.int32:
        raise RuntimeError(f"expected int32 tensor, got {t.dtype}")
    return ptr(t)


try:   # the raw handle of the current stream without building a Stream object per call
    from torch._C import _cuda_getCurrentRawStream as _raw_stream
except ImportError:   # pragma: no cover
    _raw_stream = None


def stream_ptr(device=None) -> int:
    """cudaStream_t of the current stream of `device` (a torch.device, an index or None for
    the current device), as an int."""
    if _raw_stream is not None:
        if isinstance(device, str):
            device = torch.device(device)
        idx = device.index if isinstance(device, torch.device) else device
        if idx is None:
            idx = torch.cuda.current_device()
        return _raw_stream(idx)
    return torch.cuda.current_stream(device).cuda_stream


def ptr_array(ptrs) -> C.Array:
    return (C.c_void_p * len(ptrs))(*ptrs)


def double_array(vals) -> C.Array:
    return (C.c_double * len(vals))(*[float(v) for v in vals])

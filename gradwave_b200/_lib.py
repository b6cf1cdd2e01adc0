"""ctypes binding of libgwb.so (the C ABI declared in include/gwb.h).

The library is loaded on first use. There is no fallback: if libgwb.so is
missing or CUDA is unavailable, every compute entry raises.
"""

from __future__ import annotations

import ctypes
import struct
import threading
from pathlib import Path

import torch

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgwb.so"

GWB_OK = 0
GWB_ERR_ARG = 1
GWB_ERR_CUDA = 2
GWB_ERR_NONFINITE = 3
GWB_ERR_TIMEOUT = 4
GWB_ERR_NOT_CONVERGED = 5
GWB_ERR_ALLOC = 6
GWB_ERR_BREAKDOWN = 7

GWB_C64 = 0
GWB_C128 = 1
GWB_FP32 = 0
GWB_FP64 = 1

_STATUS_NAMES = {1: "bad argument", 2: "CUDA error", 3: "non-finite value", 4: "device wait timeout",
                 5: "not converged", 6: "allocation failed", 7: "Cholesky breakdown"}


class GwbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"libgwb status {status} ({_STATUS_NAMES.get(status, '?')}): {msg}")
        self.status = status


class Geometry(ctypes.Structure):
    _fields_ = [("nk", ctypes.c_int32), ("npw_max", ctypes.c_int32), ("n", ctypes.c_int32 * 3),
                ("nproj", ctypes.c_int32), ("npw", ctypes.POINTER(ctypes.c_int64)),
                ("flat_idx", ctypes.POINTER(ctypes.c_int64))]


class DavidsonParams(ctypes.Structure):
    _fields_ = [("nk", ctypes.c_int32), ("nb", ctypes.c_int32), ("npw", ctypes.c_int32),
                ("max_dim", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("precond", ctypes.c_int32), ("flags", ctypes.c_int32), ("tol", ctypes.c_double),
                ("t_max", ctypes.c_double)]


class DavidsonStats(ctypes.Structure):
    _fields_ = [("n_iter", ctypes.c_int32), ("hit_max_iter", ctypes.c_int32), ("n_restart", ctypes.c_int32),
                ("n_cert", ctypes.c_int32), ("n_repair", ctypes.c_int32), ("n_rollback", ctypes.c_int32),
                ("n_apply_low", ctypes.c_int64), ("n_apply_full", ctypes.c_int64),
                ("max_residual", ctypes.c_double), ("apply_ms", ctypes.c_double),
                ("n_apply_calls", ctypes.c_int64), ("n_tpa_fallback", ctypes.c_int64)]


_lock = threading.Lock()
_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_SZ = ctypes.c_size_t

# name -> argtypes (every function returns int status unless listed in _RESTYPES)
_SIGNATURES = {
    "gwb_last_error": [],
    "gwb_version": [],
    "gwb_launch_count": [],
    "gwb_ham_create": [ctypes.POINTER(Geometry), ctypes.c_int, ctypes.POINTER(_P)],
    "gwb_ham_destroy": [_P],
    "gwb_ham_set_kinetic": [_P, _P, _P],
    "gwb_ham_set_potential": [_P, _P, _P],
    "gwb_ham_set_projectors": [_P, _P, _P, _P],
    "gwb_ham_apply": [_P, _P, _P, _I, _I, _I, _P],
    "gwb_ham_apply_strided": [_P, _P, _I64, _P, _I64, _I, _I, _I, _P],
    "gwb_ham_set_overlap": [_P, _P, _P],
    "gwb_ham_set_tuning": [_P, _I64, _I],
    "gwb_ham_apply_hs": [_P, _P, _I64, _P, _I64, _P, _I64, _I, _I, _I, _P],
    "gwb_ham_scratch_bytes": [_P],
    "gwb_ham_tc_status": [_P, _P],
    "gwb_ham_density": [_P, _P, _I64, _I, _I, _P, _I64, _D, _P, _P],
    "gwb_gamma_work_bytes": [_I, _I],
    "gwb_gamma_apply": [_P, _I, _I, _I, _P, _I64, _P, _I64, _P, _P, _P, _P, _I, _P, _SZ, _P],
    "gwb_zgemm": [ctypes.c_int, ctypes.c_int, _I64, _I64, _I64, _D, _D, _P, _I64, _I64, _P, _I64, _I64,
                  _D, _D, _P, _I64, _I64, _I64, _P],
    "gwb_zgemm_nh": [_I64, _I64, _I64, _D, _D, _P, _I64, _I64, _P, _I64, _I64, _D, _D, _P, _I64, _I64, _I64, _P,
                     ctypes.c_size_t, _P],
    "gwb_tc_planes": [_I64, _I64, _I64, _P, _I64, _I64, ctypes.c_int, ctypes.c_int, _P, _I64, _I64, _I64, _P],
    "gwb_zgemm_tc_work_bytes": [ctypes.c_int, _I64, _I64, _I64, _I64],
    "gwb_tc_set_wait_limit": [_I64],
    "gwb_oz_split_rows": [_I, _I64, _I64, _P, _I64, _P, _P, _I64, _I64, _I64, _P, _P],
    "gwb_oz_split_cols": [_I, _I64, _I64, _P, _I64, _P, _I64, _I64, _I64, _P, _P],
    "gwb_oz_work_bytes": [_I64, _I64, _I64],
    "gwb_oz_gemm": [_I, _I64, _I64, _I64, _P, _I64, _I64, _I64, _P, _P, _I64, _I64, _I64, _P, _D, _D, _P, _I64, _P,
                    _SZ, _P, _P],
    "gwb_tc_test_withhold": [_I],
    "gwb_ham_set_fft_threads": [_P, _I, _I],
    "gwb_sytrd_work_bytes": [_I],
    "gwb_sytrd_set_blocks": [_I],
    "gwb_sytrd_set_trace": [_P],
    "gwb_sytrd_set_cluster": [_I],
    "gwb_sytrd_cluster_rows": [_I],
    "gwb_sytrd_set_grid": [_I],
    "gwb_precond_set_kernel": [_I],
    "gwb_precond_learned_gamma_work_bytes": [_I, _I],
    "gwb_precond_learned_gamma": [_P, _I, _I, _I, _I, _P, _I64, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _SZ, _P],
    "gwb_sytrd": [_I, _P, _I64, _P, _P, _P, _P, _SZ, _P, _P],
    "gwb_sy_lowest_work_bytes": [_I, _I],
    "gwb_sy_lowest": [_I, _I, _P, _I64, _P, _P, _I64, _P, _SZ, _P, _P],
    "gwb_crt_bits": [_I],
    "gwb_crt_constants": [_I, _P, _P, _P, _P, _P],
    "gwb_crt_split_rows": [_I, _I64, _I64, _P, _I64, _P, _P, _I64, _I64, _I64, _P, _P],
    "gwb_crt_split_cols": [_I, _I64, _I64, _P, _I64, _P, _I64, _I64, _I64, _P, _P, _P],
    "gwb_crt_work_bytes": [_I, _I64, _I64, _I64],
    "gwb_crt_gemm": [_I, _I64, _I64, _I64, _P, _I64, _I64, _I64, _P, _P, _I64, _I64, _I64, _P, _D, _D, _P, _I64,
                     _P, _SZ, _P, _P],
    "gwb_zgemm_tc": [ctypes.c_int, _I64, _I64, _I64, _D, _D, _P, _I64, _I64, _P, _I64, _I64, _D, _D, _P, _I64, _I64,
                     _I64, _P, ctypes.c_size_t, _P, _P],
    "gwb_residual": [_I, _I, _I, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _P, _P],
    "gwb_conv_stats": [_I, _I, _P, _D, _P, _P],
    "gwb_select_worst": [_I, _I, _P, _I, _P, _P],
    "gwb_precond_teter": [_I, _I, _I, _I, _P, _I64, _P, _I64, _P, _P, _P, _I64, _P],
    "gwb_subspace_insert": [_I, _I, _I, _P, _P, _I, _I64, _P],
    "gwb_chol_inv": [_I, _I, _P, _I, _I64, _P, _I64, _P, _P, _P],
    "gwb_row_repair": [_I, _I, _I, _P, _I64, _P, _D, _P, _P],
    "gwb_heev_lowest": [_I, _I, _I, _P, _I, _I64, _P, _P, _P, _P, _P],
    "gwb_heev_max_dim": [],
    "gwb_heev_scratch_doubles": [_I],
    "gwb_heev_ql_count": [_P],
    "gwb_heev_lowest_noalloc": [_I, _I, _I, _P, _I, _I64, _P, _P, _P, _P],
    "gwb_mlp_param_count": [],
    "gwb_mlp_forward": [_P, _I, _P, _P, _P],
    "gwb_mlp_loss_grad": [_P, _I, _P, _P, _P, _P, _P, _P],
    "gwb_mlp_backward": [_P, _I, _P, _P, _P, _P],
    "gwb_mlp_adam": [_P, _P, _P, _P, _I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _P],
    "gwb_precond_features": [_I, _I, _I, _I, _P, _I64, _P, _I64, _P, _P, _P, _P, _P],
    "gwb_precond_learned": [_P, _I, _I, _I, _I, _P, _I64, _P, _I64, _P, _P, _P, _P, _P, _I64, _P, _SZ, _P],
    "gwb_precond_learned_work_bytes": [_I, _I, _I],
    "gwb_stall_update": [_P, _P, _P, _P, _I, _D, _I, _P],
    "gwb_davidson_workspace_bytes": [ctypes.POINTER(DavidsonParams), ctypes.POINTER(ctypes.c_size_t)],
    "gwb_davidson_solve": [_P, ctypes.POINTER(DavidsonParams), _P, _P, _P, _P, _P, ctypes.c_size_t, _P, _P, _P,
                           ctypes.POINTER(DavidsonStats), _P],
}
_RESTYPES = {"gwb_last_error": ctypes.c_char_p, "gwb_version": ctypes.c_char_p,
             "gwb_launch_count": ctypes.c_ulonglong,
             "gwb_ham_scratch_bytes": ctypes.c_size_t, "gwb_heev_scratch_doubles": ctypes.c_int64,
             "gwb_precond_learned_work_bytes": ctypes.c_int64, "gwb_precond_learned_gamma_work_bytes": ctypes.c_int64, "gwb_zgemm_tc_work_bytes": ctypes.c_int64,
             "gwb_gamma_work_bytes": ctypes.c_size_t, "gwb_oz_work_bytes": ctypes.c_int64,
             "gwb_crt_bits": ctypes.c_int32, "gwb_crt_work_bytes": ctypes.c_int64,
             "gwb_sytrd_work_bytes": ctypes.c_size_t, "gwb_sy_lowest_work_bytes": ctypes.c_size_t}


def declared_symbols() -> list[str]:
    """Every entry point the binding expects the library to export."""
    return sorted(_SIGNATURES)


def load() -> ctypes.CDLL:
    """The loaded library (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m gradwave_b200.build` "
                    "(there is no CPU fallback)")
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, args in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, ctypes.c_int)
            _lib = lib
    return _lib


def launch_count() -> int:
    """Kernels launched by libgwb.so in this process (cuBLAS/torch not included)."""
    return int(load().gwb_launch_count())


def heev_diagnostics() -> dict:
    """Subspace-eigensolver diagnostics on the current device: matrices sent to
    the QL fallback by reason, and the largest residual / |T| measured on the
    bisection path."""
    out = (ctypes.c_ulonglong * 5)()
    check(load().gwb_heev_ql_count(out))
    maxres = struct.unpack("<d", struct.pack("<Q", out[4]))[0]
    return {"ql_pool": int(out[0]), "ql_nonfinite": int(out[1]), "ql_cholqr": int(out[2]),
            "ql_residual": int(out[3]), "max_residual_rel": maxres}


def heev_ql_count() -> int:
    """Matrices the subspace eigensolver solved on its QL fallback (current device)."""
    d = heev_diagnostics()
    return d["ql_pool"] + d["ql_nonfinite"] + d["ql_cholqr"] + d["ql_residual"]


def check(status: int) -> None:
    if status != GWB_OK:
        raise GwbError(status, load().gwb_last_error().decode())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


def require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(f"{what} must be a CUDA tensor (the band-solve path has no CPU fallback)")


def stream_ptr(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def io_dtype(t: torch.Tensor) -> int:
    if t.dtype == torch.complex128:
        return GWB_C128
    if t.dtype == torch.complex64:
        return GWB_C64
    raise TypeError(f"expected complex64/complex128, got {t.dtype}")

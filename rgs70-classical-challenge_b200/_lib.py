"""ctypes binding of ``librgs_b200.so`` (declarations in ``include/rgs_b200.h``).

The library is built in-tree by ``build.py``.  There is no fallback: if the
library is missing or fails to load, every entry point raises.
"""
import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "librgs_b200.so"

RGS_OK = 0
RGS_ERR_ARG = 1
RGS_ERR_OOM = 2
RGS_ERR_CUDA = 3
RGS_ERR_NONFINITE = 4
RGS_ERR_ZERO_NORM = 5
RGS_ERR_TIMEOUT = 6
RGS_ERR_UNSUPPORTED = 7
RGS_ERR_SINGULAR = 8

PREC_C64 = 0
PREC_C64_F32 = 1
PREC_C128 = 2

_EXC = {
    RGS_ERR_ARG: ValueError,
    RGS_ERR_OOM: MemoryError,
    RGS_ERR_CUDA: RuntimeError,
    RGS_ERR_NONFINITE: ArithmeticError,
    RGS_ERR_ZERO_NORM: ArithmeticError,
    RGS_ERR_TIMEOUT: TimeoutError,
    RGS_ERR_UNSUPPORTED: NotImplementedError,
    RGS_ERR_SINGULAR: ValueError,
}

c_int32_p = ctypes.POINTER(ctypes.c_int32)


class PairInfo(ctypes.Structure):
    """``rgs_pair_info`` of include/rgs_b200.h."""
    _fields_ = [("j", ctypes.c_int32), ("code_a", ctypes.c_int32), ("code_b", ctypes.c_int32),
                ("a", ctypes.c_int32), ("m", ctypes.c_int32), ("o", ctypes.c_int32), ("dw", ctypes.c_int32),
                ("piv", ctypes.c_int32 * 3), ("pw_b", ctypes.c_uint32),
                ("mask_a", ctypes.c_uint64), ("beta_a", ctypes.c_uint64), ("comb_a", ctypes.c_uint64 * 4),
                ("la_w", ctypes.c_uint64 * 4), ("beta_b", ctypes.c_uint64), ("mb0", ctypes.c_uint64 * 2),
                ("t_b", ctypes.c_uint64), ("la_cols", ctypes.c_uint64 * 64), ("mb_cols", ctypes.c_uint64 * 64)]
c_uint64_p = ctypes.POINTER(ctypes.c_uint64)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p
c_size_t_p = ctypes.POINTER(ctypes.c_size_t)

# name -> (restype, argtypes).  Kept in the order of include/rgs_b200.h.
SIGNATURES = {
    "rgs_version": (ctypes.c_char_p, []),
    "rgs_last_error": (ctypes.c_char_p, []),
    "rgs_device_count": (ctypes.c_int, []),
    "rgs_plan_compile": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_uint8_p,
                                        ctypes.POINTER(c_void_p)]),
    "rgs_plan_destroy": (None, [c_void_p]),
    "rgs_plan_info": (ctypes.c_int, [c_void_p, c_int32_p, c_int32_p, c_int32_p]),
    "rgs_plan_ranks": (ctypes.c_int, [c_void_p, c_int32_p]),
    "rgs_plan_future_masks": (ctypes.c_int, [c_void_p, c_uint64_p]),
    "rgs_plan_step": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_int32_p, c_int32_p, c_int32_p, c_int32_p,
                                     c_uint64_p, c_uint64_p, c_int32_p, c_uint64_p]),
    "rgs_plan_step_tables": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_uint64_p, c_int32_p]),
    "rgs_rank_profile": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_uint8_p,
                                        c_int32_p]),
    "rgs_plan_set_fusion": (ctypes.c_int, [c_void_p, ctypes.c_int32]),
    "rgs_plan_pairs": (ctypes.c_int, [c_void_p, c_int32_p, c_int32_p]),
    "rgs_plan_pair_info": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_void_p]),
    "rgs_scan_workspace_bytes": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_size_t_p]),
    "rgs_scan_launch_count": (ctypes.c_int, [c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64)]),
    "rgs_order_search": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, ctypes.c_int32,
                                        ctypes.c_int64, ctypes.c_uint64, ctypes.c_int32, c_int32_p, c_int32_p,
                                        c_double_p]),
    "rgs_scan_max_batch_tile": (ctypes.c_int, [ctypes.c_int32, c_int32_p]),
    "rgs_scan_amplitudes": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int64, ctypes.c_int32,
                                           c_void_p, c_void_p, c_void_p, ctypes.c_size_t, ctypes.c_int32,
                                           c_void_p]),
    "rgs_scan_contract": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int64, ctypes.c_int32, c_void_p,
                                         c_void_p, c_void_p, ctypes.c_size_t, ctypes.c_int32, c_void_p]),
    "rgs_scan_amplitudes_noalloc": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int64, ctypes.c_int32,
                                                   c_void_p, c_void_p, c_void_p]),
    "rgs_chain_workspace_bytes": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_size_t_p]),
    "rgs_chain_launch_count": (ctypes.c_int, [c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "rgs_chain_sample": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int64, ctypes.c_uint64, c_void_p, ctypes.c_int32,
                                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_size_t,
                                        ctypes.c_int32, ctypes.c_int32, c_void_p]),
    "rgs_chain_marginals": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_int64, ctypes.c_int32, c_void_p,
                                           c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_size_t, ctypes.c_int32,
                                           ctypes.c_int32, c_void_p]),
    "rgs_batch_max_rank": (ctypes.c_int, [ctypes.c_int32, c_int32_p]),
    "rgs_batch_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(c_void_p)]),
    "rgs_batch_destroy": (None, [c_void_p]),
    "rgs_batch_add": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int64, c_void_p, c_void_p,
                                     ctypes.c_int64, ctypes.c_uint64, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_int32_p]),
    "rgs_batch_info": (ctypes.c_int, [c_void_p, c_int32_p, ctypes.POINTER(ctypes.c_int64)]),
    "rgs_batch_run": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_void_p]),
    "rgs_batch_tune": (ctypes.c_int, [c_void_p, c_void_p, c_int32_p, ctypes.POINTER(ctypes.c_float)]),
    "rgs_gemm_bf16": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_void_p, ctypes.c_int32,
                                     ctypes.c_int32, c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                     c_void_p, ctypes.c_int32, c_void_p, c_void_p, c_void_p, c_void_p,
                                     ctypes.c_int32, c_void_p]),
    "rgs_tensor_core_status": (ctypes.c_int, [c_int32_p]),
    "rgs_gemm_set_tma": (ctypes.c_int, [ctypes.c_int32]),
    "rgs_fourier_set_register_schedule": (ctypes.c_int, [ctypes.c_int32]),
    "rgs_fourier_set_tma": (ctypes.c_int, [ctypes.c_int32]),
    "rgs_mlp_fwd": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32] + [c_void_p] * 11),
    "rgs_mlp_bwd": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32] + [c_void_p] * 20
                    + [ctypes.c_int32, c_void_p]),
    "rgs_mlp_adam": (ctypes.c_int, [c_void_p] * 6 + [ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                                      ctypes.c_float, ctypes.c_int32, c_void_p]),
    "rgs_mlp_sample": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32] + [c_void_p] * 6
                       + [ctypes.c_uint64, ctypes.c_uint64] + [c_void_p] * 6),
    "rgs_mlp_logq": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32] + [c_void_p] * 12),
    "rgs_fourier_create": (ctypes.c_int, [ctypes.c_int32, c_uint8_p, c_double_p, ctypes.c_int32, c_int32_p,
                                          c_int32_p, ctypes.c_int32, ctypes.POINTER(c_void_p)]),
    "rgs_fourier_destroy": (None, [c_void_p]),
    "rgs_fourier_compute_shard": (ctypes.c_int, [c_void_p, ctypes.c_uint64, ctypes.c_int32, c_void_p, c_void_p,
                                                 ctypes.c_size_t, c_void_p]),
    "rgs_fourier_shard_mass": (ctypes.c_int, [c_void_p, c_void_p, c_double_p, c_void_p]),
    "rgs_fourier_shard_draw": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_double, ctypes.c_double,
                                              ctypes.POINTER(ctypes.c_uint64), c_void_p]),
    "rgs_fourier_info": (ctypes.c_int, [c_void_p, c_int32_p, c_int32_p, c_int32_p, ctypes.POINTER(ctypes.c_int64),
                                        c_int32_p]),
    "rgs_fourier_tables": (ctypes.c_int, [c_void_p, c_uint64_p, c_uint64_p, c_uint64_p, c_uint64_p, c_int32_p]),
    "rgs_fourier_workspace_bytes": (ctypes.c_int, [c_void_p, c_size_t_p]),
    "rgs_fourier_tune": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_size_t, c_void_p, c_int32_p,
                                        ctypes.POINTER(ctypes.c_float)]),
    "rgs_fourier_compute": (ctypes.c_int, [c_void_p, ctypes.c_uint64, c_void_p, c_void_p, ctypes.c_size_t, c_void_p,
                                           ctypes.POINTER(ctypes.c_float)]),
    "rgs_fourier_compute_permute": (ctypes.c_int, [c_void_p, ctypes.c_uint64, c_void_p, c_void_p, c_void_p,
                                                   ctypes.c_size_t, c_void_p]),
    "rgs_fourier_masses": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_double_p, c_double_p, c_void_p]),
    "rgs_fourier_draw": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, c_uint64_p, c_double_p, c_double_p, c_void_p]),
    "rgs_fourier_index_map": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "rgs_fourier_quadphase": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "rgs_fwht": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_void_p]),
    "rgs_fwht_precision": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          c_void_p]),
    "rgs_product": (ctypes.c_int, [c_void_p, ctypes.c_int32, c_void_p, ctypes.c_int32, ctypes.c_int32, c_void_p]),
    "rgs_block_mass": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.c_int32, c_void_p, c_void_p]),
}

_lib = None


class LibraryMissing(RuntimeError):
    """The CUDA library is not built or cannot be loaded; there is no CPU fallback."""


def lib():
    """Load the library once; raise LibraryMissing if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("RGS_B200_LIB", str(LIB_PATH)))
    if not path.exists():
        raise LibraryMissing(f"{path} not found: build it with __graft_entry__.build() "
                             "(the engine has no CPU fallback)")
    try:
        handle = ctypes.CDLL(str(path))
    except OSError as exc:
        raise LibraryMissing(f"cannot load {path}: {exc}") from exc
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return _lib


def check(status):
    """Raise the Python exception mapped from a status code."""
    if status == RGS_OK:
        return
    msg = lib().rgs_last_error().decode(errors="replace")
    raise _EXC.get(status, RuntimeError)(f"rgs_b200 error {status}: {msg}")


def ptr(array, ctype):
    """ctypes pointer to a contiguous numpy array."""
    return array.ctypes.data_as(ctypes.POINTER(ctype))

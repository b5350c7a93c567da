"""ctypes binding of libvlasov_b200.so (the C ABI in include/vlasov_b200.h).

The library is the only compute path: if it is missing or fails to load,
every entry point raises. There is no CPU or eager-torch fallback.
"""
from __future__ import annotations

import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvlasov_b200.so")

VP_F32, VP_F64, VP_BF16 = 0, 1, 2
DIAG_COUNT = 8
STATUS_WAIT_TIMEOUT = 1  # VP_STATUS_* bits of the steps' device status word
STATUS_NONFINITE = 2
DIAG_NAMES = ("field_energy", "mass", "l2", "kinetic", "kinetic_pre", "max_shift")

_DTYPE_CODE = {torch.float32: VP_F32, torch.float64: VP_F64, torch.bfloat16: VP_BF16}


class VlasovError(RuntimeError):
    """A library call returned a non-zero status."""


def dtype_code(dt: torch.dtype) -> int:
    try:
        return _DTYPE_CODE[dt]
    except KeyError:
        raise TypeError(f"unsupported storage dtype {dt}; use float32, float64 or bfloat16") from None


def compute_dtype(dt: torch.dtype) -> torch.dtype:
    """Arithmetic type of a storage type: float64 for float64, else float32."""
    return torch.float64 if dt == torch.float64 else torch.float32


P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int32
D = ctypes.c_double
SZ = ctypes.c_size_t


class Step2dDesc(ctypes.Structure):
    _fields_ = [
        ("dtype", I32), ("nx", I64), ("ny", I64), ("nvx", I64), ("nvy", I64),
        ("dt", D), ("dx", D), ("dy", D), ("dvx", D), ("dvy", D),
        ("physics_mode", I32), ("window", I32), ("diagnostics", I32),
        ("shift_spread_x", I32), ("shift_spread_y", I32),
        ("f_in", P), ("f_out", P), ("f_tmp", P),
        ("shift_x", P), ("W_x", P), ("shift_y", P), ("W_y", P),
        ("kx", P), ("ky", P), ("inv_ksq", P), ("vx", P), ("vy", P),
        ("drho", P), ("phi", P), ("ex", P), ("ey", P), ("diag", P),
        ("workspace", P), ("workspace_bytes", SZ), ("events", P),
        ("eq_vx", P), ("eq_vy", P), ("eq_moment", D),
        ("sweeps_only", I32),
        ("status", P), ("test_stall", I32),
    ]


class Step1dDesc(ctypes.Structure):
    _fields_ = [
        ("dtype", I32), ("nx", I64), ("nv", I64),
        ("dt", D), ("dx", D), ("dv", D),
        ("physics_mode", I32), ("window", I32), ("diagnostics", I32), ("shift_spread", I32),
        ("f_in", P), ("f_out", P), ("f_tmp", P),
        ("shift", P), ("W", P), ("inv_kx", P), ("inv_kx_sq", P), ("v", P),
        ("rho", P), ("phi", P), ("e", P), ("diag", P),
        ("workspace", P), ("workspace_bytes", SZ), ("events", P),
        ("eq_v", P), ("eq_moment", D),
        ("status", P),
    ]


class BatchRun(ctypes.Structure):
    _fields_ = [
        ("nx", I32), ("ny", I32), ("nvx", I32), ("nvy", I32),
        ("dt", D), ("dx", D), ("dy", D), ("dvx", D), ("dvy", D),
        ("window", I32), ("shift_spread_x", I32), ("shift_spread_y", I32), ("segments_x", I32),
        ("segments_y", I32), ("test_stall", I32),
        ("f", P), ("s1", P), ("s2", P),
        ("shift_x", P), ("W_x", P), ("shift_y", P), ("W_y", P),
        ("kx", P), ("ky", P), ("inv_ksq", P),
        ("drho", P), ("phi", P), ("diag", P), ("diag_slot_stride", I64),
        ("workspace", P), ("workspace_bytes", SZ), ("status", P),
    ]


BATCH_KINDS = 3


class BatchTiles(ctypes.Structure):
    _fields_ = [("block", I32 * BATCH_KINDS), ("ctas_per_sm", I32 * BATCH_KINDS), ("segments", I32 * BATCH_KINDS),
                ("sweeps_only", I32)]


# name -> (restype, argtypes)
SIGNATURES = {
    "vp_version": (ctypes.c_char_p, []),
    "vp_last_error": (ctypes.c_char_p, []),
    "vp_launch_count": (ctypes.c_uint64, []),
    "vp_drift": (ctypes.c_int, [P, P, ctypes.c_int, I64, I64, I64, I64, I64, P, I32, P, P]),
    "vp_drift_rho": (ctypes.c_int, [P, P, ctypes.c_int, I64, I64, I64, I64, I64, P, I32, P, D, P, P, SZ, P]),
    "vp_drift_rho_workspace_bytes": (SZ, [I64, I64, I64]),
    "vp_drift_pair": (ctypes.c_int, [P, P, ctypes.c_int, I64, I64, I64, I64, I32, I64, I64, P, P, P, P, D, P, P, SZ,
                                     P]),
    "vp_drift_pair_workspace_bytes": (SZ, [I64, I64, I64, I64]),
    "vp_kick": (ctypes.c_int, [P, P, ctypes.c_int, I64, I64, I64, P, ctypes.c_int, I64, D, D, I32, P]),
    "vp_kick2d": (ctypes.c_int, [P, P, ctypes.c_int, I64, I64, I64, P, P, D, D, D, I32, P, P, P, P]),
    "vp_advect_gather": (ctypes.c_int, [P, P, ctypes.c_int, I64, I64, I64, P, I64, I64, I64, D, D, ctypes.c_int, P]),
    "vp_rho": (ctypes.c_int, [P, ctypes.c_int, I64, I64, D, D, P, ctypes.c_int, P]),
    "vp_lagrange_interp": (ctypes.c_int, [P, P, P, ctypes.c_int, I64, P]),
    "vp_init_product": (ctypes.c_int, [P, P, P, ctypes.c_int, I64, I64, P]),
    "vp_lagrange_weights": (ctypes.c_int, [P, P, ctypes.c_int, I64, P]),
    "vp_poisson2d": (ctypes.c_int, [P, I64, I64, P, P, P, D, D, P, P, P, P, P, P, SZ, P]),
    "vp_poisson2d_workspace_bytes": (SZ, [I64, I64]),
    "vp_poisson2d_static": (ctypes.c_int, [P, I64, I64, P, P, P, D, D, P, P, P, P, P, P]),
    "vp_poisson1d": (ctypes.c_int, [P, I64, P, P, D, P, P, P, P, P, SZ, P]),
    "vp_poisson1d_workspace_bytes": (SZ, [I64]),
    "vp_step2d": (ctypes.c_int, [ctypes.POINTER(Step2dDesc), P]),
    "vp_step2d_passes": (ctypes.c_int, [ctypes.POINTER(Step2dDesc), P]),
    "vp_batch2d_table_bytes": (SZ, [I32]),
    "vp_batch2d_plan": (ctypes.c_int, [I32, I32, I32, ctypes.POINTER(BatchRun), I32, ctypes.POINTER(BatchTiles), P,
                                       SZ]),
    "vp_batch2d_step": (ctypes.c_int, [P, P, I32, P, P]),
    "vp_mlp_drift": (ctypes.c_int, [P, P, I64, I64, I64, I64, I64, P, P, P, P, P, P]),
    "vp_mlp_train": (ctypes.c_int, [P, P, I64, I64, I64, I64, I64, P, P, P, P, D, P, P, P, P]),
    "vp_mlp_kick": (ctypes.c_int, [P, P, I64, I64, I64, P, I64, D, D, P, P, P]),
    "vp_mlp_train_kick": (ctypes.c_int, [P, P, I64, I64, I64, P, I64, D, D, P, D, P, P, P, P]),
    "vp_step2d_workspace_bytes": (SZ, [I64, I64, I64, I64]),
    "vp_step1d": (ctypes.c_int, [ctypes.POINTER(Step1dDesc), P]),
    "vp_step1d_workspace_bytes": (SZ, [I64, I64]),
}

_LIB = None


def load() -> ctypes.CDLL:
    """Load (once) and return the CUDA library; raises if it is not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise VlasovError(
                f"{LIB_PATH} is not built; run __graft_entry__.build() or "
                "python -c \"import importlib; importlib.import_module('jax-pytorch-vlasov_b200.build').build()\"")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def call(name: str, *args) -> None:
    """Call an int-returning entry point; raise VlasovError on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.vp_last_error().decode(errors="replace")
        raise VlasovError(f"{name} failed with status {rc}: {msg}")


def query(name: str, *args) -> int:
    return int(getattr(load(), name)(*args))


def ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_of(t: torch.Tensor):
    """The current torch stream of t's device, as the library's void* stream."""
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def require_cuda(*tensors: torch.Tensor) -> None:
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise ValueError("tensors must live on a CUDA device (the library has no CPU path)")
        if dev is None:
            dev = t.device
        elif t.device != dev:
            raise ValueError(f"tensors on different devices: {dev} and {t.device}")
        if not t.is_contiguous():
            raise ValueError("tensors must be contiguous (row-major)")

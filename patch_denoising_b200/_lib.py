"""ctypes binding of ``libpd_b200.so`` (the C ABI in ``include/patch_denoise_b200.h``).

The library is loaded lazily on first use. If it has not been built the load
fails loudly: there is no CPU fallback for the denoising path.
"""

from __future__ import annotations

import ctypes
import pathlib
import threading

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "libpd_b200.so"

PD_OK = 0
PD_ERR_INVALID = 1
PD_ERR_UNSUPPORTED = 2
PD_ERR_CUDA = 3
PD_ERR_WORKSPACE = 4

METHOD = {"mp-pca": 0, "hybrid-pca": 1, "raw": 2, "nordic": 2, "optimal": 3, "adaptive": 4}
ADAPTIVE_MODE = {"sure": 0, "gsure": 1, "qut": 2}
ADAPTIVE_MAX_GAMMA = 32
RECOMBINATION = {"weighted": 0, "average": 1, "center": 2}
LOSS = {"fro": 0, "nuc": 1, "ope": 2}
PRECISION = {"fp32": 0, "mixed": 1}

c_i32, c_i64, c_dbl, c_vp, c_sz = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t


class Geometry(ctypes.Structure):
    """``pd_geometry``."""

    _fields_ = [
        ("shape", c_i64 * 4),
        ("patch", c_i64 * 4),
        ("step", c_i64 * 4),
        ("grid", c_i64 * 4),
        ("n_patches", c_i64),
        ("rows", c_i64),
        ("cols", c_i64),
    ]


class Params(ctypes.Structure):
    """``pd_params``."""

    _fields_ = [
        ("method", c_i32),
        ("recombination", c_i32),
        ("loss", c_i32),
        ("precision", c_i32),
        ("is_complex", c_i32),
        ("has_prior", c_i32),
        ("threshold_scale", c_dbl),
        ("threshold", c_dbl),
        ("mp_median", c_dbl),
    ]


class Adaptive(ctypes.Structure):
    """``pd_adaptive``."""

    _fields_ = [
        ("mode", c_i32),
        ("n_gamma", c_i32),
        ("has_tau0", c_i32),
        ("reserved", c_i32),
        ("tau0", c_dbl),
        ("qut_level", c_dbl),
        ("gamma", c_dbl * 32),
    ]


class Volume(ctypes.Structure):
    """``pd_volume``."""

    _fields_ = [
        ("geometry", Geometry),
        ("d_in", c_vp),
        ("d_noise_std", c_vp),
        ("d_patch_list", c_vp),
        ("n_selected", c_i64),
        ("d_out_acc", c_vp),
        ("d_weight_acc", c_vp),
        ("d_noise_acc", c_vp),
        ("d_noise_ctr", c_vp),
        ("d_rank_map", c_vp),
        ("d_patch_rank", c_vp),
        ("d_patch_noise", c_vp),
        ("threshold", c_dbl),
        ("mp_median", c_dbl),
    ]


class BatchTuning(ctypes.Structure):
    """``pd_batch_tuning``."""

    _fields_ = [("synth_row_blocks", c_i32), ("order_by_cost", c_i32), ("chunk_patches", c_i64)]


BATCH_MAX_VOLUMES = 64

G_P = ctypes.POINTER(Geometry)
P_P = ctypes.POINTER(Params)
A_P = ctypes.POINTER(Adaptive)

# name -> (restype, argtypes); every symbol declared in include/patch_denoise_b200.h
SIGNATURES = {
    "pd_version": (c_i32, []),
    "pd_last_error": (ctypes.c_char_p, []),
    "pd_geometry_init": (c_i32, [c_i32, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), G_P]),
    "pd_mp_median": (c_i32, [c_dbl, c_dbl, ctypes.POINTER(c_dbl)]),
    "pd_select_workspace_size": (c_i32, [G_P, ctypes.POINTER(c_sz)]),
    "pd_select_patches": (c_i32, [G_P, c_vp, c_i32, c_dbl, c_vp, c_vp, c_vp, c_sz, c_vp]),
    "pd_denoise_workspace_size": (c_i32, [G_P, P_P, c_i64, ctypes.POINTER(c_sz)]),
    "pd_denoise_patches": (
        c_i32,
        [G_P, P_P, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_sz, c_vp],
    ),
    "pd_finalize": (c_i32, [G_P, P_P, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp]),
    "pd_nordic_workspace_size": (c_i32, [c_i64, c_i64, c_i32, ctypes.POINTER(c_sz)]),
    "pd_nordic_mc_threshold": (c_i32, [c_i64, c_i64, c_i32, ctypes.c_uint64, c_i32, ctypes.POINTER(c_dbl), c_vp, c_sz, c_vp]),
    "pd_nordic_denoise_patches": (
        c_i32,
        [G_P, P_P, c_dbl, c_i64, c_i32, ctypes.c_uint64, c_vp, c_vp, c_sz, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp,
         c_vp, c_vp, c_vp, c_vp, c_vp, c_sz, c_vp],
    ),
    "pd_adaptive_qut_level": (c_i32, [c_i64, c_i64, c_i32, ctypes.c_uint64, c_i32, ctypes.POINTER(c_dbl), c_vp, c_sz, c_vp]),
    "pd_adaptive_denoise_patches": (
        c_i32,
        [G_P, P_P, A_P, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_sz, c_vp],
    ),
    "pd_denoise_patches_noalloc": (
        c_i32,
        [G_P, P_P, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp],
    ),
    "pd_noalloc_check": (c_i32, [c_vp]),
    "pd_denoise_batch_workspace_size": (c_i32, [ctypes.POINTER(Volume), c_i32, P_P, c_i64, ctypes.POINTER(c_sz)]),
    "pd_denoise_batch": (c_i32, [ctypes.POINTER(Volume), c_i32, P_P, ctypes.POINTER(BatchTuning), c_vp, c_sz, c_vp]),
    "pd_lowrank_backward_workspace_size": (c_i32, [G_P, c_i64, ctypes.POINTER(c_sz)]),
    "pd_lowrank_backward": (
        c_i32,
        [G_P, c_i32, c_i32, c_vp, c_vp, c_dbl, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_sz, c_vp],
    ),
    "pd_estimate_noise_workspace_size": (c_i32, [c_i32, ctypes.POINTER(c_i64), c_i32, ctypes.POINTER(c_sz)]),
    "pd_estimate_noise": (c_i32, [c_i32, ctypes.POINTER(c_i64), c_i32, c_vp, c_i32, c_vp, c_vp, c_sz, c_vp]),
    "pd_workspace_check": (c_i32, [c_vp, c_vp]),
    "pd_profile_enable": (c_i32, [c_i32]),
    "pd_profile_collect": (c_i32, [ctypes.c_char_p, c_sz]),
}


def profile_enable(on: bool) -> None:
    """Bracket every library kernel launch with CUDA events (see pd_profile_enable)."""
    load().pd_profile_enable(1 if on else 0)


def profile_collect() -> dict:
    """{kernel name: (launches, total_ms)} since the last collect; synchronises."""
    buf = ctypes.create_string_buffer(1 << 16)
    load().pd_profile_collect(buf, len(buf))
    res = {}
    for line in buf.value.decode().splitlines():
        name, n, ms = line.split()
        res[name] = (int(n), float(ms))
    return res

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load the shared library (once) and declare every entry point."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH.name} is not built: run `python -m patch_denoising_b200.build` "
                    "(the denoising path has no CPU fallback)"
                )
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


class PDError(RuntimeError):
    """A CUDA or workspace failure inside the library."""


def check(status: int) -> None:
    """Map a ``pd_status`` to the exception the reference would raise."""
    if status == PD_OK:
        return
    msg = load().pd_last_error().decode(errors="replace")
    if status == PD_ERR_INVALID:
        raise ValueError(msg)
    if status == PD_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise PDError(f"status {status}: {msg}")

"""ctypes binding of ``libsteam_b200.so`` (the C ABI of include/steam_b200.h).

Device memory is owned by torch tensors; their pointers and torch's current
CUDA stream are handed to the library.  There is no CPU fallback: without a
CUDA device, or without the built library, every entry point raises.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libsteam_b200.so"

STEAM_F32 = 0
STEAM_F64 = 1
STEAM_EPI_STORE = 0
STEAM_EPI_FLUX = 1
STEAM_EPI_STORE_WIDE = 2

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_u32 = ctypes.c_uint32
c_dbl = ctypes.c_double
c_size = ctypes.c_size_t
c_vp = ctypes.c_void_p
c_dp = ctypes.POINTER(ctypes.c_double)
c_i64p = ctypes.POINTER(ctypes.c_int64)


class Region(ctypes.Structure):
    """steam_region_t"""
    _fields_ = [("shape", c_i64 * 3), ("origin", c_i64 * 3), ("world", c_i64 * 3),
                ("sparsity", c_i32 * 3), ("key", c_u32 * 3)]


class Window(ctypes.Structure):
    """steam_window_t"""
    _fields_ = [("x0", c_i64), ("x1", c_i64), ("y0", c_i64), ("y1", c_i64)]


class BAProblem(ctypes.Structure):
    """steam_ba_problem_t: one field of a grouped bounded add."""
    _fields_ = [("nx", c_i64), ("ny", c_i64), ("nz", c_i64), ("pert", ctypes.c_void_p),
                ("increment", ctypes.c_void_p), ("mean", ctypes.c_void_p),
                ("phi_min", ctypes.c_double), ("phi_max", ctypes.c_double),
                ("has_window", c_i32), ("window", Window), ("ledger", ctypes.c_void_p)]


class ConvProblem(ctypes.Structure):
    """steam_conv_problem_t: one field of a grouped convolution."""
    _fields_ = [("nx", c_i64), ("ny", c_i64), ("nz", c_i64), ("in_", ctypes.c_void_p),
                ("out", ctypes.c_void_p), ("pre", ctypes.c_void_p), ("has_window", c_i32),
                ("window", Window), ("sums", ctypes.c_void_p)]


class ThermoProblem(ctypes.Structure):
    """steam_thermo_problem_t: one field of a grouped thermodynamics launch."""
    _fields_ = [("nx", c_i64), ("ny", c_i64), ("nz", c_i64), ("h", ctypes.c_void_p),
                ("qt", ctypes.c_void_p), ("prof", ctypes.c_void_p), ("compose", c_i32),
                ("bounds", ctypes.c_double * 4), ("surface_pressure", ctypes.c_double),
                ("ps_field", ctypes.c_void_p), ("T", ctypes.c_void_p), ("qv", ctypes.c_void_p),
                ("qc", ctypes.c_void_p), ("qi", ctypes.c_void_p), ("p", ctypes.c_void_p)]


class SepConv(ctypes.Structure):
    """steam_sepconv_t"""
    _fields_ = [("kz", c_i32), ("ky", c_i32), ("kx", c_i32),
                ("cz", c_i32), ("cy", c_i32), ("cx", c_i32),
                ("n_z", c_i32), ("n_y", c_i32), ("n_x", c_i32), ("n_pairs", c_i32),
                ("pair_z", c_i32 * 16), ("pair_y", c_i32 * 16), ("mix", c_dbl * 64)]


_SIGNATURES = {
    "steam_last_error": (ctypes.c_char_p, []),
    "steam_version": (ctypes.c_int, []),
    "steam_launch_count": (ctypes.c_ulonglong, []),
    "steam_keyed_uniforms": (ctypes.c_int, [c_vp, c_i64, c_vp, c_i64, c_vp, c_i64,
                                            c_u32, c_u32, c_u32, c_vp, c_vp, c_vp]),
    "steam_levy_field": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Region), c_dbl,
                                        c_vp, c_vp]),
    "steam_flux_noise_workspace_bytes": (c_size, []),
    "steam_flux_noise": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Region), c_dbl,
                                        c_dbl, c_dbl, c_i32, c_i32, c_i32, c_vp, c_vp,
                                        ctypes.POINTER(Window), c_dp, c_vp, c_size, c_vp]),
    "steam_conv_workspace_bytes": (c_size, [ctypes.c_int, c_i64, c_i64, c_i64,
                                            ctypes.POINTER(SepConv)]),
    "steam_conv_separable": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64,
                                            ctypes.POINTER(SepConv), c_dp, c_dp, c_dp,
                                            c_vp, c_dp, c_dp, c_vp, c_i32,
                                            ctypes.POINTER(Window), c_dp, c_vp, c_size,
                                            c_vp]),
    "steam_conv_set_xchunk": (ctypes.c_int, [c_i64, c_i64, c_i64, c_i32]),
    "steam_conv_get_xchunk": (ctypes.c_int, [c_i64, c_i64, c_i64]),
    "steam_conv_set_tile_rows": (ctypes.c_int, [c_i64, c_i64, c_i64, c_i32]),
    "steam_conv_get_tile_rows": (ctypes.c_int, [c_i64, c_i64, c_i64]),
    "steam_conv_set_flux_wide": (ctypes.c_int, [c_i32]),
    "steam_conv_group_workspace_bytes": (ctypes.c_size_t, [c_i32, ctypes.POINTER(ConvProblem)]),
    "steam_conv_group_prepare": (ctypes.c_int, [ctypes.POINTER(SepConv), c_dp, c_dp, c_dp,
                                                c_i32, ctypes.POINTER(ConvProblem), c_i32,
                                                c_vp, ctypes.c_size_t]),
    "steam_conv_group_async": (ctypes.c_int, [c_vp, c_vp]),
    "steam_conv_group_release": (ctypes.c_int, [c_vp]),
    "steam_take_wait_errors": (ctypes.c_int, [ctypes.POINTER(c_i32)]),
    "steam_set_copy_wait": (ctypes.c_int, [c_i64, c_i32]),
    "steam_conv_packed_launches": (c_i64, []),
    "steam_conv_fft_spectrum_bytes": (c_size, []),
    "steam_conv_fft_spectrum": (ctypes.c_int, [c_vp, c_i32, c_i32, c_i32, c_vp, c_vp]),
    "steam_conv_fft_workspace_bytes": (c_size, [c_i64, c_i64, c_i64]),
    "steam_conv_fft": (ctypes.c_int, [c_i64, c_i64, c_i64, c_i32, c_i32, c_i32, c_i32, c_i32,
                                      c_vp, c_vp, c_dp, c_dp, c_vp, c_i32,
                                      ctypes.POINTER(Window), c_dp, c_vp, c_size, c_vp]),
    "steam_conv_fft_async": (ctypes.c_int, [c_i64, c_i64, c_i64, c_i32, c_i32, c_i32, c_i32,
                                            c_i32, c_vp, c_vp, c_vp, c_vp, c_i32,
                                            ctypes.POINTER(Window), c_vp, c_vp, c_size, c_vp]),
    "steam_conv_direct_workspace_bytes": (c_size, [c_i64, c_i64, c_i64]),
    "steam_conv_direct": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_i32,
                                         c_i32, c_i32, c_i32, c_i32, c_vp, c_dp, c_dp, c_vp,
                                         c_i32, ctypes.POINTER(Window), c_dp, c_vp, c_size,
                                         c_vp]),
    "steam_conv_direct_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                               c_i32, c_i32, c_i32, c_i32, c_i32, c_vp, c_vp,
                                               c_vp, c_i32, ctypes.POINTER(Window), c_vp, c_vp,
                                               c_size, c_vp]),
    "steam_scale": (ctypes.c_int, [ctypes.c_int, c_i64, c_vp, c_dbl, c_i32, c_vp]),
    "steam_tile_extract": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_i64,
                                          c_i64, c_i64, c_i64, c_i64, c_i64, c_dbl, c_i32,
                                          c_vp, c_vp]),
    "steam_accumulate_levels": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                               c_vp, c_vp, c_dp, c_vp]),
    "steam_add_levels_clamp": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_dp,
                                              c_dbl, c_dbl, c_vp]),
    "steam_slab_zmajor": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_i64, c_i64,
                                         c_vp, c_vp]),
    "steam_flux_clip_workspace_bytes": (c_size, [c_i64, c_i64, c_i64]),
    "steam_flux_clip_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_vp,
                                             ctypes.POINTER(Window), c_vp, c_vp, c_size,
                                             c_vp]),
    "steam_box_h2d": (ctypes.c_int, [c_i32, c_vp, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64,
                                     c_i64, c_i64, c_i64, c_vp, c_vp]),
    "steam_box_d2h": (ctypes.c_int, [c_i32, c_vp, c_i64, c_i64, c_i64, c_i64, c_i64, c_i64,
                                     c_i64, c_i64, c_i64, c_vp, c_i64, c_i64, c_i64, c_i64,
                                     c_i64, c_i64, c_vp]),
    "steam_level_sums_workspace_bytes": (c_size, [c_i64]),
    "steam_level_sums": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                        ctypes.POINTER(Window), c_dp, c_vp, c_size, c_vp]),
    "steam_level_sums_noalloc_scratch_bytes": (c_size, []),
    "steam_level_sums_noalloc": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                                ctypes.POINTER(Window), c_dp, c_vp]),
    "steam_scalar_pattern_workspace_bytes": (c_size, [c_i64, c_i64, c_i64]),
    "steam_scalar_pattern": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_dp,
                                            c_vp, c_dbl, c_dbl, c_dbl, c_dp, c_dp, c_dp,
                                            c_dbl, c_dbl, c_vp, ctypes.POINTER(Window),
                                            c_dp, c_vp, c_size, c_vp]),
    "steam_bounded_add_workspace_bytes": (c_size, [c_i64, c_i32]),
    "steam_bounded_add": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_dp,
                                         c_vp, c_dbl, c_dbl, ctypes.POINTER(Window), c_i32,
                                         c_i32, c_dp, c_vp, c_size, c_vp]),
    "steam_set_barrier_spin_limit": (ctypes.c_int, [c_i64]),
    "steam_bounded_add_group_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int, c_i32,
                                                                 ctypes.POINTER(BAProblem),
                                                                 c_i32]),
    "steam_bounded_add_group_prepare": (ctypes.c_int, [ctypes.c_int, c_i32,
                                                       ctypes.POINTER(BAProblem), c_i32, c_vp,
                                                       ctypes.c_size_t]),
    "steam_bounded_add_group_async": (ctypes.c_int, [c_vp, c_vp]),
    "steam_bounded_add_group_release": (ctypes.c_int, [c_vp]),
    "steam_thermo_group_workspace_bytes": (ctypes.c_size_t, [c_i32, c_vp]),
    "steam_thermo_group_prepare": (ctypes.c_int, [ctypes.c_int, c_i32, c_vp, c_vp,
                                                  ctypes.c_size_t]),
    "steam_thermo_group_async": (ctypes.c_int, [c_vp, c_vp]),
    "steam_thermo_group_release": (ctypes.c_int, [c_vp]),
    "steam_bounded_add_ledger_doubles": (c_size, [c_i32]),
    "steam_project_bounds_replay": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                                   c_dp, c_dbl, c_dbl, c_dp, c_vp, c_size,
                                                   c_vp]),
    "steam_bounded_add_replay_workspace_bytes": (c_size, [c_i64, c_i32]),
    "steam_bounded_add_replay": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_dp,
                                                c_vp, c_dbl, c_dbl, c_i32, c_i32, c_dp, c_vp,
                                                c_size, c_vp]),
    "steam_bounded_add_replay_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                                      c_vp, c_vp, c_dbl, c_dbl, c_i32, c_i32,
                                                      c_vp, c_vp, c_size, c_vp]),
    "steam_project_bounds": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_dp,
                                            c_dbl, c_dbl, ctypes.POINTER(Window), c_dp,
                                            c_vp, c_size, c_vp]),
    "steam_regrid": (ctypes.c_int, [ctypes.c_int, c_vp, c_i64, c_i64, c_i64, c_vp, c_i64,
                                    c_i64, c_i64, c_i32, c_i32, c_vp]),
    "steam_thermo": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_vp, c_dp,
                                    c_dp, c_dp, c_dp, c_dbl, c_vp, c_vp, c_vp, c_vp, c_vp,
                                    c_vp, c_vp]),
    "steam_kernel_build": (ctypes.c_int, [ctypes.c_int, c_dbl, c_dbl, c_dbl, c_dbl, c_dbl,
                                          c_i32, c_vp, c_i64p, c_vp]),
    "steam_flux_noise_async": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Region), c_dbl,
                                              c_dbl, c_dbl, c_i32, c_i32, c_i32, c_vp, c_vp,
                                              ctypes.POINTER(Window), c_vp, c_vp, c_size,
                                              c_vp]),
    "steam_conv_separable_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64,
                                                  ctypes.POINTER(SepConv), c_dp, c_dp, c_dp,
                                                  c_vp, c_vp, c_vp, c_i32,
                                                  ctypes.POINTER(Window), c_vp, c_vp, c_size,
                                                  c_vp]),
    "steam_flux_finish_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_vp, c_vp, c_vp, c_dbl,
                                               c_vp, c_vp]),
    "steam_scalar_pattern_vectors": (ctypes.c_int, [ctypes.c_int, c_i64, c_dp, c_dp, c_dp,
                                                    c_dp, c_vp, c_vp]),
    "steam_scalar_pattern_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp,
                                                  c_vp, c_vp, c_vp, c_dbl, c_dbl, c_dp, c_i32,
                                                  c_dbl, c_dbl, c_vp, ctypes.POINTER(Window),
                                                  c_vp, c_vp, c_size, c_vp]),
    "steam_pattern_norm_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_vp, c_vp, c_vp, c_vp]),
    "steam_bounded_add_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_vp,
                                               c_vp, c_dbl, c_dbl, ctypes.POINTER(Window),
                                               c_i32, c_i32, c_vp, c_vp, c_size, c_vp]),
    "steam_thermo_async": (ctypes.c_int, [ctypes.c_int, c_i64, c_i64, c_i64, c_vp, c_vp, c_vp,
                                          c_i32, c_dp, c_dbl, c_vp, c_vp, c_vp, c_vp, c_vp,
                                          c_vp, c_vp]),
}

_lock = threading.Lock()
_lib = None


def exported_symbols() -> list[str]:
    """Names of every entry point the binding expects the library to export."""
    return sorted(_SIGNATURES)


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Load (once) and return the library; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = Path(path) if path is not None else LIB_PATH
        if not p.exists():
            raise RuntimeError(
                f"steam_b200: CUDA library {p} is missing; build it with "
                f"`python -m steam_b200.build` (nvcc, sm_100a). There is no CPU "
                f"fallback.")
        lib = ctypes.CDLL(str(p))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


_ERRORS = {1: ValueError, 2: RuntimeError, 3: MemoryError, 4: NotImplementedError}


def check(rc: int) -> None:
    if rc != 0:
        msg = load().steam_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, RuntimeError)(msg)


def require_cuda(who: str):
    """The torch module, after checking that a CUDA device is usable."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError(f"{who}: device='cuda' requested but torch.cuda is unavailable")
    return torch


def stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def dtype_code(t) -> int:
    import torch
    if t.dtype == torch.float32:
        return STEAM_F32
    if t.dtype == torch.float64:
        return STEAM_F64
    raise TypeError(f"steam_b200 computes in float32 or float64, got {t.dtype}")


def ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def dvec(values) -> ctypes.Array:
    a = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
    return (ctypes.c_double * max(1, a.size))(*a.ravel().tolist())


def dout(n: int) -> ctypes.Array:
    return (ctypes.c_double * max(1, n))()


class Workspace:
    """Scratch buffer per (device, stream), grown on demand.  Calls on one
    stream are ordered, so they may share it; calls on different streams get
    different buffers.  torch's caching allocator owns the memory."""

    def __init__(self):
        self._buf = {}

    def get(self, nbytes: int):
        import torch
        key = (torch.cuda.current_device(), torch.cuda.current_stream().cuda_stream)
        buf = self._buf.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")
            self._buf[key] = buf
        return buf

    def release(self):
        self._buf.clear()


WORKSPACE = Workspace()


def window_arg(window):
    if window is None:
        return None
    x0, x1, y0, y1 = (int(v) for v in window)
    return ctypes.byref(Window(x0, x1, y0, y1))

"""ctypes binding of libmvs_b200.so (include/mvs_b200.h).

The library is loaded from this package directory only; there is no fallback. A missing or
stale library raises at import of the calling module (``ensure()``), and every status code is
turned into the reference's exception type (ValueError / MemoryError / TimeoutError /
RuntimeError).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import threading

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
# MVS_LIBRARY=debug-bounds loads the bounds-checked debug build (python -m py_ortho_b200.build
# --debug-bounds) instead of the release library
LIB_PATH = os.path.join(HERE, "libmvs_b200_debug.so" if os.environ.get("MVS_LIBRARY") == "debug-bounds"
                        else "libmvs_b200.so")

MAX_SOURCES = 16
MAX_RADIUS = 7
MAX_PLANES_PER_CALL = 1024
BAND_MIN_POINTS = 50

OK, ERR_VALUE, ERR_MEMORY, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED = range(6)
HYP_MAPS, HYP_LINEAR, HYP_REFINE, HYP_PLANES = range(4)
PREC_FP32, PREC_FP16, PREC_FP64_SUMS, PREC_FP32_COMP, PREC_FP16_COMP = 0, 1, 2, 3, 4

vp = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64


class Hyp(C.Structure):
    _fields_ = [("kind", i32), ("n", i32), ("maps", vp), ("map_stride", i64), ("base", vp), ("step", vp),
                ("t0", i32), ("pad_", i32), ("planes", vp)]


class SweepArgs(C.Structure):
    _fields_ = [("H", i32), ("W", i32), ("ref", vp), ("mu", vp), ("sd", vp), ("ray", vp),
                ("n_src", i32), ("precision", i32), ("src", vp * MAX_SOURCES),
                ("src_h", i32 * MAX_SOURCES), ("src_w", i32 * MAX_SOURCES), ("geo", vp), ("ref_cam", vp),
                ("hyp", Hyp), ("i0", i32), ("i1", i32), ("r", i32), ("top_k", i32), ("plane_chunks", i32),
                ("tile_h", i32), ("best", vp), ("prev", vp), ("s_prev_best", vp), ("s_next_best", vp),
                ("idx", vp)]


class PMArgs(C.Structure):
    _fields_ = [("H", i32), ("W", i32), ("ref", vp), ("ray", vp), ("Cr", vp), ("S", i32), ("precision", i32),
                ("src", vp * MAX_SOURCES), ("src_depth", vp * MAX_SOURCES), ("src_h", i32 * MAX_SOURCES),
                ("src_w", i32 * MAX_SOURCES), ("par", vp), ("depth", vp), ("normal", vp), ("score", vp),
                ("active", vp), ("r", i32), ("step", i32), ("top_k", i32), ("iters", i32),
                ("geo_w", C.c_double), ("geo_tol", C.c_double), ("dmin", C.c_double), ("dmax", C.c_double),
                ("seed", C.c_uint32), ("it0", i32), ("changed", vp), ("rng_state", vp)]


class ConsArgs(C.Structure):
    _fields_ = [("H", i32), ("W", i32), ("depth", vp), ("cam", vp), ("n_nb", i32), ("pad_", i32),
                ("nb_depth", vp * MAX_SOURCES), ("nb_h", i32 * MAX_SOURCES), ("nb_w", i32 * MAX_SOURCES),
                ("nb_cam", vp), ("rel_tol", vp), ("px_tol", C.c_double), ("count", vp), ("grey", vp),
                ("score", vp), ("min_ncc", C.c_double), ("min_views", i32), ("pad2_", i32), ("active", vp)]


class FuseArgs(C.Structure):
    _fields_ = [("H", i32), ("W", i32), ("depth", vp), ("used", vp), ("cam", vp), ("n_nb", i32),
                ("point_stride", i32), ("nb_depth", vp * MAX_SOURCES), ("nb_used", vp * MAX_SOURCES),
                ("nb_h", i32 * MAX_SOURCES), ("nb_w", i32 * MAX_SOURCES), ("nb_cam", vp), ("rel_tol", vp),
                ("px_tol", C.c_double), ("min_views", i32), ("pad_", i32), ("keep", vp), ("xyz", vp),
                ("count", vp)]


class SampleViewArgs(C.Structure):
    _fields_ = [("h", i32), ("w", i32), ("nch", i32), ("img", vp), ("cam", vp), ("X0", C.c_double),
                ("Y0", C.c_double), ("gsd", C.c_double), ("D", i32), ("H", i32), ("W", i32), ("Z", vp),
                ("out", vp), ("valid", vp)]


class HeightScoreArgs(C.Structure):
    _fields_ = [("V", i32), ("D", i32), ("H", i32), ("W", i32), ("topk", i32), ("pad_", i32),
                ("full", C.c_double), ("min_texture", C.c_double), ("full_texture", C.c_double), ("M", vp),
                ("S2", vp), ("VA", vp), ("PP", vp), ("cxs", vp), ("cys", vp), ("cam_xy", vp), ("score", vp),
                ("st", vp), ("ref", vp)]


class DepthBandArgs(C.Structure):
    _fields_ = [("H", i32), ("W", i32), ("block", i32), ("n_pts", i32), ("X", vp), ("cam", vp), ("lo", C.c_double),
                ("hi", C.c_double), ("margin", C.c_double), ("nd", i32), ("pad_", i32), ("base", vp), ("step", vp),
                ("inv_hi", vp)]


class BatchJob(C.Structure):
    _fields_ = [("sweep", SweepArgs), ("depth", vp)]


class BatchTuning(C.Structure):
    _fields_ = [("plane_chunk", i32), ("ctas_per_sm", i32), ("tile_h", i32)]


# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "mvs_sweep": (i32, [vp, vp]),
    "mvs_sweep_noalloc": (i32, [vp, vp]),
    "mvs_sweep_hypothesis": (i32, [i32, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, i32, i32, i32,
                                   vp, vp, vp, vp, vp, vp]),
    "mvs_sweep_finalize": (i32, [i32, i32, vp, vp, vp, vp, vp, vp, vp]),
    "mvs_box_zero_mean": (i32, [i32, i32, vp, i32, i32, vp, vp]),
    "mvs_ref_stats": (i32, [i32, i32, vp, i32, vp, vp, vp]),
    "mvs_rays_grid": (i32, [i32, i32, vp, vp, vp]),
    "mvs_hyp_linear": (i32, [i32, i32, vp, vp, i64, vp, vp]),
    "mvs_hyp_refine": (i32, [i32, i32, vp, vp, i64, vp, vp]),
    "mvs_depth_view": (i32, [i32, i32, vp, vp, vp, vp, vp, vp, vp]),
    "mvs_half": (i32, [i32, i32, i32, vp, vp, vp]),
    "mvs_to_fp16": (i32, [i64, vp, vp, vp]),
    "mvs_tie_depths": (i32, [i32, vp, vp, i32, i32, vp, vp]),
    "mvs_depth_band": (i32, [vp, vp]),
    "mvs_pm_refine": (i32, [vp, vp]),
    "mvs_pm_stream_advance": (C.c_uint32, [C.c_uint32, C.c_uint64]),
    "mvs_batch_create": (i32, [vp, i32, vp, vp]),
    "mvs_batch_run": (i32, [vp, i32, vp]),
    "mvs_batch_stats": (i32, [vp, vp, vp]),
    "mvs_batch_destroy": (None, [vp]),
    "mvs_server_create": (i32, [i32, i32, i32, i32, vp]),
    "mvs_server_set_job": (i32, [vp, i32, vp, vp, i32]),
    "mvs_server_step": (i32, [vp, vp, vp, i32, vp]),
    "mvs_server_destroy": (None, [vp]),
    "mvs_consistency": (i32, [vp, vp]),
    "mvs_init_normals": (i32, [i32, i32, vp, vp, vp, vp]),
    "mvs_fuse_view": (i32, [vp, vp]),
    "mvs_sample_view": (i32, [vp, vp]),
    "mvs_box_sat_mean": (i32, [i32, i32, i32, vp, i32, vp, vp]),
    "mvs_height_score": (i32, [vp, vp]),
    "mvs_sgm": (i32, [i32, i32, i32, vp, C.c_float, C.c_float, vp, vp]),
    "mvs_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "mvs_device_faults": (i32, [vp]),
    "mvs_set_wait_limit": (C.c_uint32, [C.c_uint32]),
    "mvs_debug_bound_violations": (i32, [vp]),
    "mvs_version": (C.c_char_p, []),
}

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Loads the library (once). Raises if it has not been built: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"libmvs_b200.so is not built ({LIB_PATH}); run `python -m py_ortho_b200.build`")
            lib = C.CDLL(LIB_PATH)
            missing = [n for n in SIGNATURES if not hasattr(lib, n)]
            if missing:
                raise ImportError(f"libmvs_b200.so is stale: missing {', '.join(missing)}; rebuild it")
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    load().mvs_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    if status == OK:
        return
    msg = last_error() or what
    if status == ERR_VALUE:
        raise ValueError(msg)
    if status == ERR_MEMORY:
        raise MemoryError(msg)
    if status == ERR_TIMEOUT:
        raise TimeoutError(msg)
    if status == ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)


@contextlib.contextmanager
def nvtx(name: str):
    """An NVTX range around a phase of the host drivers (visible to Nsight Systems / ncu's NVTX
    filters); a no-op where NVTX is unavailable."""
    try:
        torch.cuda.nvtx.range_push(name)
        pushed = True
    except Exception:      # noqa: BLE001 - profiling aid only
        pushed = False
    try:
        yield
    finally:
        if pushed:
            torch.cuda.nvtx.range_pop()


def check_device_faults() -> None:
    """Raises TimeoutError when a bounded device-side wait gave up since the last check (the
    sweep's wait for its reference-tile copy: such tiles keep their previous state). Synchronises
    with the device; clears the count."""
    n = C.c_uint32(0)
    check(load().mvs_device_faults(C.byref(n)), "device faults")


def stream_handle(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("py_ortho_b200 runs on a CUDA device (sm_100a); no CUDA device is visible")
    return torch.device("cuda", torch.cuda.current_device())


def ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def host_f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, np.float64))


def host_ptr(a: np.ndarray) -> int:
    return int(a.ctypes.data)

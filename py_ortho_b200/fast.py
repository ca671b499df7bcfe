"""Drop-in replacements for the reference's depth-map helpers (``orthomosaic._fast``) that feed
the sweep: ``box_zero_mean``, ``hyp_linear``, ``hyp_refine``, ``rays_grid`` / ray grid, and
``depth_view``. Each is bit-identical to the reference helper (same float32 / float64 rounding
steps) and runs on the device. NumPy inputs return NumPy; torch CUDA inputs return torch.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L


def _in(a, dtype=torch.float32):
    dev = L.require_cuda()
    if isinstance(a, torch.Tensor):
        if a.dtype != dtype:
            a = a.to(dtype)
        return a.to(dev).contiguous(), False
    arr = np.ascontiguousarray(np.asarray(a), dtype=torch.empty((), dtype=dtype).numpy().dtype)
    return torch.from_numpy(arr).to(dev), True


def _out(t: torch.Tensor, host: bool):
    if host:
        torch.cuda.current_stream().synchronize()
        return t.cpu().numpy()
    return t


def box_zero_mean(a, r: int):
    """Zero-padded (2r+1)^2 window mean, float32 cumulative sums (_fast.pyx:661-713)."""
    if r < 0:
        raise ValueError("box_zero_mean needs r >= 0")
    t, host = _in(a)
    if t.ndim != 2:
        raise ValueError("box_zero_mean expects a 2-D array")
    out = torch.empty_like(t)
    L.check(L.load().mvs_box_zero_mean(t.shape[0], t.shape[1], t.data_ptr(), int(r), 0, out.data_ptr(),
                                       L.stream_handle()), "box_zero_mean")
    return _out(out, host)


def ref_stats(ref, r: int):
    """(mu, sd) of densify._sweep (densify.py:327-328) on the device."""
    t, host = _in(ref)
    mu = torch.empty_like(t)
    sd = torch.empty_like(t)
    L.check(L.load().mvs_ref_stats(t.shape[0], t.shape[1], t.data_ptr(), int(r), mu.data_ptr(), sd.data_ptr(),
                                   L.stream_handle()), "ref_stats")
    return _out(mu, host), _out(sd, host)


def hyp_linear(base, step, i: int):
    """(base + i * step) in float32 (_fast.pyx:628-641)."""
    b, host = _in(base)
    s, _ = _in(step)
    if b.shape != s.shape:
        raise ValueError("hyp_linear: shapes differ")
    out = torch.empty_like(b)
    L.check(L.load().mvs_hyp_linear(b.shape[0], b.shape[1], b.data_ptr(), s.data_ptr(), int(i), out.data_ptr(),
                                    L.stream_handle()), "hyp_linear")
    return _out(out, host)


def hyp_refine(iu, ds, t: int):
    """np.maximum(iu + t * ds, 1e-6) in float32, NaN propagating (_fast.pyx:644-658)."""
    a, host = _in(iu)
    d, _ = _in(ds)
    if a.shape != d.shape:
        raise ValueError("hyp_refine: shapes differ")
    out = torch.empty_like(a)
    L.check(L.load().mvs_hyp_refine(a.shape[0], a.shape[1], a.data_ptr(), d.data_ptr(), int(t), out.data_ptr(),
                                    L.stream_handle()), "hyp_refine")
    return _out(out, host)


def cam_row(cam) -> np.ndarray:
    """18-double camera row R(9) C(3) f k1 k2 k3 cx cy (the reference's PatchMatch `par` layout)."""
    return np.r_[np.asarray(cam.R, np.float64).ravel(), np.asarray(cam.C, np.float64),
                 [cam.f, cam.k1, cam.k2, cam.k3, cam.cx, cam.cy]].astype(np.float64)


def rays_world(shape, cam, host: bool = False):
    """(3, H, W) float32 world rays of every pixel (densify._rays_world with _fast.rays_grid,
    densify.py:288-297, _fast.pyx:145-198)."""
    H, W = int(shape[0]), int(shape[1])
    dev = L.require_cuda()
    out = torch.empty((3, H, W), dtype=torch.float32, device=dev)
    row = cam_row(cam)
    L.check(L.load().mvs_rays_grid(H, W, L.host_ptr(row), out.data_ptr(), L.stream_handle()), "rays_grid")
    return _out(out, host)


def init_normals(D, ray) -> torch.Tensor:
    """(3, H, W) float32 initial PatchMatch normals of depth map D (densify._init_normals,
    densify.py:481-496) on the device, bit-identical to the reference."""
    d_t, _ = _in(D)
    r_t, _ = _in(ray)
    H, W = int(d_t.shape[0]), int(d_t.shape[1])
    if tuple(r_t.shape) != (3, H, W):
        raise ValueError("init_normals: ray must be (3, H, W)")
    out = torch.empty((3, H, W), dtype=torch.float32, device=d_t.device)
    L.check(L.load().mvs_init_normals(H, W, d_t.data_ptr(), r_t.data_ptr(), out.data_ptr(), L.stream_handle()),
            "init_normals")
    return out


def depth_view(rgb, gain=None, bias=None, mask=None):
    """uint8 RGB -> (grey float32 with NaN = masked, rgb8 uint8) (_fast.pyx:577-624)."""
    t, host = _in(rgb, torch.uint8)
    if t.ndim != 3 or t.shape[2] != 3:
        raise ValueError("depth_view expects (h, w, 3) RGB")
    h, w = int(t.shape[0]), int(t.shape[1])
    m = None
    if mask is not None:
        m, _ = _in(np.asarray(mask, bool).view(np.uint8) if not isinstance(mask, torch.Tensor) else mask, torch.uint8)
        if tuple(m.shape) != (h, w):
            raise ValueError("mask shape differs from the image")
    g = None if gain is None else np.ascontiguousarray(np.asarray(gain, np.float32).reshape(-1)[:3])
    b = None if bias is None else np.ascontiguousarray(np.asarray(bias, np.float32).reshape(-1)[:3])
    grey = torch.empty((h, w), dtype=torch.float32, device=t.device)
    rgb8 = torch.empty((h, w, 3), dtype=torch.uint8, device=t.device)
    L.check(L.load().mvs_depth_view(h, w, t.data_ptr(), None if g is None else L.host_ptr(g),
                                    None if b is None else L.host_ptr(b), None if m is None else m.data_ptr(),
                                    grey.data_ptr(), rgb8.data_ptr(), L.stream_handle()), "depth_view")
    return _out(grey, host), _out(rgb8, host)


def half(g):
    """densify._half (densify.py:127-130) for (h, w) or stacked (c, h, w) float32 arrays."""
    t, host = _in(g)
    planes = 1 if t.ndim == 2 else int(t.shape[0])
    h, w = int(t.shape[-2]), int(t.shape[-1])
    shape = (h // 2, w // 2) if t.ndim == 2 else (planes, h // 2, w // 2)
    out = torch.empty(shape, dtype=torch.float32, device=t.device)
    L.check(L.load().mvs_half(planes, h, w, t.data_ptr(), out.data_ptr(), L.stream_handle()), "half")
    return _out(out, host)


def to_fp16(img: torch.Tensor, stream=None) -> torch.Tensor:
    """float32 device image -> FP16 storage copy (round to nearest) for MVS_PREC_FP16 sweeps."""
    t = img.contiguous()
    out = torch.empty(t.shape, dtype=torch.float16, device=t.device)
    L.check(L.load().mvs_to_fp16(t.numel(), t.data_ptr(), out.data_ptr(), L.stream_handle(stream)), "to_fp16")
    return out

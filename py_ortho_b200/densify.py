"""Drop-in replacement for the depth-map part of ``orthomosaic.densify``: ``_sweep`` and
``depth_map`` with the reference's arguments and outputs, running every pixel-level step on the
device (libmvs_b200) and only the small per-image geometry (depth range, tie-point band, number
of hypotheses) on the host, as the reference does in NumPy.

Reference: densify.py:57-81 (DepthOptions), :94-130 (_box, _norm, _half), :133-160 (_Cam),
:208-284 (depth range / band / count), :288-313 (_rays_world, _Hypotheses), :316-361 (_sweep),
:373-437 (depth_map), :481-496 (_init_normals).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import fast
from .dense import C_addr, Hypotheses, finalize, new_state, sweep


@dataclass
class DepthOptions:
    """The reference's depth-map options (densify.py:57-81), same names and defaults."""
    max_image_dim: int = 1600
    neighbors: int = 4
    num_depths: int = 64
    refine_steps: int = 3
    window: int = 5
    top_k: int = 2
    min_ncc: float = 0.3
    min_texture: float = 0.5
    min_views: int = 0
    consistency_px: float = 0.0
    consistency_depth: float = 0.0
    patchmatch: bool = False
    pm_iters: int = 2
    pm_window: int = 4
    pm_step: int = 2
    pm_geo_weight: float = 0.5
    layer_gap: float = 1.0
    keep_depthmaps: bool = False
    point_stride: int = 2
    cache_mb: int = 1200
    workers: int = 0
    precision: int = L.PREC_FP32      # PREC_FP16: FP16 source storage (constant-plane sweeps only);
    #                                   PREC_FP64_SUMS: window sums in float64 as the reference keeps them
    pm_precision: str = "fp64"        # PatchMatch cost: "fp64" (the reference's arithmetic) or "fp32"


class _Cam:
    """Pinhole + 3-term radial model, pixel centres at integers (densify.py:133-160)."""

    def __init__(self, R, C, f, k1, k2, cx, cy, w, h, k3=0.0):
        self.R, self.C = np.asarray(R, np.float64), np.asarray(C, np.float64)
        self.f, self.k1, self.k2, self.k3, self.cx, self.cy, self.w, self.h = f, k1, k2, k3, cx, cy, w, h

    def scaled(self, s: float, w: int, h: int) -> "_Cam":
        return _Cam(self.R, self.C, self.f * s, self.k1, self.k2, (self.cx + 0.5) * s - 0.5,
                    (self.cy + 0.5) * s - 0.5, w, h, self.k3)

    def project_cam(self, xc0, xc1, xc2):
        z = np.maximum(xc2, 1e-6)
        x, y = xc0 / z, xc1 / z
        r2 = x * x + y * y
        d = self.f * (1 + r2 * (self.k1 + r2 * (self.k2 + r2 * self.k3)))
        return d * x + self.cx, d * y + self.cy


class _Hypotheses:
    """Lazily generated inverse-depth maps (densify.py:300-313): ``make(i)`` -> (H, W) float32."""

    def __init__(self, make, n):
        self._make, self._n = make, n

    def __len__(self):
        return self._n

    def __getitem__(self, i):
        if not -self._n <= i < self._n:
            raise IndexError(i)
        return self._make(i % self._n)


def _pinhole(*cams) -> bool:
    return all(float(c.k1) == 0.0 and float(c.k2) == 0.0 and float(c.k3) == 0.0 for c in cams)


def _dev(a, dtype=torch.float32) -> torch.Tensor:
    dev = L.require_cuda()
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a), dtype=torch.empty((), dtype=dtype).numpy().dtype)).to(dev)


def _box(a, r: int):
    """Zero-padded window mean (densify.py:94-103), on the device."""
    return fast.box_zero_mean(a, r)


def _norm(grey):
    return ((np.asarray(grey) - 128.0) / 64.0).astype(np.float32)


def _half(g):
    return fast.half(g)


def _rays_world(shape, cam_r, host: bool = True):
    """(3, H, W) float32 world rays (densify.py:288-297), computed on the device."""
    return fast.rays_world(shape, cam_r, host=host)


def _geo(cam_r, cams_s) -> np.ndarray:
    rows = []
    for cs in cams_s:
        Rs = np.asarray(cs.R, np.float64)
        b = Rs @ (np.asarray(cam_r.C, np.float64) - np.asarray(cs.C, np.float64))
        rows.append(np.r_[Rs.ravel(), b, [cs.f, cs.k1, cs.k2, cs.k3, cs.cx, cs.cy]])
    return np.array(rows, np.float64)


def sweep_device(ref, cam_r, srcs, cams_s, hyp: Hypotheses, opt, ray=None, precision=None, plane_chunks=0):
    """The device form of _sweep: device tensors in, (depth, best, sd, state) device tensors out."""
    r = int(opt.window)
    precision = opt.precision if precision is None else precision
    ref_t = _dev(ref)
    H, W = int(ref_t.shape[0]), int(ref_t.shape[1])
    mu = torch.empty_like(ref_t)
    sd = torch.empty_like(ref_t)
    L.check(L.load().mvs_ref_stats(H, W, ref_t.data_ptr(), r, mu.data_ptr(), sd.data_ptr(), L.stream_handle()),
            "ref_stats")
    if precision == L.PREC_FP16:
        src_t = [s if (isinstance(s, torch.Tensor) and s.dtype == torch.float16 and s.is_cuda) else fast.to_fp16(_dev(s))
                 for s in srcs]
    else:
        src_t = [_dev(s) for s in srcs]
    geo = _geo(cam_r, cams_s)
    ray_t = None
    if hyp.kind != L.HYP_PLANES:
        ray_t = _dev(ray) if ray is not None else fast.rays_world((H, W), cam_r)
    ref_cam = fast.cam_row(cam_r) if hyp.kind == L.HYP_PLANES else None
    state = sweep(ref_t, mu, sd, ray_t, src_t, geo, hyp, r, int(opt.top_k), ref_cam=ref_cam, precision=precision,
                  plane_chunks=plane_chunks)
    depth = finalize(hyp, state)
    return depth, state[0], sd, state


def _sweep(ref, cam_r, srcs, cams_s, inv_list, opt, ray=None):
    """Winner-take-all over the inverse-depth hypotheses `inv_list` with the parabola refinement
    (densify.py:316-361). `inv_list` may be the reference's per-pixel maps (a list or _Hypotheses;
    they are streamed to the device in blocks) or a py_ortho_b200.dense.Hypotheses (generated on
    the device: constant planes, linear band, refinement). Returns (depth, best, sd) as NumPy
    arrays when `ref` is NumPy, else as device tensors."""
    host = not isinstance(ref, torch.Tensor)
    if isinstance(inv_list, Hypotheses):
        if inv_list.kind == L.HYP_PLANES and not _pinhole(cam_r, *cams_s):
            raise ValueError("_sweep: constant-plane hypotheses need pinhole cameras")
        depth, best, sd, _ = sweep_device(ref, cam_r, srcs, cams_s, inv_list, opt, ray)
    else:
        depth, best, sd = _sweep_maps(ref, cam_r, srcs, cams_s, inv_list, opt, ray)
    if host:
        torch.cuda.current_stream().synchronize()
        return depth.cpu().numpy(), best.cpu().numpy(), sd.cpu().numpy()
    return depth, best, sd


def _sweep_maps(ref, cam_r, srcs, cams_s, inv_list, opt, ray, block: int = 32):
    r = int(opt.window)
    ref_t = _dev(ref)
    H, W = int(ref_t.shape[0]), int(ref_t.shape[1])
    mu = torch.empty_like(ref_t)
    sd = torch.empty_like(ref_t)
    L.check(L.load().mvs_ref_stats(H, W, ref_t.data_ptr(), r, mu.data_ptr(), sd.data_ptr(), L.stream_handle()),
            "ref_stats")
    ray_t = _dev(ray) if ray is not None else fast.rays_world((H, W), cam_r)
    src_t = [_dev(s) for s in srcs]
    geo = _geo(cam_r, cams_s)
    n = len(inv_list)
    state = new_state(H, W, ref_t.device)
    first2 = []
    from .dense import sweep_args, C_addr
    for i0 in range(0, n, block):
        i1 = min(n, i0 + block)
        maps = torch.stack([_dev(inv_list[i]) for i in range(i0, i1)])
        if i0 == 0:
            first2 = [maps[0]] + ([maps[1]] if i1 > 1 else [])
        hyp = Hypotheses(L.HYP_MAPS, n, maps=maps)
        a, keep = sweep_args(ref_t, mu, sd, ray_t, src_t, geo, None, hyp, r, int(opt.top_k), state, i0=i0, i1=i1)
        L.check(L.load().mvs_sweep(C_addr(a), L.stream_handle()), "sweep")
        del keep
    fin = torch.stack(first2) if len(first2) == 2 else torch.stack([first2[0], first2[0]])
    depth = finalize(Hypotheses(L.HYP_MAPS, n, maps=fin), state)
    return depth, state[0], sd


# ------------------------------------------------------------------ tie-point priors of a view
def _cam_row(R, C, f, k1, k2, k3, cx, cy) -> np.ndarray:
    return np.ascontiguousarray(np.r_[np.asarray(R, np.float64).ravel(), np.asarray(C, np.float64), f, k1, k2, k3,
                                      cx, cy], np.float64)


def _depth_range(rec, k):
    """Depth search range of view k (densify.py:208-230). Every tie point of the block is
    projected into the view on the device (mvs_tie_depths); from the depths of those that land
    inside, the 1st-99th percentile interval is stretched far enough to reach the block's lowest
    ground (the 0.5th percentile of tie-point heights) along the optical axis - whose downward
    cosine is floored at 0.2 - and then padded: 20 % of the span each side, plus 1 m below the
    near end (kept above 30 % of it) and 2 m beyond the far end. None below 10 points."""
    intr = rec.intr[rec.cam_group[k]]
    X = np.ascontiguousarray(rec.X, np.float64)
    if X.shape[0] == 0:
        return None
    row = _cam_row(rec.R[k], rec.C[k], intr.f, 0.0, 0.0, 0.0, intr.cx, intr.cy)
    d_X = torch.from_numpy(X).to(L.require_cuda())
    z = torch.empty(X.shape[0], dtype=torch.float64, device=d_X.device)
    L.check(L.load().mvs_tie_depths(X.shape[0], d_X.data_ptr(), L.host_ptr(row), int(intr.width), int(intr.height),
                                    z.data_ptr(), L.stream_handle()), "tie_depths")
    z = z.cpu().numpy()
    seen = z[~np.isnan(z)]
    if seen.size < 10:
        return None
    near, far = np.percentile(seen, [1, 99])
    ground = float(np.percentile(X[:, 2], 0.5))
    cos_down = max(-float(rec.R[k][2, 2]), 0.2)
    far = max(far, (float(rec.C[k][2]) - ground) / cos_down)
    span = far - near
    return max(0.3 * near, near - 0.2 * span - 1.0), far + 0.2 * span + 2.0


def _band_maps(rec, k, cam, shape, rng, nd: int, block: int = 32, margin: float = 1.0):
    """The coarse sweep's linear hypothesis maps over the per-pixel inverse-depth band that view
    k's own tie points give (densify.py:233-274, 409-411), computed on the device
    (mvs_depth_band). Returns device tensors (base, step, inv_hi) at `shape`."""
    H, W = shape
    dev = L.require_cuda()
    pts = np.ascontiguousarray(rec.X[rec.obs_pt[rec.obs_cam == k]], np.float64)
    d_pts = torch.from_numpy(pts).to(dev) if len(pts) >= L.BAND_MIN_POINTS else None
    out = [torch.empty((H, W), dtype=torch.float32, device=dev) for _ in range(3)]
    row = _cam_row(cam.R, cam.C, cam.f, cam.k1, cam.k2, cam.k3, cam.cx, cam.cy)
    a = L.DepthBandArgs()
    a.H, a.W, a.block, a.n_pts = int(H), int(W), int(block), int(len(pts))
    a.X = 0 if d_pts is None else d_pts.data_ptr()
    a.cam = L.host_ptr(row)
    a.lo, a.hi, a.margin = float(rng[0]), float(rng[1]), float(margin)
    a.nd = int(nd)
    a.base, a.step, a.inv_hi = (t.data_ptr() for t in out)
    L.check(L.load().mvs_depth_band(C_addr(a), L.stream_handle()), "depth_band")
    return tuple(out)


def _num_depths(rec, k, nbrs_k, rng, f_coarse, base: int) -> int:
    """Coarse-sweep hypothesis count (densify.py:277-284): about one hypothesis per pixel of
    disparity that the median baseline to the neighbours spans over the depth range at the
    coarse focal length, kept within [base, 3 base]."""
    if not nbrs_k:
        return base
    baseline = float(np.median([np.linalg.norm(rec.C[k] - rec.C[j]) for j in nbrs_k]))
    span_px = f_coarse * baseline * (1.0 / rng[0] - 1.0 / rng[1])
    return int(min(max(math.ceil(span_px), base), 3 * base))


def _upsample2(a: torch.Tensor, H: int, W: int) -> torch.Tensor:
    """np.repeat(np.repeat(a, 2, 0), 2, 1)[:H, :W] padded with edge values to (H, W)."""
    up = a.repeat_interleave(2, 0).repeat_interleave(2, 1)[:H, :W]
    ph, pw = H - up.shape[0], W - up.shape[1]
    if ph or pw:
        up = torch.nn.functional.pad(up[None, None], (0, pw, 0, ph), mode="replicate")[0, 0]
    return up.contiguous()


def _per_pixel_precision(opt) -> int:
    """Sweeps over per-pixel hypothesis maps read float32 images; only the float64-sums mode
    carries over from the options (FP16 storage needs constant planes)."""
    return L.PREC_FP64_SUMS if opt.precision == L.PREC_FP64_SUMS else L.PREC_FP32


def depth_map(k, nbrs, rec, views, opt: DepthOptions):
    """Depth (camera-axis, metres) and NCC score for reference image `k` at matching scale, with the
    reference's coarse-to-fine schedule (densify.py:373-437): full sweep at 1/4 resolution over a
    per-pixel inverse-depth band, then +-refine_steps at 1/2 and full resolution. Returns
    (depth float32 with NaN, score float32, low_texture bool) as NumPy arrays, or None."""
    out = depth_map_device(k, nbrs, rec, views, opt)
    if out is None:
        return None
    depth, score, low = out
    torch.cuda.current_stream().synchronize()
    L.check_device_faults()
    return depth.cpu().numpy(), score.cpu().numpy(), low.cpu().numpy()


def depth_map_device(k, nbrs, rec, views, opt: DepthOptions):
    """depth_map with its results left on the device: (depth, score, low_texture) tensors, or None."""
    with L.nvtx(f"depth_map view {k}"):
        return _depth_map_device(k, nbrs, rec, views, opt)


def _depth_map_device(k, nbrs, rec, views, opt: DepthOptions):
    with L.nvtx("depth range"):
        rng = _depth_range(rec, k)
    if rng is None or not nbrs:
        return None
    ref, _, cam_r = views(k)
    ref = np.asarray(ref, np.float32)
    ref_mask = ~np.isfinite(ref)
    ref = np.ascontiguousarray(np.where(ref_mask, 0.0, ref), np.float32)
    src = [views(j) for j in nbrs]
    lv = 2
    pyr_r, pyr_c = [_dev(ref)], [cam_r]
    pyr_s, pyr_cs = [[_dev(s[0]) for s in src]], [[s[2] for s in src]]
    for _ in range(lv):
        r_ = fast.half(pyr_r[-1])
        pyr_r.append(r_)
        pyr_c.append(pyr_c[-1].scaled(0.5, r_.shape[1], r_.shape[0]))
        s_ = [fast.half(x) for x in pyr_s[-1]]
        pyr_s.append(s_)
        pyr_cs.append([c.scaled(0.5, x.shape[1], x.shape[0]) for c, x in zip(pyr_cs[-1], s_)])
    rays = [fast.rays_world(ref.shape, cam_r)]
    for lvl in range(1, lv + 1):
        h, w = pyr_r[lvl].shape
        rays.append(fast.half(rays[-1][:, :2 * h, :2 * w].contiguous()))
    nd = _num_depths(rec, k, nbrs, rng, pyr_c[lv].f, opt.num_depths)
    shape = tuple(pyr_r[lv].shape)
    with L.nvtx("tie-point band"):
        base_t, step_t, _ = _band_maps(rec, k, pyr_c[lv], shape, rng, nd, block=max(8, shape[1] // 16))
    with L.nvtx(f"coarse sweep {nd} hypotheses"):
        d, _, _, _ = sweep_device(pyr_r[lv], pyr_c[lv], pyr_s[lv], pyr_cs[lv], Hypotheses.linear(base_t, step_t, nd),
                                  opt, rays[lv], precision=_per_pixel_precision(opt))
    dstep = step_t / 2
    score = sd = None
    for lvl in range(lv - 1, -1, -1):
        H, W = pyr_r[lvl].shape
        up = _upsample2(d, H, W)
        dstep = _upsample2(dstep, H, W)
        iu = (1.0 / up).contiguous()
        with L.nvtx(f"refine level {lvl}"):
            d, score, sd, _ = sweep_device(pyr_r[lvl], pyr_c[lvl], pyr_s[lvl], pyr_cs[lvl],
                                           Hypotheses.refine(iu, dstep, opt.refine_steps), opt, rays[lvl],
                                           precision=_per_pixel_precision(opt))
        dstep = dstep / 2
    mask = torch.from_numpy(ref_mask).to(d.device)
    depth = torch.where(mask | (d < rng[0]) | (d > rng[1]), torch.full_like(d, float("nan")), d)
    low_texture = (sd * 64.0) < opt.min_texture
    return depth, score, low_texture


def _init_normals(D, ray):
    """World-frame normals from 2-px central differences, facing the camera (densify.py:481-496),
    computed on the device (mvs_init_normals); NumPy in, NumPy out."""
    n = fast.init_normals(D, ray)
    torch.cuda.current_stream().synchronize()
    return n.cpu().numpy()

"""The reference's legacy ground-grid height sweep (``mvs.dense_reconstruct``, mvs.py:138-434) on
the device: the thermal / ``dense_method="sweep"`` path of pyOrthomosaic, whose sampler is the
reference's only CUDA kernel on a dense path (CuPy ``sample_view``, _cuda.py:88-124).

For every cell of a north-up ground grid, heights are swept coarse-to-fine per tile: the full
range with semi-global matching on the coarsest level, then +-refine_steps around the upsampled
surface (with a parabola on the finest); the score is the windowed NCC of each view against the
cell's nearest fully-valid camera, averaged over the best half of the views and scaled by the
texture strength. A final pass at the chosen heights blends the true-ortho colour.

Device kernels (libmvs_b200): ``mvs_sample_view`` (bit-exact with the reference's CPU sampler
``_mvs.sample_view``), ``mvs_box_sat_mean`` (bit-exact with ``_fast.box_sat_mean``), the fused
``mvs_height_score`` and ``mvs_sgm`` (bit-exact with ``_mvs.sgm``). The per-tile host logic - grid
extent, view choice, blending of tiles - keeps the reference's NumPy code paths and values.
The reference's image loader is not part of this path: ``load_rgb(frame, scale)`` is passed in.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np
import torch

from . import _lib as L


@dataclass
class DenseOptions:
    """mvs.DenseOptions (mvs.py:31-51), same names and defaults."""
    gsd: Optional[float] = None
    levels: int = 3
    window: int = 3
    max_views: int = 6
    min_score: float = 0.5
    tile: int = 160
    overlap: int = 12
    max_cells: float = 40e6
    refine_steps: int = 4
    min_texture: float = 4.0
    full_texture: float = 8.0
    sgm_p1: float = 0.05
    sgm_p2: float = 0.6
    refine_min_score: float = 0.2
    view_angle_power: float = 1.5
    cache_mb: int = 1536
    workers: int = 0
    extent_trim: float = 1.0


@dataclass
class DenseResult:
    """mvs.DenseResult (mvs.py:54-63)."""
    Z: np.ndarray
    score: np.ndarray
    rgb: np.ndarray
    covered: np.ndarray
    minX: float
    maxY: float
    gsd: float
    stepped: Optional[np.ndarray] = None


def _dev():
    return L.require_cuda()


# ------------------------------------------------------------------ kernels
def sample_view(img: torch.Tensor, cam, X0: float, Y0: float, gsd: float, Z: torch.Tensor):
    """backend.sample_view (backend.py:67-76): img (h, w, ch) float32 on the device, cam = (R, C, f,
    k1, k2, k3, cx, cy) in img pixels, Z (H, W) or (D, H, W) heights -> (samples (..., ch), valid)."""
    img = img.contiguous()
    Zs = Z.to(torch.float32).contiguous()
    lead = Zs.shape[:-2]
    D = int(np.prod(lead)) if len(lead) else 1
    H, W = int(Zs.shape[-2]), int(Zs.shape[-1])
    h, w, nch = (int(v) for v in img.shape)
    out = torch.empty(tuple(Zs.shape) + (nch,), dtype=torch.float32, device=img.device)
    valid = torch.empty(tuple(Zs.shape), dtype=torch.uint8, device=img.device)
    R, C, f, k1, k2, k3, cx, cy = cam
    row = L.host_f64(np.r_[np.asarray(R, np.float64).ravel(), np.asarray(C, np.float64), [f, k1, k2, k3, cx, cy]])
    a = L.SampleViewArgs()
    a.h, a.w, a.nch, a.img, a.cam = h, w, nch, img.data_ptr(), L.host_ptr(row)
    a.X0, a.Y0, a.gsd = float(X0), float(Y0), float(gsd)
    a.D, a.H, a.W, a.Z, a.out, a.valid = D, H, W, Zs.data_ptr(), out.data_ptr(), valid.data_ptr()
    L.check(L.load().mvs_sample_view(ctypes.addressof(a), L.stream_handle()), "sample_view")
    return out, valid


def box(a: torch.Tensor, r: int) -> torch.Tensor:
    """backend.box on the CPU backend (_fast.box_sat_mean, float64 summed-area mean)."""
    a = a.to(torch.float32).contiguous()
    H, W = int(a.shape[-2]), int(a.shape[-1])
    B = int(a.numel() // max(H * W, 1))
    out = torch.empty_like(a)
    L.check(L.load().mvs_box_sat_mean(B, H, W, a.data_ptr(), int(r), out.data_ptr(), L.stream_handle()), "box")
    return out


def sgm(cost: torch.Tensor, P1: float, P2: float) -> torch.Tensor:
    """_mvs.sgm: 8-path aggregation of a (D, H, W) float32 cost volume."""
    cost = cost.to(torch.float32).contiguous()
    D, H, W = (int(v) for v in cost.shape)
    agg = torch.empty_like(cost)
    L.check(L.load().mvs_sgm(D, H, W, cost.data_ptr(), float(P1), float(P2), agg.data_ptr(), L.stream_handle()),
            "sgm")
    return agg


# ------------------------------------------------------------------ grid, views, tiles
@dataclass
class Grid:
    """The north-up DSM grid: top-left cell corner (minX, maxY), size, cell size and the image
    scale that makes one image pixel about one cell."""
    minX: float
    maxY: float
    W: int
    H: int
    gsd: float
    img_scale: float


def _ground_corners(rec, z: float) -> np.ndarray:
    """The image corners of every used camera on the plane Z = z (rays pointing down only)."""
    out = []
    for k in range(len(rec.used)):
        it = rec.intr[rec.cam_group[k]]
        Rt, C = rec.R[k].T, rec.C[k]
        for u, v in ((0, 0), (it.width, 0), (it.width, it.height), (0, it.height)):
            ray = Rt @ np.array([(u - it.cx) / it.f, (v - it.cy) / it.f, 1.0])
            if ray[2] < -1e-6:
                out.append(C + ray * (z - C[2]) / ray[2])
    return np.array(out)


def grid_extent(rec, gsd: float, native_gsd: float, max_cells: float = 40e6, trim: float = 1.0) -> Grid:
    """The grid of mvs.grid_extent (mvs.py:95-135): the camera footprints on the 20th-percentile
    tie-point height, `trim` percent of the extreme corners dropped per side, snapped outwards to
    whole cells; the cell grows when the area would exceed max_cells."""
    zg = float(np.percentile(rec.X[:, 2], 20)) if len(rec.X) else 0.0
    P = _ground_corners(rec, zg)

    def snap(g):
        lo_x = math.floor(np.percentile(P[:, 0], trim) / g) * g
        hi_x = math.ceil(np.percentile(P[:, 0], 100 - trim) / g) * g
        lo_y = math.floor(np.percentile(P[:, 1], trim) / g) * g
        hi_y = math.ceil(np.percentile(P[:, 1], 100 - trim) / g) * g
        return lo_x, hi_x, lo_y, hi_y

    x0, x1, y0, y1 = snap(gsd)
    if (x1 - x0) * (y1 - y0) / gsd ** 2 > max_cells:
        gsd = math.sqrt((x1 - x0) * (y1 - y0) / max_cells)
        x0, x1 = math.floor(x0 / gsd) * gsd, math.ceil(x1 / gsd) * gsd
        y0, y1 = math.floor(y0 / gsd) * gsd, math.ceil(y1 / gsd) * gsd
    return Grid(x0, y1, int(round((x1 - x0) / gsd)), int(round((y1 - y0) / gsd)), gsd, min(1.0, native_gsd / gsd))


def _halve(g: np.ndarray) -> np.ndarray:
    """One 2x2-mean pyramid step of an (h, w, 1) float32 image (odd edges dropped)."""
    h, w = g.shape[0] // 2 * 2, g.shape[1] // 2 * 2
    q = g[:h, :w, 0]
    return ((q[0::2, 0::2] + q[1::2, 0::2] + q[0::2, 1::2] + q[1::2, 1::2]) * 0.25)[..., None].astype(np.float32)


def _feather(h: int, w: int) -> np.ndarray:
    """Colour weight: distance to the nearest image border over half the short side, clipped to 1."""
    s = 0.5 * min(h, w)
    fy = np.minimum(np.arange(h) + 0.5, h - 0.5 - np.arange(h)) / s
    fx = np.minimum(np.arange(w) + 0.5, w - 0.5 - np.arange(w)) / s
    return np.clip(np.minimum(fy[:, None], fx[None, :]), 0, 1).astype(np.float32)


class _View:
    """A camera with its grey pyramid (h, w, 1) and feathered RGBW image (h, w, 4) on the device."""

    def __init__(self, pyr, rgbw, R, C, f, k1, k2, k3, cx, cy):
        self.pyr, self.rgbw, self.R, self.C = pyr, rgbw, R, C
        self.f, self.k1, self.k2, self.k3, self.cx, self.cy = f, k1, k2, k3, cx, cy

    def cam(self, level: int):
        """(R, C, f, k1, k2, k3, cx, cy) in the pixels of pyramid level `level`."""
        s = 0.5 ** level
        return self.R, self.C, self.f * s, self.k1, self.k2, self.k3, (self.cx + 0.5) * s - 0.5, (self.cy + 0.5) * s - 0.5


def _make_view(rec, k, frame, rgb_u8, gains, biases, levels, dev) -> _View:
    """The view of used camera k: gains / offsets, BT.601 grey, pyramid, feather channel."""
    i = rec.used[k]
    rgb = rgb_u8.astype(np.float32)
    if gains.get(i) is not None:
        rgb *= np.asarray(gains[i], np.float32)
    if biases is not None and biases.get(i) is not None:
        rgb += np.asarray(biases[i], np.float32)
    grey = np.ascontiguousarray((0.299 * rgb[..., 0] + 0.587 * rgb[..., 1] + 0.114 * rgb[..., 2])[..., None], np.float32)
    pyr = [grey]
    while len(pyr) < levels:
        pyr.append(np.ascontiguousarray(_halve(pyr[-1])))
    rgbw = np.ascontiguousarray(np.dstack([rgb, _feather(*rgb.shape[:2])]))
    it = rec.intr[rec.cam_group[k]]
    sx = rgb.shape[1] / frame.width
    return _View([torch.from_numpy(p).to(dev) for p in pyr], torch.from_numpy(rgbw).to(dev),
                 np.ascontiguousarray(rec.R[k]), np.ascontiguousarray(rec.C[k]), it.f * sx, it.k1, it.k2, it.k3,
                 (it.cx + 0.5) * sx - 0.5, (it.cy + 0.5) * sx - 0.5)


@dataclass
class _Tile:
    tx: int
    ty: int
    tw: int
    th: int
    pad: int
    X0: float                 # top-left corner of the padded tile
    Y0: float
    PW: int
    PH: int
    views: list               # used-camera indices, most central first (the first sees the whole tile)


def _tile_views(rec, g: Grid, tx, ty, tw, th, pad, z_fallback, max_views):
    """The views of a tile: by distance of their camera to the tile centre, those that see the
    whole padded tile at the tile's sparse-point height band (5th-95th percentile, or the global
    range with fewer than 20 points); cameras that see part of it only fill up a tile that has
    fewer than two. None if fewer than two cameras see it at all."""
    X0, Y0 = g.minX + (tx - pad) * g.gsd, g.maxY - (ty - pad) * g.gsd
    PW, PH = tw + 2 * pad, th + 2 * pad
    Xs = rec.X
    m = (Xs[:, 0] > X0) & (Xs[:, 0] < X0 + PW * g.gsd) & (Xs[:, 1] < Y0) & (Xs[:, 1] > Y0 - PH * g.gsd)
    z_lo, z_hi = np.percentile(Xs[m, 2], [5, 95]) if m.sum() >= 20 else z_fallback
    xy = np.array([[X0, Y0], [X0 + PW * g.gsd, Y0], [X0, Y0 - PH * g.gsd], [X0 + PW * g.gsd, Y0 - PH * g.gsd]])
    box = np.concatenate([np.column_stack([xy, np.full(4, z)]) for z in (z_lo, z_hi)])
    centre = (g.minX + (tx + tw / 2) * g.gsd, g.maxY - (ty + th / 2) * g.gsd)
    order = np.argsort(np.hypot(rec.C[:, 0] - centre[0], rec.C[:, 1] - centre[1]))
    full, part = [], []
    for k in order:
        it = rec.intr[rec.cam_group[k]]
        xc = (box - rec.C[k]) @ rec.R[k].T
        if np.any(xc[:, 2] <= 0):
            continue
        u = it.f * xc[:, 0] / xc[:, 2] + it.cx
        v = it.f * xc[:, 1] / xc[:, 2] + it.cy
        seen = (u >= 0) & (u <= it.width - 1) & (v >= 0) & (v <= it.height - 1)
        (full if seen.all() else part if seen.any() else []).append(int(k))
        if len(full) >= max_views:
            break
    views = full if len(full) >= 2 else (full + part)[:max_views]
    if len(views) < 2:
        return None
    return _Tile(tx, ty, tw, th, pad, X0, Y0, PW, PH, views)


def _serpentine(W: int, H: int, T: int):
    """Tile origins row by row, every other row reversed (neighbouring tiles share views)."""
    for r, ty in enumerate(range(0, H, T)):
        row = list(range(0, W, T))
        for tx in (row if r % 2 == 0 else row[::-1]):
            yield tx, ty


def _median3(a: torch.Tensor) -> torch.Tensor:
    """3x3 median with edge padding (mvs._median3, mvs.py:64-68): the middle of the 9 sorted shifts."""
    p = torch.nn.functional.pad(a[None, None], (1, 1, 1, 1), mode="replicate")[0, 0]
    H, W = a.shape
    return torch.sort(torch.stack([p[dy:dy + H, dx:dx + W] for dy in range(3) for dx in range(3)]), dim=0).values[4]


# ------------------------------------------------------------------ one tile on the device
class _TileSweep:
    """Coarse-to-fine height search of one tile (mvs.py:224-380 semantics) on the device."""

    def __init__(self, tile: _Tile, views, opt: DenseOptions, gsd: float, dev):
        self.t, self.views, self.opt, self.gsd, self.dev = tile, views, opt, gsd, dev
        V = len(views)
        self.topk = max(1, V // 2)
        self.cams = [np.asarray(v.C, np.float64) for v in views]
        self.cam_xy = L.host_f64(np.array([[c[0], c[1]] for c in self.cams], np.float64))
        ia, ib = np.triu_indices(V, 1)
        self.ia = torch.as_tensor(ia, device=dev)
        self.ib = torch.as_tensor(ib, device=dev)

    def score(self, Z: torch.Tensor, level: int, gsd_l: float, detail: bool = False):
        """Photo-consistency of every cell of the height stack Z (..., HH, WW): the samples of every
        view, all box means in one call, then the fused per-cell score kernel."""
        t, V, dev, opt = self.t, len(self.views), self.dev, self.opt
        HH, WW = int(Z.shape[-2]), int(Z.shape[-1])
        smp, val = [], []
        for v in self.views:
            out, ok = sample_view(v.pyr[min(level, len(v.pyr) - 1)], v.cam(level), t.X0, t.Y0, gsd_l, Z)
            smp.append(out[..., 0])
            val.append(ok)
        S = torch.stack(smp)
        boxes = box(torch.cat([S, S * S, torch.stack(val).to(torch.float32), S[self.ia] * S[self.ib]]), opt.window)
        lead = tuple(Z.shape[:-2])
        score = torch.empty(lead + (HH, WW), dtype=torch.float32, device=dev)
        st = torch.empty((V,) + lead + (HH, WW), dtype=torch.float32, device=dev) if detail else None
        ref = torch.empty(lead + (HH, WW), dtype=torch.int32, device=dev) if detail else None
        cxs = torch.as_tensor(np.asarray(t.X0 + (np.arange(WW) + 0.5) * gsd_l, np.float32), device=dev)
        cys = torch.as_tensor(np.asarray(t.Y0 - (np.arange(HH) + 0.5) * gsd_l, np.float32), device=dev)
        a = L.HeightScoreArgs()
        a.V, a.D, a.H, a.W, a.topk = V, int(np.prod(lead)) if lead else 1, HH, WW, self.topk
        a.full, a.min_texture, a.full_texture = 1.0 - 1e-6, float(opt.min_texture), float(opt.full_texture)
        a.M, a.S2, a.VA, a.PP = (boxes[:V].data_ptr(), boxes[V:2 * V].data_ptr(), boxes[2 * V:3 * V].data_ptr(),
                                 boxes[3 * V:].data_ptr())
        a.cxs, a.cys, a.cam_xy, a.score = cxs.data_ptr(), cys.data_ptr(), L.host_ptr(self.cam_xy), score.data_ptr()
        a.st, a.ref = (st.data_ptr(), ref.data_ptr()) if detail else (0, 0)
        L.check(L.load().mvs_height_score(ctypes.addressof(a), L.stream_handle()), "height score")
        return (score, st, val, ref.to(torch.int64)) if detail else score

    def coarse(self, level, zlo, zhi):
        """Every height from zlo to zhi in steps of one cell, 64 at a time; cost 1 - score,
        8-path SGM, the cheapest height per cell."""
        t, dev = self.t, self.dev
        s = 2 ** level
        HH, WW, gsd_l = (t.PH + s - 1) // s, (t.PW + s - 1) // s, self.gsd * s
        zs = np.arange(zlo, zhi + gsd_l, gsd_l).astype(np.float32)
        vol = torch.cat([self.score(torch.as_tensor(zs[c:c + 64], device=dev)[:, None, None].expand(-1, HH, WW)
                                    .contiguous(), level, gsd_l) for c in range(0, len(zs), 64)])
        agg = sgm((1.0 - torch.clamp(vol, -1.0, 1.0)).contiguous(), self.opt.sgm_p1, self.opt.sgm_p2)
        return torch.as_tensor(zs, device=dev)[torch.argmin(agg, dim=0)]

    def refine(self, Zc, level):
        """+-refine_steps cells around the upsampled coarser surface; cells whose best score is
        weak keep it; on the finest level a parabola through the neighbours' scores."""
        t, opt, dev = self.t, self.opt, self.dev
        s = 2 ** level
        HH, WW, gsd_l = (t.PH + s - 1) // s, (t.PW + s - 1) // s, self.gsd * s
        up = Zc.repeat_interleave(2, 0).repeat_interleave(2, 1)[:HH, :WW]
        if tuple(up.shape) != (HH, WW):
            up = torch.nn.functional.pad(up[None, None], (0, WW - up.shape[1], 0, HH - up.shape[0]),
                                         mode="replicate")[0, 0]
        n = opt.refine_steps
        offs = torch.as_tensor((np.arange(-n, n + 1) * gsd_l).astype(np.float32), device=dev)
        sc = self.score((up[None] + offs[:, None, None]).to(torch.float32), level, gsd_l)
        bi = torch.argmax(sc, dim=0)
        pick = lambda i: torch.gather(sc, 0, i[None])[0]
        bi = torch.where(pick(bi) < np.float32(opt.refine_min_score), torch.full_like(bi, n), bi)
        best = pick(bi)
        frac = torch.zeros_like(best)
        if level == 0:
            s_lo, s_hi = pick(torch.clamp(bi - 1, 0, 2 * n)), pick(torch.clamp(bi + 1, 0, 2 * n))
            den = s_lo - 2 * best + s_hi
            ok = (den < np.float32(-1e-6)) & (bi > 0) & (bi < 2 * n)
            den = torch.where(ok, den, torch.full_like(den, -1.0))
            frac = torch.where(ok, torch.clamp(0.5 * (s_lo - s_hi) / den, -0.5, 0.5), torch.zeros_like(den))
        return up + offs[bi] + frac * np.float32(gsd_l)

    def colour(self, Z, st, ref):
        """True-ortho colour at the chosen heights: feather^2 x agreement with the cell's reference
        x validity x cos(incidence)^power weighted mean of the views' RGB."""
        t, dev = self.t, self.dev
        cx = torch.as_tensor((t.X0 + (np.arange(t.PW) + 0.5) * self.gsd).astype(np.float32), device=dev)
        cy = torch.as_tensor((t.Y0 - (np.arange(t.PH) + 0.5) * self.gsd).astype(np.float32), device=dev)
        p = float(self.opt.view_angle_power)
        acc = torch.zeros(tuple(Z.shape) + (3,), dtype=torch.float32, device=dev)
        wsum = torch.zeros(tuple(Z.shape), dtype=torch.float32, device=dev)
        for vi, v in enumerate(self.views):
            rgbw, ok = sample_view(v.rgbw, v.cam(0), t.X0, t.Y0, self.gsd, Z)
            agree = torch.where(ref == vi, torch.ones_like(st[vi]),
                                torch.clamp((st[vi] + np.float32(0.2)) / np.float32(0.6), 0.0, 1.0))
            C = self.cams[vi]
            dz = np.float32(C[2]) - Z
            dx = cx[None, :] - np.float32(C[0])
            dy = cy[:, None] - np.float32(C[1])
            cos_inc = torch.clamp(dz / torch.sqrt(dx * dx + dy * dy + dz * dz + np.float32(1e-6)), 0.0, 1.0)
            w = rgbw[..., 3] ** 2 * agree * ok.to(torch.float32) * cos_inc ** p
            acc = acc + rgbw[..., :3] * w[..., None]
            wsum = wsum + w
        return acc / torch.clamp(wsum, min=1e-6)[..., None]


# ------------------------------------------------------------------ the sweep
def dense_reconstruct(ar, rec, gains: dict, native_gsd: float, opt: DenseOptions, biases: Optional[dict] = None,
                      load_rgb: Callable = None) -> DenseResult:
    """mvs.dense_reconstruct (mvs.py:138-434) on the device, one tile after another in serpentine
    order (the reference's schedule for GPU backends). ``load_rgb(frame, scale)`` returns the frame's
    uint8 RGB at `scale` (the reference's imageio.load_rgb). Same arguments and result type."""
    dev = _dev()
    g = grid_extent(rec, opt.gsd or native_gsd, native_gsd, opt.max_cells, opt.extent_trim)
    levels = max(1, opt.levels)
    zg = float(np.percentile(rec.X[:, 2], 20)) if len(rec.X) else 0.0
    if len(rec.X):
        q1, q99 = np.percentile(rec.X[:, 2], [1, 99])
        z_band = (q1 - (0.1 * (q99 - q1) + 1.0), q99 + (0.1 * (q99 - q1) + 1.0))
    else:
        z_band = (zg - 5, zg + 30)
    zlo, zhi = z_band[0] - 1.0, z_band[1] + 1.0
    pad = opt.window * (2 ** (levels - 1)) + 4
    ov = min(pad, opt.overlap)
    Zacc = np.zeros((g.H, g.W), np.float32)
    Wacc = np.zeros((g.H, g.W), np.float32)
    out = DenseResult(None, np.full((g.H, g.W), -1.0, np.float32), np.zeros((g.H, g.W, 3), np.uint8),
                      np.zeros((g.H, g.W), bool), g.minX, g.maxY, g.gsd)
    views = {}

    def view(k):
        if k not in views:
            fr = ar.frames[rec.used[k]]
            views[k] = _make_view(rec, k, fr, load_rgb(fr, g.img_scale), gains, biases, levels, dev)
        return views[k]

    T = opt.tile
    for tx, ty in _serpentine(g.W, g.H, T):
        tw, th = min(T, g.W - tx), min(T, g.H - ty)
        tile = _tile_views(rec, g, tx, ty, tw, th, pad, (zlo, zhi), opt.max_views)
        if tile is None:
            continue
        sw = _TileSweep(tile, [view(k) for k in tile.views], opt, g.gsd, dev)
        Z = None
        for level in range(levels - 1, -1, -1):
            Z = sw.coarse(level, zlo, zhi) if Z is None else sw.refine(Z, level)
            Z = _median3(Z.to(torch.float32)) if level > 0 else Z.to(torch.float32)
        score, st, valids, ref = sw.score(Z, 0, g.gsd, detail=True)
        colour = sw.colour(Z, st, ref)
        nvalid = sum(v.to(torch.int32) for v in valids)
        # heights leave the tile with an overlap margin, blended by a linear ramp
        e = (max(0, tx - ov), max(0, ty - ov), min(g.W, tx + tw + ov), min(g.H, ty + th + ov))
        ry, rx = np.arange(e[1], e[3]), np.arange(e[0], e[2])
        wy = np.clip(np.minimum(ry - (ty - ov) + 0.5, (ty + th + ov) - ry - 0.5) / max(2 * ov, 1), 0, 1)
        wx = np.clip(np.minimum(rx - (tx - ov) + 0.5, (tx + tw + ov) - rx - 0.5) / max(2 * ov, 1), 0, 1)
        ramp = (np.minimum(wy[:, None], wx[None, :]) if ov > 0 else np.ones((len(ry), len(rx)))).astype(np.float32)
        z = Z[e[1] - ty + pad:e[3] - ty + pad, e[0] - tx + pad:e[2] - tx + pad].cpu().numpy()
        Zacc[e[1]:e[3], e[0]:e[2]] += z * ramp
        Wacc[e[1]:e[3], e[0]:e[2]] += ramp
        inner = (slice(pad, pad + th), slice(pad, pad + tw))
        out.score[ty:ty + th, tx:tx + tw] = score[inner].cpu().numpy()
        out.rgb[ty:ty + th, tx:tx + tw] = np.clip(colour[inner].cpu().numpy(), 0, 255).astype(np.uint8)
        out.covered[ty:ty + th, tx:tx + tw] = (nvalid[inner] >= 2).cpu().numpy()
    out.Z = np.where(Wacc > 0, Zacc / np.maximum(Wacc, 1e-6), np.nan).astype(np.float32)
    return out

"""Multi-view depth maps: passes 1 and 2 of the reference's densification (densify.py:513-640) on
the device, views sharded over the ranks of a ``torch.distributed`` group.

* Pass 1 - one depth map per view (``densify.depth_map_device``: coarse-to-fine plane sweep).
* Exchange - every pass-1 map that a view on another rank names as a neighbour is broadcast from
  the rank that made it. This is the path's only data exchange (NCCL over NVLink between GPUs;
  gloo on CPU in the tests); views themselves are independent.
* Pass 2 - per view, the geometric consistency count against the neighbours' maps
  (``mvs_consistency``), PatchMatch repair of the pixels it selects with the neighbours' maps in
  the geometric term (``mvs_pm_refine``), then the final score / texture filter (``repair``,
  densify.py:611-640).

Views are assigned to ranks by longest-processing-time order on their pixel x neighbour cost,
deterministically, so every rank computes the same assignment and takes the same collective
steps in the same order.

The reference keeps pass-1 maps on disk between the passes (``p*.npy`` float32 depth,
``s*.npy`` float16 score, ``t*.npy`` bool low-texture mask, densify.py:587-593); here they stay
in device memory with the same value formats (the score is rounded through float16, as the
reference's pass 2 reads it).
"""
from __future__ import annotations

import ctypes
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from . import dense, fast
from .densify import DepthOptions, _depth_range, depth_map_device


# ------------------------------------------------------------------ device kernels
def cam_row(cam) -> np.ndarray:
    """R (9), C (3), f, k1, k2, k3, cx, cy of a densify._Cam-like camera (float64)."""
    return fast.cam_row(cam)


def _dev32(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float32).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)


def consistency(D, cam_r, nb_maps: Sequence, nb_cams: Sequence, px_tol: float, rel_tol: Sequence[float],
                grey=None, score=None, min_ncc: float = 0.0, min_views: int = 0):
    """Agreeing-neighbour count per pixel of depth map D (densify._consistency, densify.py:441-478)
    and, with ``grey`` and ``score``, pass 2's PatchMatch mask (densify.py:621). Device tensors in,
    device tensors out: (count int16, active uint8 or None)."""
    dev = L.require_cuda()
    d_t = _dev32(D, dev)
    H, W = int(d_t.shape[0]), int(d_t.shape[1])
    n = len(nb_maps)
    if n != len(nb_cams) or n != len(rel_tol):
        raise ValueError("consistency: nb_maps, nb_cams and rel_tol differ in length")
    if n > L.MAX_SOURCES:
        raise ValueError(f"consistency: {n} neighbours (at most {L.MAX_SOURCES})")
    maps = [_dev32(m, dev) for m in nb_maps]
    row = L.host_f64(cam_row(cam_r))
    rows = L.host_f64(np.array([cam_row(c) for c in nb_cams], np.float64).reshape(-1) if n else np.zeros(1))
    tol = L.host_f64(np.asarray(rel_tol, np.float64).reshape(-1) if n else np.zeros(1))
    count = torch.empty((H, W), dtype=torch.int16, device=dev)
    a = L.ConsArgs()
    a.H, a.W, a.depth, a.cam, a.n_nb = H, W, d_t.data_ptr(), L.host_ptr(row), n
    for j, m in enumerate(maps):
        a.nb_depth[j] = m.data_ptr()
        a.nb_h[j], a.nb_w[j] = int(m.shape[0]), int(m.shape[1])
    a.nb_cam, a.rel_tol, a.px_tol = L.host_ptr(rows), L.host_ptr(tol), float(px_tol)
    a.count = count.data_ptr()
    active = None
    if grey is not None:
        g_t, s_t = _dev32(grey, dev), _dev32(score, dev)
        if tuple(g_t.shape) != (H, W) or tuple(s_t.shape) != (H, W):
            raise ValueError("consistency: grey / score shape differs from the depth map")
        active = torch.empty((H, W), dtype=torch.uint8, device=dev)
        a.grey, a.score, a.active = g_t.data_ptr(), s_t.data_ptr(), active.data_ptr()
        a.min_ncc, a.min_views = float(min_ncc), int(min_views)
    L.check(L.load().mvs_consistency(dense.C_addr(a), L.stream_handle()), "consistency")
    return count, active


def _consistency(k, D, nbrs_k, dm, cams, px_tol, rel_tol) -> np.ndarray:
    """Drop-in for densify._consistency (densify.py:441-478): int16 NumPy counts."""
    js = [j for j in nbrs_k if j in dm]
    cnt, _ = consistency(D, cams[k], [dm[j] for j in js], [cams[j] for j in js], px_tol, [rel_tol[j] for j in js])
    torch.cuda.current_stream().synchronize()
    return cnt.cpu().numpy()


init_normals = fast.init_normals


# ------------------------------------------------------------------ host geometry (NumPy, as the reference)
def neighbours(rec, n_nb: int) -> List[List[int]]:
    """Source views per image (densify._neighbours, densify.py:183-205): views sharing at least 15
    tie points, ranked by shared points weighted by triangulation angle (full weight from 8 deg,
    a fifth above 45 deg)."""
    N = len(rec.used)
    shared = np.zeros((N, N), np.int32)
    order = np.argsort(rec.obs_pt, kind="stable")
    pts, cams = rec.obs_pt[order], rec.obs_cam[order]
    for grp in np.split(cams, np.flatnonzero(np.diff(pts)) + 1):
        if len(grp) > 1:
            g = np.unique(grp)
            shared[np.ix_(g, g)] += 1
    np.fill_diagonal(shared, 0)
    depth = np.array([_median_depth(rec, k) if np.any(rec.obs_cam == k) else 1.0 for k in range(N)])
    out = []
    for k in range(N):
        ang = np.degrees(np.linalg.norm(rec.C - rec.C[k], axis=1) / max(depth[k], 1e-3))
        score = shared[k] * (np.clip(ang / 8.0, 0, 1) ** 2 * np.where(ang > 45, 0.2, 1.0))
        out.append([j for j in np.argsort(-score) if score[j] > 0 and shared[k, j] >= 15][:n_nb])
    return out


def _median_depth(rec, k) -> float:
    """Median camera-axis depth of the tie points image k observes."""
    return float(np.median((rec.R[k] @ (rec.X[rec.obs_pt[rec.obs_cam == k]] - rec.C[k]).T)[2]))


class PassSettings:
    """The data-driven pass-2 settings of the reference (densify.py:563-584): reprojection
    tolerance in pixels, minimum agreeing views, and per-neighbour relative depth tolerances."""

    def __init__(self, rec, cams: Dict[int, object], nbrs: List[List[int]], opt: DepthOptions,
                 scales: Optional[Dict[int, float]] = None):
        N = len(nbrs)
        scale_med = float(np.median(list(scales.values()))) if scales else 1.0
        self.px_tol = opt.consistency_px or float(np.clip(2.0 * rec.rms_px * scale_med, 1.0, 3.0))
        n_good = np.array([len(x) for x in nbrs])
        self.min_views = opt.min_views or (3 if np.median(n_good) >= 3 else 2)
        self.dmed = {k: _median_depth(rec, k) for k in range(N) if np.any(rec.obs_cam == k)}
        self._cams, self._nbrs, self._rec, self._opt = cams, nbrs, rec, opt

    def rel_tols(self, k) -> Dict[int, float]:
        """Depth change that moves a point by px_tol pixels between views k and j, relative."""
        out = {}
        ck = self._cams[k]
        for j in self._nbrs[k]:
            B = float(np.linalg.norm(self._rec.C[k] - self._rec.C[j]))
            out[j] = (self._opt.consistency_depth or
                      float(np.clip(self.px_tol * self.dmed.get(k, 1.0) / max(ck.f * B, 1e-9), 0.01, 0.05)))
        return out


# ------------------------------------------------------------------ pass 2 on the device
def repair(k: int, raw: Dict[int, torch.Tensor], score: torch.Tensor, low: torch.Tensor, views, nbrs_k: Sequence[int],
           rec, settings: PassSettings, opt: DepthOptions):
    """Pass 2 for view k (densify.py:611-640): consistency count, PatchMatch repair of the pixels
    it selects (the neighbours' pass-1 maps in its geometric term), final filter. ``raw`` holds
    the pass-1 maps of k and of every neighbour that has one (device tensors); ``score`` is k's
    pass-1 score (float16-rounded) and is updated in place. Returns (depth, changed, n_active)."""
    D = raw[k].clone()
    S = score
    changed, n_active = 0, 0
    tol = settings.rel_tols(k)
    if opt.patchmatch:
        grey, _, cr = views(k)
        dev = D.device
        g_t = _dev32(grey, dev)
        js = [j for j in nbrs_k if j in raw]
        _, active = consistency(D, cr, [raw[j] for j in js], [views(j)[2] for j in js], settings.px_tol,
                                [tol[j] for j in js], grey=g_t, score=S, min_ncc=opt.min_ncc,
                                min_views=settings.min_views)
        n_active = int(active.sum().item())
        if n_active and js:
            ray = fast.rays_world(tuple(D.shape), cr)
            normal = init_normals(D, ray)
            srcs = [_dev32(views(j)[0], dev) for j in js]
            par = np.array([cam_row(views(j)[2]) for j in js], np.float64)
            rng = _depth_range(rec, k)
            if rng is None:
                rng = (float(torch.nan_to_num(D, nan=float("inf")).min()),
                       float(torch.nan_to_num(D, nan=float("-inf")).max()))
            ref = torch.where(torch.isfinite(g_t), g_t, torch.full_like(g_t, float("nan")))
            changed = dense.pm_refine(ref, ray, np.asarray(cr.C, np.float64), srcs, [raw[j] for j in js], par, D,
                                      normal, S, active, opt.pm_window, opt.pm_step, opt.top_k, opt.pm_geo_weight,
                                      float(np.median(list(tol.values()))), opt.pm_iters, rng[0], rng[1],
                                      k * 2654435761 % 2**32, precision=getattr(opt, "pm_precision", "fp64"))
    D = torch.where((S < opt.min_ncc) | low, torch.full_like(D, float("nan")), D)
    return D, changed, n_active


# ------------------------------------------------------------------ pass 3: point fusion
def fuse(order: Sequence[int], maps: Dict[int, object], cams, nbrs, rel_tols, px_tol: float, min_views: int,
         point_stride: int, rgbs):
    """Point fusion of the final depth maps (densify._fuse, densify.py:676-762) on the device:
    views in `order` (the reference fuses sorted(have)), one ``mvs_fuse_view`` launch each, the
    used masks carried from view to view on the device. maps[k]: (H, W) depth (NaN = none);
    nbrs[k]: neighbour ids; rel_tols[k][j]: relative depth tolerance; rgbs[k]: (H, W, 3) uint8.
    Returns (xyz float64 (n, 3), colours uint8 (n, 3), views uint8 (n,), owner int32 (n,)) as
    torch CUDA tensors in the reference's order (views in order, pixels row-major), and the
    used masks {k: bool tensor}."""
    dev = L.require_cuda()
    lib = L.load()
    D = {k: _dev32(m, dev) for k, m in maps.items()}
    used = {k: torch.zeros(tuple(D[k].shape), dtype=torch.uint8, device=dev) for k in D}
    pts, cols, nv, owner = [], [], [], []
    sh = L.stream_handle()
    for k in order:
        if k not in D:
            continue
        H, W = (int(v) for v in D[k].shape)
        nb = [j for j in nbrs[k] if j in D and j != k]
        if len(nb) > L.MAX_SOURCES:
            raise ValueError(f"fuse: view {k} has {len(nb)} neighbours (at most {L.MAX_SOURCES})")
        cam = L.host_f64(cam_row(cams[k]))
        nb_cam = L.host_f64(np.array([cam_row(cams[j]) for j in nb], np.float64).reshape(-1) if nb else np.zeros(1))
        tol = L.host_f64(np.array([rel_tols[k][j] for j in nb], np.float64) if nb else np.zeros(1))
        keep = torch.empty((H, W), dtype=torch.uint8, device=dev)
        xyz = torch.empty((3, H, W), dtype=torch.float64, device=dev)
        cnt = torch.empty((H, W), dtype=torch.int32, device=dev)
        a = L.FuseArgs()
        a.H, a.W, a.depth, a.used, a.cam = H, W, D[k].data_ptr(), used[k].data_ptr(), L.host_ptr(cam)
        a.n_nb, a.point_stride = len(nb), int(point_stride)
        for i, j in enumerate(nb):
            a.nb_depth[i], a.nb_used[i] = D[j].data_ptr(), used[j].data_ptr()
            a.nb_h[i], a.nb_w[i] = int(D[j].shape[0]), int(D[j].shape[1])
        a.nb_cam, a.rel_tol, a.px_tol, a.min_views = L.host_ptr(nb_cam), L.host_ptr(tol), float(px_tol), int(min_views)
        a.keep, a.xyz, a.count = keep.data_ptr(), xyz.data_ptr(), cnt.data_ptr()
        L.check(lib.mvs_fuse_view(ctypes.addressof(a), sh), "fuse")
        sel = torch.nonzero(keep.view(-1)).squeeze(1)          # row-major, as np.nonzero
        if sel.numel() == 0:
            continue
        pts.append(xyz.view(3, -1)[:, sel].T)
        rgb = torch.as_tensor(np.ascontiguousarray(rgbs[k]), device=dev) if not isinstance(rgbs[k], torch.Tensor) \
            else rgbs[k].to(dev)
        cols.append(rgb.reshape(-1, 3)[sel])
        nv.append(cnt.view(-1)[sel].clamp(max=255).to(torch.uint8))
        owner.append(torch.full((sel.numel(),), k, dtype=torch.int32, device=dev))

    def cat(a, shape, dt):
        return torch.cat(a) if a else torch.zeros(shape, dtype=dt, device=dev)
    return (cat(pts, (0, 3), torch.float64), cat(cols, (0, 3), torch.uint8), cat(nv, (0,), torch.uint8),
            cat(owner, (0,), torch.int32), {k: u.bool() for k, u in used.items()})


# ------------------------------------------------------------------ sharding and the exchange
def assign_views(costs: Sequence[float], world: int) -> List[int]:
    """Owner rank of every view: longest-processing-time first onto the least-loaded rank (ties to
    the lower view index and the lower rank). Deterministic, so every rank derives the same map."""
    owner = [0] * len(costs)
    load = [0.0] * max(world, 1)
    for k in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        r = min(range(len(load)), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += float(costs[k])
    return owner


def wanted_maps(owner: Sequence[int], nbrs: Sequence[Sequence[int]], have: Sequence[int]) -> List[int]:
    """Views whose pass-1 map a view on another rank uses, in view order."""
    return sorted(map_destinations(owner, nbrs, have))


def map_destinations(owner: Sequence[int], nbrs: Sequence[Sequence[int]], have: Sequence[int]) -> Dict[int, List[int]]:
    """For every pass-1 map that views on other ranks read: the ranks that read it (sorted)."""
    hv = set(have)
    out: Dict[int, set] = {}
    for k, nb in enumerate(nbrs):
        if k not in hv:
            continue
        for j in nb:
            if j in hv and owner[j] != owner[k]:
                out.setdefault(j, set()).add(owner[k])
    return {j: sorted(r) for j, r in out.items()}


def exchange_maps(local: Dict[int, torch.Tensor], owner: Sequence[int], shapes: Dict[int, tuple],
                  dests: Dict[int, List[int]], rank: int, group=None, device=None) -> Dict[int, torch.Tensor]:
    """Point to point: each map goes from its owner to the ranks whose views read it, and to no
    other rank. Every rank walks the maps in view order, so the sends and receives between any two
    ranks pair up in the same order. Returns ``local`` plus the maps received."""
    import torch.distributed as dist
    out = dict(local)
    reqs = []
    for j in sorted(dests):
        if owner[j] == rank:
            buf = local[j].contiguous()
            for dst in dests[j]:
                reqs.append(dist.isend(buf, dst=_global_rank(dst, group), group=group))
        elif rank in dests[j]:
            buf = torch.empty(shapes[j], dtype=torch.float32, device=device)
            reqs.append(dist.irecv(buf, src=_global_rank(owner[j], group), group=group))
            out[j] = buf
    for q in reqs:
        q.wait()
    return out


def _global_rank(r: int, group) -> int:
    import torch.distributed as dist
    return r if group is None else dist.get_global_rank(group, r)


def run_passes(n_views: int, nbrs: Sequence[Sequence[int]], costs: Sequence[float], shapes: Dict[int, tuple],
               pass1: Callable[[int], Optional[torch.Tensor]], pass2: Callable[[int, Dict[int, torch.Tensor]], object],
               group=None, device=None) -> Dict[int, object]:
    """Pass 1 on this rank's views, the exchange, pass 2 on this rank's views. ``pass1(k)``
    returns view k's map or None (no depth map); ``pass2(k, maps)`` gets every map it may read
    (its own and its neighbours'). Which views have a map is agreed by an all-gather of flags
    before the exchange. Returns {k: pass2 result} for this rank's views that have a map."""
    import torch.distributed as dist
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    owner = assign_views(costs, world)
    mine = [k for k in range(n_views) if owner[k] == rank]
    local = {}
    for k in mine:
        m = pass1(k)
        if m is not None:
            local[k] = m
    flags = torch.zeros(n_views, dtype=torch.int32, device=device)
    for k in local:
        flags[k] = 1
    if world > 1:
        dist.all_reduce(flags, op=dist.ReduceOp.SUM, group=group)
    have = [k for k, f in enumerate(flags.tolist()) if f]
    maps = local
    if world > 1:
        maps = exchange_maps(local, owner, shapes, map_destinations(owner, nbrs, have), rank, group, device)
    return {k: pass2(k, maps) for k in mine if k in local}


def densify_views(rec, views, opt: DepthOptions, nbrs: Optional[List[List[int]]] = None,
                  scales: Optional[Dict[int, float]] = None, group=None):
    """Passes 1 and 2 for every view of a reconstruction (densify.py:513-640 without the fusion):
    returns {k: (final depth float32 NumPy with NaN, PatchMatch changes, PatchMatch pixels)} for
    this rank's views. ``views(k)`` returns (grey float32 with NaN = masked, rgb, camera at
    matching scale), as the reference's image cache does."""
    N = len(rec.used)
    nbrs = neighbours(rec, opt.neighbors) if nbrs is None else nbrs
    cams = {k: views(k)[2] for k in range(N)}
    settings = PassSettings(rec, cams, nbrs, opt, scales)
    shapes = {k: (int(cams[k].h), int(cams[k].w)) for k in range(N)}
    costs = [shapes[k][0] * shapes[k][1] * max(len(nbrs[k]), 1) for k in range(N)]
    dev = L.require_cuda()
    extra: Dict[int, tuple] = {}

    def pass1(k):
        with L.nvtx(f"pass 1 view {k}"):
            r = depth_map_device(k, nbrs[k], rec, views, opt)
        if r is None:
            return None
        depth, score, low = r
        extra[k] = (score.half().float(), low)      # pass 2 reads the score through float16
        return depth

    def pass2(k, maps):
        score, low = extra[k]
        with L.nvtx(f"pass 2 view {k}"):
            D, ch, na = repair(k, maps, score, low, views, nbrs[k], rec, settings, opt)
        torch.cuda.current_stream().synchronize()
        L.check_device_faults()      # a sweep tile of pass 1 or 2 that gave up raises here
        return D.cpu().numpy(), ch, na

    return run_passes(N, nbrs, costs, shapes, pass1, pass2, group=group, device=dev)

"""Seeded synthetic scenes for the depth-map workloads (the reference's flights are not
available, so these stand in for them, with the shapes and value distributions of the
benchmark configurations):

* terrain z(x, y): Gaussian hills (sigma 5-20 m, amplitude 0-6 m) plus axis-aligned flat-roofed box
  buildings (3-12 m above the terrain at their centre);
* texture: 4-octave value noise (periods 3, 6, 12, 24 ground pixels) of (x + 0.37 z, y - 0.61 z),
  quantised to uint8 grey (walls get texture that varies with height);
* nadir pinhole cameras (R = diag(1, -1, -1) with a seeded 0.3 deg attitude error, image x = east,
  y = south, principal point at the image centre, pixel centres at integers), rendered by ray
  casting the heightfield: a 0.25 m march along camera-axis depth, then 24 bisection steps.

Rendering uses torch and runs on any device (CPU for the small test scenes, the GPU for the
full-size ones); it is set-up work, outside every timed region.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class Camera:
    """Pinhole + radial k1..k3 camera with the reference's attributes (densify._Cam)."""
    R: np.ndarray
    C: np.ndarray
    f: float
    cx: float
    cy: float
    w: int
    h: int
    k1: float = 0.0
    k2: float = 0.0
    k3: float = 0.0

    def row(self) -> np.ndarray:
        """R(9) C(3) f k1 k2 k3 cx cy."""
        return np.r_[np.asarray(self.R, np.float64).ravel(), np.asarray(self.C, np.float64),
                     [self.f, self.k1, self.k2, self.k3, self.cx, self.cy]]


NADIR = np.diag([1.0, -1.0, -1.0])


def attitude(rng, sigma_deg: float) -> np.ndarray:
    """World -> camera rotation of a nadir camera with a small seeded attitude error (Rodrigues
    rotation of normal(0, sigma) radians per axis applied after the nadir rotation). Real
    flights never have exactly parallel optical axes; without it the along-track sources would
    map image edges exactly onto source image edges, a measure-zero tie of the sample-validity
    test that rounding decides arbitrarily."""
    w = rng.normal(0.0, np.radians(sigma_deg), 3)
    th = float(np.linalg.norm(w))
    if th == 0.0:
        return NADIR.copy()
    k = w / th
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return (np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K) @ NADIR


@dataclass
class SceneConfig:
    name: str
    width: int
    height: int
    focal: float
    altitude: float
    hills: int
    boxes: int
    sources: int                 # 4: +-along, +-across; 8: adds the four diagonals
    forward_overlap: float       # along x (the long side)
    side_overlap: float          # along y
    planes: int
    depth_range: tuple           # (near, far) metres, uniform in inverse depth
    radius: int
    top_k: int = 2
    pm_iters: int = 0
    pm_radius: int = 3
    pm_step: int = 1


CONFIGS = {
    # plain plane sweep, CPU-runnable size
    "c1": SceneConfig("c1-640x480-4src-128planes-5x5", 640, 480, 600.0, 50.0, 8, 6, 4, 0.8, 0.7, 128,
                      (35.0, 55.0), 2),
    # full-resolution sweep + PatchMatch
    "c2": SceneConfig("c2-4000x3000-8src-256planes-7x7-pm4", 4000, 3000, 3600.0, 80.0, 20, 20, 8, 0.8, 0.7, 256,
                      (60.0, 90.0), 3, pm_iters=4, pm_radius=3, pm_step=1),
}


@dataclass
class Terrain:
    hills: np.ndarray            # (n, 4): x0, y0, sigma, amplitude
    boxes: np.ndarray            # (m, 5): x0, x1, y0, y1, top
    tex_seed: int
    gsd: float

    def zmax(self) -> float:
        top = float(self.boxes[:, 4].max()) if len(self.boxes) else 0.0
        return max(top, float(self.hills[:, 3].sum()) if len(self.hills) else 0.0)


@dataclass
class Scene:
    config: SceneConfig
    ref: np.ndarray              # (H, W) uint8
    srcs: list                   # [(h, w) uint8]
    ref_cam: Camera
    src_cams: list
    planes_inv: np.ndarray       # (n,) float32 inverse depths, far -> near
    depth_true: np.ndarray       # (H, W) float32 camera-axis depth of the reference
    terrain: Terrain = field(repr=False, default=None)

    def grey(self, img: np.ndarray) -> np.ndarray:
        """densify's normalised grey (mean(rgb) - 128) / 64 for a grey uint8 image (exact)."""
        return ((img.astype(np.float32) - np.float32(128.0)) / np.float32(64.0)).astype(np.float32)


def _hills_z(x: torch.Tensor, y: torch.Tensor, hills: torch.Tensor) -> torch.Tensor:
    z = torch.zeros_like(x)
    for k in range(hills.shape[0]):
        x0, y0, s, a = hills[k]
        z = z + a * torch.exp(-((x - x0) ** 2 + (y - y0) ** 2) / (2 * s * s))
    return z


def _height(x: torch.Tensor, y: torch.Tensor, hills: torch.Tensor, boxes: torch.Tensor) -> torch.Tensor:
    z = _hills_z(x, y, hills)
    for k in range(boxes.shape[0]):
        x0, x1, y0, y1, top = boxes[k]
        inside = (x >= x0) & (x <= x1) & (y >= y0) & (y <= y1)
        z = torch.where(inside, torch.maximum(z, top.expand_as(z)), z)
    return z


def _lattice(ix: torch.Tensor, iy: torch.Tensor, seed: int) -> torch.Tensor:
    """Hash of integer lattice points -> uniform [0, 1) (64-bit integer mixing)."""
    h = (ix * 374761393 + iy * 668265263 + seed * 2147483647) & 0xFFFFFFFF
    h = ((h ^ (h >> 13)) * 1274126177) & 0xFFFFFFFF
    h = h ^ (h >> 16)
    return (h & 0xFFFFFF).to(torch.float64) / 16777216.0


def _value_noise(x: torch.Tensor, y: torch.Tensor, period: float, seed: int) -> torch.Tensor:
    fx, fy = x / period, y / period
    x0, y0 = torch.floor(fx), torch.floor(fy)
    tx, ty = fx - x0, fy - y0
    sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
    ix, iy = x0.to(torch.int64), y0.to(torch.int64)
    v00 = _lattice(ix, iy, seed)
    v10 = _lattice(ix + 1, iy, seed)
    v01 = _lattice(ix, iy + 1, seed)
    v11 = _lattice(ix + 1, iy + 1, seed)
    a = v00 + (v10 - v00) * sx
    b = v01 + (v11 - v01) * sx
    return a + (b - a) * sy


def _texture(x: torch.Tensor, y: torch.Tensor, z: torch.Tensor, terr: Terrain) -> torch.Tensor:
    u, v = x + 0.37 * z, y - 0.61 * z
    acc = torch.zeros_like(x)
    amp, norm = 1.0, 0.0
    for o in range(4):
        period = terr.gsd * 3.0 * (2 ** (3 - o))
        acc = acc + amp * (_value_noise(u, v, period, terr.tex_seed + 7919 * o) - 0.5)
        norm += amp
        amp *= 0.6
    return acc / norm


def render(cam: Camera, terr: Terrain, device="cpu", rows_per_chunk: int = 0):
    """Ray-casts the heightfield into `cam`. Returns (uint8 image, float32 camera-axis depth)."""
    dev = torch.device(device)
    hills = torch.as_tensor(terr.hills, dtype=torch.float64, device=dev)
    boxes = torch.as_tensor(terr.boxes, dtype=torch.float64, device=dev)
    Rt = torch.as_tensor(np.asarray(cam.R, np.float64).T, device=dev)
    C = torch.as_tensor(np.asarray(cam.C, np.float64), device=dev)
    zmin, zmax = -0.5, terr.zmax() + 0.5
    img = np.empty((cam.h, cam.w), np.uint8)
    dep = np.empty((cam.h, cam.w), np.float32)
    uu = torch.arange(cam.w, dtype=torch.float64, device=dev)
    if rows_per_chunk <= 0:
        rows_per_chunk = cam.h if dev.type == "cuda" else 256
    for r0 in range(0, cam.h, rows_per_chunk):
        r1 = min(cam.h, r0 + rows_per_chunk)
        vv = torch.arange(r0, r1, dtype=torch.float64, device=dev)
        V, U = torch.meshgrid(vv, uu, indexing="ij")
        rc = torch.stack([(U - cam.cx) / cam.f, (V - cam.cy) / cam.f, torch.ones_like(U)])
        d = torch.einsum("ij,jhw->ihw", Rt, rc)            # world direction, camera-axis depth 1
        dz = d[2]
        # march along camera-axis depth t: the ray is C + t d
        t_lo = (C[2] - zmax) / (-dz)
        t_hi = (C[2] - zmin) / (-dz)
        step = 0.25
        nsteps = int(math.ceil(float((t_hi - t_lo).max()) / step)) + 1
        hit_lo = t_lo.clone()
        hit_hi = torch.full_like(t_lo, float("nan"))
        found = torch.zeros_like(t_lo, dtype=torch.bool)
        prev_t = t_lo.clone()
        for k in range(1, nsteps + 1):
            t = torch.minimum(t_lo + k * step, t_hi)
            P = C[:, None, None] + t[None] * d
            below = P[2] <= _height(P[0], P[1], hills, boxes)
            new = below & ~found
            hit_lo = torch.where(new, prev_t, hit_lo)
            hit_hi = torch.where(new, t, hit_hi)
            found = found | below
            prev_t = t
            if bool(found.all()):
                break
        hit_hi = torch.where(found, hit_hi, t_hi)
        lo, hi = hit_lo, hit_hi
        for _ in range(24):
            mid = 0.5 * (lo + hi)
            P = C[:, None, None] + mid[None] * d
            below = P[2] <= _height(P[0], P[1], hills, boxes)
            hi = torch.where(below, mid, hi)
            lo = torch.where(below, lo, mid)
        P = C[:, None, None] + hi[None] * d
        zs = _height(P[0], P[1], hills, boxes)
        g = _texture(P[0], P[1], zs, terr)
        grey = torch.clamp(torch.round(128.0 + 300.0 * g), 0, 255).to(torch.uint8)
        img[r0:r1] = grey.cpu().numpy()
        dep[r0:r1] = hi.to(torch.float32).cpu().numpy()
    return img, dep


def _terrain(cfg: SceneConfig, seed: int, half_x: float, half_y: float) -> Terrain:
    rng = np.random.default_rng(seed)
    hills = np.column_stack([rng.uniform(-half_x, half_x, cfg.hills), rng.uniform(-half_y, half_y, cfg.hills),
                             rng.uniform(5.0, 20.0, cfg.hills), rng.uniform(0.0, 6.0, cfg.hills)])
    boxes = []
    for _ in range(cfg.boxes):
        cx, cy = rng.uniform(-half_x, half_x), rng.uniform(-half_y, half_y)
        sx, sy = rng.uniform(3.0, 10.0), rng.uniform(3.0, 10.0)
        base = float(sum(a * math.exp(-((cx - x0) ** 2 + (cy - y0) ** 2) / (2 * s * s)) for x0, y0, s, a in hills))
        boxes.append([cx - sx / 2, cx + sx / 2, cy - sy / 2, cy + sy / 2, base + rng.uniform(3.0, 12.0)])
    gsd = cfg.altitude / cfg.focal
    return Terrain(hills, np.array(boxes, np.float64).reshape(-1, 5), int(rng.integers(1, 2**31 - 1)), gsd)


def source_offsets(cfg: SceneConfig):
    fx = cfg.width * cfg.altitude / cfg.focal
    fy = cfg.height * cfg.altitude / cfg.focal
    bx, by = (1 - cfg.forward_overlap) * fx, (1 - cfg.side_overlap) * fy
    offs = [(bx, 0.0), (-bx, 0.0), (0.0, by), (0.0, -by)]
    if cfg.sources >= 8:
        offs += [(bx, by), (-bx, by), (bx, -by), (-bx, -by)]
    return offs[:cfg.sources]


def plane_list(near: float, far: float, n: int) -> np.ndarray:
    """n inverse depths uniform over [1/far, 1/near], far -> near (float32)."""
    lo, hi = 1.0 / far, 1.0 / near
    return np.array([lo + i * (hi - lo) / max(n - 1, 1) for i in range(n)], np.float32)


def make_scene(cfg: SceneConfig | str, seed: int = 0, device="cpu", width: int | None = None,
               height: int | None = None) -> Scene:
    """Seeded scene for a configuration (optionally at another image size, same geometry)."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    W = width or cfg.width
    H = height or cfg.height
    f = cfg.focal * W / cfg.width
    half_x = 0.5 * W * cfg.altitude / f + 25.0
    half_y = 0.5 * H * cfg.altitude / f + 25.0
    terr = _terrain(cfg, seed, half_x, half_y)
    terr.gsd = cfg.altitude / f

    att = np.random.default_rng(seed + 7777)

    def cam_at(x, y):
        return Camera(attitude(att, 0.3), np.array([x, y, cfg.altitude]), f, (W - 1) / 2.0, (H - 1) / 2.0, W, H)

    ref_cam = cam_at(0.0, 0.0)
    src_cams = [cam_at(x, y) for x, y in source_offsets(cfg)]
    ref, dtrue = render(ref_cam, terr, device)
    srcs = [render(c, terr, device)[0] for c in src_cams]
    planes = plane_list(cfg.depth_range[0], cfg.depth_range[1], cfg.planes)
    return Scene(cfg, ref, srcs, ref_cam, src_cams, planes, dtrue, terr)


def geo_rows(ref_cam: Camera, src_cams) -> np.ndarray:
    """densify.py:329-338 geo rows: Rs(9) b(3) f k1 k2 k3 cx cy with b = Rs (C_ref - C_src)."""
    rows = []
    for cs in src_cams:
        Rs = np.asarray(cs.R, np.float64)
        b = Rs @ (np.asarray(ref_cam.C, np.float64) - np.asarray(cs.C, np.float64))
        rows.append(np.r_[Rs.ravel(), b, [cs.f, cs.k1, cs.k2, cs.k3, cs.cx, cs.cy]])
    return np.array(rows, np.float64)


def tilted_normals(H: int, W: int, seed: int, max_deg: float = 30.0) -> np.ndarray:
    """(3, H, W) float32 unit normals within `max_deg` of vertical, facing up (+z world) - the
    seeded initial PatchMatch normals of the full-resolution configuration."""
    rng = np.random.default_rng(seed)
    th = np.radians(max_deg) * np.sqrt(rng.random((H, W)))
    ph = rng.uniform(0, 2 * np.pi, (H, W))
    n = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    return np.ascontiguousarray(n, np.float32)

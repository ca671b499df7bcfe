"""Generates the golden fixtures in tests/golden/ by running the REFERENCE implementation
(pyOrthomosaic 0.9.3: its own densify.py with its own _dense / _fast kernels compiled from
source into oracle/_ref) on seeded inputs.

Run where the reference tree exists:  make -C oracle ref && python tests/golden/make_golden.py
(optionally followed by the names of the cases to regenerate, e.g. ``pm_case8``).
The fixtures travel with the repository; nothing at test time needs the reference.

Fixtures (each .npz holds the inputs and the reference outputs):
  sweep_cases.npz  - _dense.sweep_hypothesis over several hypotheses for shapes of the
                     reference's own parity tests (H, W, n, r, top_k, n_hyp), with 2 % NaN source
                     pixels, +-3 px source size jitter, inv = inf and inv < 0 injected; final
                     winner state and every hypothesis' top-k score (the `prev` array after each
                     call, _sweep.h:212); plus one flat-image tie case
  sweep_e2e.npz    - densify._sweep end to end (lazy hypotheses, parabola) -> depth, best, sd
  scene_small.npz  - a seeded synthetic nadir scene (uint8 images, pinhole cameras, constant
                     inverse-depth planes) through densify._sweep -> depth, best, sd and the
                     best-to-second hypothesis score gap
  helpers.npz      - _fast.box_zero_mean, hyp_linear, hyp_refine, depth_view, densify._rays_world
  pm_case.npz      - _dense.pm_refine (the reference's xorshift draws) on a small case
  pm_case8.npz     - _dense.pm_refine on a rendered 192 x 144 scene with 8 sources, 7 x 7 window,
                     2 iterations (uint8 images; the grey inputs are (g - 128) / 64)
  depth_map.npz    - densify.depth_map end to end (3-level pyramid, tie-point depth band, coarse
                     sweep + 2 refinement levels) on a rendered scene with a synthetic
                     reconstruction (tie points on the terrain, their in-image observations)
  views_case.npz   - densify._densify passes 1 and 2 end to end on a rendered 5-view scene
                     (depth maps, geometric consistency, PatchMatch repair with the neighbours'
                     depth maps, final filter), recording what the reference's own
                     _consistency, _init_normals and _dense.pm_refine received and returned
  fuse_case.npz    - densify._fuse (point fusion) on views_case's pass-2 maps, in two settings
  height_case.npz  - the legacy height sweep (mvs.py): _mvs.sample_view, _fast.box_sat_mean and
                     _mvs.sgm kernel cases, and mvs.dense_reconstruct (CPU backend) end to end
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refpkg  # noqa: E402
from oracle import oracle as O  # noqa: E402

SHAPES = [(37, 53, 4, 5, 2, 9), (64, 48, 1, 3, 2, 5), (11, 9, 3, 5, 2, 4), (5, 4, 2, 5, 1, 3),
          (30, 31, 5, 2, 3, 6), (2, 40, 2, 1, 2, 3), (40, 3, 4, 4, 4, 3), (48, 64, 8, 3, 2, 7),
          (33, 47, 16, 2, 9, 4)]


def rotation(rng, tilt):
    """Rotation near a nadir view (180 deg about x) with a random tilt (Rodrigues)."""
    w = rng.normal(0, tilt, 3) + np.array([np.pi, 0, 0])
    th = np.linalg.norm(w)
    k = w / th
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K


def random_case(rng, H, W, n, r, nhyp, nan_frac=0.02):
    ref = rng.normal(0, 1, (H, W)).astype(np.float32)
    srcs = []
    for _ in range(n):
        h = max(H + int(rng.integers(-3, 4)), 2)
        w = max(W + int(rng.integers(-3, 4)), 2)
        s = rng.normal(0, 1, (h, w)).astype(np.float32)
        s[rng.random(s.shape) < nan_frac] = np.nan
        srcs.append(np.ascontiguousarray(s))
    ray = rng.normal(0, 0.3, (3, H, W)).astype(np.float32)
    ray[2] = 1.0 + rng.normal(0, 0.01, (H, W)).astype(np.float32)
    geo = []
    for _ in range(n):
        Rs = rotation(rng, 0.05) @ rotation(rng, 0.0).T
        b = rng.normal(0, 0.5, 3)
        f = float(rng.uniform(0.8, 1.2) * W)
        geo.append(np.r_[Rs.ravel(), b, [f, rng.normal(0, 0.05), rng.normal(0, 0.01), rng.normal(0, 0.003),
                                         (W - 1) / 2 + rng.normal(0, 2), (H - 1) / 2 + rng.normal(0, 2)]])
    base = rng.uniform(0.02, 0.2, (H, W)).astype(np.float32)
    step = rng.uniform(1e-4, 5e-3, (H, W)).astype(np.float32)
    hyps = np.stack([(base + i * step).astype(np.float32) for i in range(nhyp)])
    if nhyp > 2:
        hyps[1, 0, 0] = np.inf
        hyps[2, -1, -1] = -0.01
    return ref, srcs, ray, np.array(geo, np.float64), hyps


def run_reference_sweep(R, ref, srcs, ray, geo, hyps, r, top_k):
    H, W = ref.shape
    mu = R._fast.box_zero_mean(ref, r)
    sd = np.sqrt(np.maximum(R._fast.box_zero_mean(np.ascontiguousarray(ref * ref), r) - mu * mu, 1e-6)).astype(
        np.float32)
    best, prev, spb, snb, idx = O.init_state(H, W)
    scores = np.empty((len(hyps), H, W), np.float32)
    for i, inv in enumerate(hyps):
        R._dense.sweep_hypothesis(ref, mu, sd, srcs, ray, geo, np.ascontiguousarray(inv), r, top_k, i, best, prev,
                                  spb, snb, idx)
        scores[i] = prev
    return mu, sd, best, prev, spb, snb, idx, scores


def sweep_cases(R):
    rng = np.random.default_rng(7)
    out = {}
    for k, (H, W, n, r, top_k, nh) in enumerate(SHAPES):
        ref, srcs, ray, geo, hyps = random_case(rng, H, W, n, r, nh)
        mu, sd, best, prev, spb, snb, idx, scores = run_reference_sweep(R, ref, srcs, ray, geo, hyps, r, top_k)
        p = f"c{k}_"
        out.update({p + "meta": np.array([H, W, n, r, top_k, nh]), p + "ref": ref, p + "ray": ray, p + "geo": geo,
                    p + "hyps": hyps, p + "mu": mu, p + "sd": sd, p + "best": best, p + "prev": prev,
                    p + "spb": spb, p + "snb": snb, p + "idx": idx, p + "scores": scores})
        for j, s in enumerate(srcs):
            out[p + f"src{j}"] = s
    # flat sources: equal scores everywhere, ties keep the first hypothesis
    ref, srcs, ray, geo, hyps = random_case(rng, 20, 24, 3, 2, 5, 0.0)
    flat = [np.ones_like(s) for s in srcs]
    mu, sd, best, prev, spb, snb, idx, scores = run_reference_sweep(R, ref, flat, ray, geo, hyps, 2, 2)
    k = len(SHAPES)
    p = f"c{k}_"
    out.update({p + "meta": np.array([20, 24, 3, 2, 2, 5]), p + "ref": ref, p + "ray": ray, p + "geo": geo,
                p + "hyps": hyps, p + "mu": mu, p + "sd": sd, p + "best": best, p + "prev": prev, p + "spb": spb,
                p + "snb": snb, p + "idx": idx, p + "scores": scores})
    for j, s in enumerate(flat):
        out[p + f"src{j}"] = s
    out["ncases"] = np.array(k + 1)
    np.savez_compressed(os.path.join(HERE, "sweep_cases.npz"), **out)


class _Cam:
    def __init__(self, R, C, f, k1, k2, k3, cx, cy, w=0, h=0):
        self.R, self.C = np.asarray(R, np.float64), np.asarray(C, np.float64)
        self.f, self.k1, self.k2, self.k3, self.cx, self.cy, self.w, self.h = f, k1, k2, k3, cx, cy, w, h


def sweep_e2e(D):
    rng = np.random.default_rng(3)
    H, W = 45, 61
    ref, srcs, ray, geo, hyps = random_case(rng, H, W, 4, 5, 19)
    cam_r = _Cam(np.eye(3), np.zeros(3), float(W), 0.0, 0.0, 0.0, W / 2, H / 2)
    cams_s = []
    for g in geo:
        Rs = g[:9].reshape(3, 3)
        Cs = -Rs.T @ g[9:12]                   # so that Rs (C_ref - C_src) == b
        cams_s.append(_Cam(Rs, Cs, g[12], g[13], g[14], g[15], g[16], g[17]))
    opt = D.DepthOptions()
    opt.window = 5
    lazy = D._Hypotheses(lambda i: hyps[i].copy(), len(hyps))
    depth, best, sd = D._sweep(ref, cam_r, srcs, cams_s, lazy, opt, ray)
    out = {"ref": ref, "ray": ray, "geo": geo, "hyps": hyps, "depth": depth, "best": best, "sd": sd,
           "meta": np.array([H, W, 4, 5, 2, 19])}
    for j, s in enumerate(srcs):
        out[f"src{j}"] = s
    np.savez_compressed(os.path.join(HERE, "sweep_e2e.npz"), **out)


def scene_small(D):
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=3, width=160, height=120)
    planes = S.plane_list(35.0, 55.0, 32)
    ref = sc.grey(sc.ref)
    srcs = [sc.grey(s) for s in sc.srcs]

    def cam(c):
        return _Cam(c.R, c.C, c.f, 0.0, 0.0, 0.0, c.cx, c.cy, c.w, c.h)

    cam_r = cam(sc.ref_cam)
    cams_s = [cam(c) for c in sc.src_cams]
    H, W = ref.shape
    opt = D.DepthOptions()
    opt.window = 2
    opt.top_k = 2
    ray = D._rays_world(ref.shape, cam_r)
    hyps = D._Hypotheses(lambda i: np.full((H, W), planes[i], np.float32), len(planes))
    depth, best, sd = D._sweep(ref, cam_r, srcs, cams_s, hyps, opt, ray)
    geo = O.geo_rows(cam_r, cams_s)
    R = O.reference()
    *_, scores = run_reference_sweep(R, ref, srcs, ray, geo, np.stack([hyps[i] for i in range(len(planes))]), 2, 2)
    srt = np.sort(scores, axis=0)
    gap = (srt[-1] - srt[-2]).astype(np.float32)          # best minus second-best hypothesis score
    out = {"ref_u8": sc.ref, "planes": planes, "ray": ray, "geo": geo, "depth": depth, "best": best, "sd": sd,
           "gap": gap, "ref_cam": np.r_[cam_r.R.ravel(), cam_r.C, [cam_r.f, 0, 0, 0, cam_r.cx, cam_r.cy]],
           "meta": np.array([H, W, len(srcs), 2, 2, len(planes)]), "depth_true": sc.depth_true}
    for j, s in enumerate(sc.srcs):
        out[f"src{j}_u8"] = s
    np.savez_compressed(os.path.join(HERE, "scene_small.npz"), **out)


def helpers(D, R):
    rng = np.random.default_rng(14)
    out = {}
    a = rng.normal(0, 1, (37, 53)).astype(np.float32)
    a[a > 1.5] = -0.0
    out["box_in"] = a
    for r in (0, 1, 2, 5, 7):
        out[f"box_r{r}"] = R._fast.box_zero_mean(a, r)
        out[f"box_sq_r{r}"] = R._fast.box_zero_mean(np.ascontiguousarray(a * a), r)
    base = rng.uniform(0.01, 0.05, (37, 53)).astype(np.float32)
    step = rng.uniform(1e-5, 1e-3, (37, 53)).astype(np.float32)
    out["hyp_base"], out["hyp_step"] = base, step
    for i in (0, 1, 7, 191):
        out[f"hyp_linear_{i}"] = R._fast.hyp_linear(base, step, i)
    iu = rng.uniform(-1e-3, 0.05, (37, 53)).astype(np.float32)
    iu[0, 0] = np.nan
    out["hyp_iu"] = iu
    for t in (-3, -1, 0, 2, 3):
        out[f"hyp_refine_{t + 3}"] = R._fast.hyp_refine(iu, step, t)
    rgb = rng.integers(0, 256, (29, 41, 3)).astype(np.uint8)
    m = rng.random((29, 41)) < 0.7
    out["dv_rgb"], out["dv_mask"] = rgb, m
    out["dv_gain"], out["dv_bias"] = np.array([1.07, 0.93, 1.21]), np.array([-3.5, 2.25, 0.0])
    g1, r1 = R._fast.depth_view(rgb, (1.07, 0.93, 1.21), (-3.5, 2.25, 0.0), m)
    g0, r0 = R._fast.depth_view(rgb, None, None, None)
    out["dv_grey"], out["dv_rgb8"], out["dv_grey0"], out["dv_rgb80"] = g1, r1, g0, r0
    cam = D._Cam(rotation(rng, 0.1), np.array([1.0, -2.0, 50.0]), 1000.0, -0.05, 0.01, 511.3, 383.7, 1024, 768,
                 0.003)
    out["rays_cam"] = np.r_[cam.R.ravel(), cam.C, [cam.f, cam.k1, cam.k2, cam.k3, cam.cx, cam.cy]]
    out["rays"] = D._rays_world((96, 128), cam)
    half_in = rng.normal(0, 1, (3, 31, 45)).astype(np.float32)
    out["half_in"] = half_in
    out["half_out"] = np.stack([D._half(x) for x in half_in])
    np.savez_compressed(os.path.join(HERE, "helpers.npz"), **out)


def pm_case(R):
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=5, width=40, height=32)
    ref = sc.grey(sc.ref)
    srcs = [sc.grey(s) for s in sc.srcs[:3]]
    H, W = ref.shape
    ray = O.rays_world((H, W), sc.ref_cam)
    par = np.array([c.row() for c in sc.src_cams[:3]], np.float64)
    rng = np.random.default_rng(9)
    depth = (sc.depth_true * (1 + rng.normal(0, 0.01, (H, W)))).astype(np.float32)
    depth[rng.random((H, W)) < 0.05] = np.nan
    normal = S.tilted_normals(H, W, 11)        # +z: facing the nadir camera (rays point down)
    score = np.zeros((H, W), np.float32)
    active = (rng.random((H, W)) < 0.8).astype(np.uint8)
    sdeps = [None, np.ascontiguousarray(sc.depth_true[:H, :W] * 1.001, np.float32), None]
    args = dict(r=2, step=1, top_k=2, geo_w=0.5, geo_tol=0.02, iters=2, dmin=35.0, dmax=55.0, seed=12345)
    out = {"ref": ref, "ray": ray, "par": par, "Cr": np.asarray(sc.ref_cam.C, np.float64), "depth0": depth.copy(),
           "normal0": normal.copy(), "score0": score.copy(), "active": active, "sdep1": sdeps[1],
           "args": np.array([args["r"], args["step"], args["top_k"], args["iters"], args["seed"]]),
           "fargs": np.array([args["geo_w"], args["geo_tol"], args["dmin"], args["dmax"]])}
    for j, s in enumerate(srcs):
        out[f"src{j}"] = s
    ch = R._dense.pm_refine(ref, ray, out["Cr"], srcs, sdeps, par, depth, normal, score, active, args["r"],
                            args["step"], args["top_k"], args["geo_w"], args["geo_tol"], args["iters"], args["dmin"],
                            args["dmax"], args["seed"])
    out.update({"depth": depth, "normal": normal, "score": score, "changed": np.array(ch)})
    np.savez_compressed(os.path.join(HERE, "pm_case.npz"), **out)


def pm_case8(R):
    from py_ortho_b200 import scene as S
    W, H = 192, 144
    sc = S.make_scene("c2", seed=21, width=W, height=H)
    ref_u8 = np.ascontiguousarray(sc.ref)
    src_u8 = np.stack([np.ascontiguousarray(s) for s in sc.srcs[:8]])
    ref = sc.grey(ref_u8)
    srcs = [sc.grey(s) for s in src_u8]
    ray = O.rays_world((H, W), sc.ref_cam)
    par = np.array([c.row() for c in sc.src_cams[:8]], np.float64)
    rng = np.random.default_rng(23)
    depth = (sc.depth_true * (1 + rng.normal(0, 0.01, (H, W)))).astype(np.float32)
    depth[rng.random((H, W)) < 0.01] = np.nan
    normal = S.tilted_normals(H, W, 29)
    score = np.zeros((H, W), np.float32)
    active = (rng.random((H, W)) < 0.8).astype(np.uint8)
    zr = float(sc.ref_cam.C[2])
    args = dict(r=3, step=1, top_k=2, geo_w=0.0, geo_tol=0.02, iters=2, dmin=zr - 40.0, dmax=zr + 5.0, seed=4242)
    out = {"ref_u8": ref_u8, "src_u8": src_u8, "ray": ray, "par": par, "Cr": np.asarray(sc.ref_cam.C, np.float64),
           "depth0": depth.copy(), "normal0": normal.copy(), "active": active,
           "args": np.array([args["r"], args["step"], args["top_k"], args["iters"], args["seed"]]),
           "fargs": np.array([args["geo_w"], args["geo_tol"], args["dmin"], args["dmax"]])}
    ch = R._dense.pm_refine(ref, ray, out["Cr"], srcs, [None] * 8, par, depth, normal, score, active, args["r"],
                            args["step"], args["top_k"], args["geo_w"], args["geo_tol"], args["iters"], args["dmin"],
                            args["dmax"], args["seed"])
    out.update({"depth": depth, "normal": normal, "score": score, "changed": np.array(ch)})
    print("pm_case8: changes", ch)
    np.savez_compressed(os.path.join(HERE, "pm_case8.npz"), **out)


def depth_map_case(D):
    """Reference densify.depth_map on a rendered 5-view scene with synthetic tie points."""
    import torch
    from types import SimpleNamespace
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=8, width=320, height=240)
    cams = [sc.ref_cam] + list(sc.src_cams)
    imgs = [sc.ref] + list(sc.srcs)
    rng = np.random.default_rng(17)
    # tie points: random terrain points inside the reference footprint
    n = 3000
    xs = rng.uniform(-12.0, 12.0, n)
    ys = rng.uniform(-9.0, 9.0, n)
    t = sc.terrain
    z = S._height(torch.from_numpy(xs), torch.from_numpy(ys), torch.from_numpy(t.hills), torch.from_numpy(t.boxes)).numpy()
    X = np.column_stack([xs, ys, z])
    obs_cam, obs_pt = [], []
    for k, c in enumerate(cams):
        xc = (X - c.C) @ c.R.T
        u = c.f * xc[:, 0] / xc[:, 2] + c.cx
        v = c.f * xc[:, 1] / xc[:, 2] + c.cy
        ok = (xc[:, 2] > 0) & (u >= 0) & (v >= 0) & (u < c.w) & (v < c.h)
        obs_cam.append(np.full(ok.sum(), k, np.int32))
        obs_pt.append(np.flatnonzero(ok).astype(np.int32))
    intr = [SimpleNamespace(f=cams[0].f, cx=cams[0].cx, cy=cams[0].cy, width=cams[0].w, height=cams[0].h,
                            k1=0.0, k2=0.0, k3=0.0)]
    rec = SimpleNamespace(intr=intr, cam_group=np.zeros(len(cams), np.int32), X=X,
                          C=np.array([c.C for c in cams]), R=np.array([c.R for c in cams]),
                          obs_cam=np.concatenate(obs_cam), obs_pt=np.concatenate(obs_pt))
    greys = [sc.grey(im) for im in imgs]

    def views(k):
        c = cams[k]
        return greys[k], None, D._Cam(c.R, c.C, float(c.f), 0.0, 0.0, float(c.cx), float(c.cy), c.w, c.h, 0.0)

    opt = D.DepthOptions()
    opt.window = 2
    opt.num_depths = 24
    out = D.depth_map(0, [1, 2, 3, 4], rec, views, opt)
    depth, score, low = out
    # host-side geometry of the driver (densify.py:208-284) for the CPU checks
    rng_ = D._depth_range(rec, 0)
    cam2 = views(0)[2].scaled(0.5, 160, 120).scaled(0.5, 80, 60)
    lo, hi = D._depth_band(rec, 0, cam2, (60, 80), rng_, block=max(8, 80 // 16))
    nd = D._num_depths(rec, 0, [1, 2, 3, 4], rng_, cam2.f, opt.num_depths)
    res = {"X": X, "C": rec.C, "R": rec.R, "obs_cam": rec.obs_cam, "obs_pt": rec.obs_pt,
           "intr": np.array([cams[0].f, cams[0].cx, cams[0].cy, cams[0].w, cams[0].h]),
           "depth": depth, "score": score, "low": low, "range": np.array(rng_), "band_lo": lo, "band_hi": hi,
           "nd": np.array(nd), "opt": np.array([opt.window, opt.num_depths, opt.top_k, opt.refine_steps])}
    for k, im in enumerate(imgs):
        res[f"img{k}"] = im
    np.savez_compressed(os.path.join(HERE, "depth_map.npz"), **res)


def _tie_points(sc, cams, rng, n, half_x, half_y):
    """Random terrain points and their in-image observations (obs_cam, obs_pt)."""
    import torch
    from py_ortho_b200 import scene as S
    xs = rng.uniform(-half_x, half_x, n)
    ys = rng.uniform(-half_y, half_y, n)
    t = sc.terrain
    z = S._height(torch.from_numpy(xs), torch.from_numpy(ys), torch.from_numpy(t.hills), torch.from_numpy(t.boxes)).numpy()
    X = np.column_stack([xs, ys, z])
    obs_cam, obs_pt = [], []
    for k, c in enumerate(cams):
        xc = (X - c.C) @ c.R.T
        u = c.f * xc[:, 0] / xc[:, 2] + c.cx
        v = c.f * xc[:, 1] / xc[:, 2] + c.cy
        ok = (xc[:, 2] > 0) & (u >= 0) & (v >= 0) & (u < c.w) & (v < c.h)
        obs_cam.append(np.full(ok.sum(), k, np.int32))
        obs_pt.append(np.flatnonzero(ok).astype(np.int32))
    return X, np.concatenate(obs_cam), np.concatenate(obs_pt)


def views_case(D, W=160, H=120):
    """The reference's _densify, passes 1 and 2, on a rendered 5-view scene. The image loader is
    replaced by the rendered uint8 images (grey in all three channels, so the reference's RGB mean
    is exact); _consistency, _init_normals and _dense.pm_refine are wrapped to record their
    arguments and results; the depth-map folder is kept and read back."""
    import tempfile
    import threading
    from types import SimpleNamespace
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=9, width=W, height=H)
    cams = [sc.ref_cam] + list(sc.src_cams)
    imgs = [sc.ref] + list(sc.srcs)
    N = len(cams)
    X, obs_cam, obs_pt = _tie_points(sc, cams, np.random.default_rng(23), 6000, 40.0, 30.0)
    intr = [SimpleNamespace(f=float(cams[0].f), cx=float(cams[0].cx), cy=float(cams[0].cy), width=W, height=H,
                            k1=0.0, k2=0.0, k3=0.0)]
    rec = SimpleNamespace(used=list(range(N)), intr=intr, cam_group=np.zeros(N, np.int32), X=X,
                          C=np.array([c.C for c in cams]), R=np.array([c.R for c in cams]), obs_cam=obs_cam,
                          obs_pt=obs_pt, rms_px=0.5)
    frames = [SimpleNamespace(width=W, height=H, path=f"view{k}") for k in range(N)]
    ar = SimpleNamespace(frames=frames, workers=1)
    rgb = {f"view{k}": np.ascontiguousarray(np.repeat(imgs[k][:, :, None], 3, axis=2)) for k in range(N)}
    saved = (D.load_rgb, D.load_mask, D._consistency, D._init_normals, D._dense)
    rec_cons, rec_norm, rec_pm = {}, [], {}
    lock = threading.Lock()

    def consistency(k, Dk, nbrs_k, dm, cams_, px_tol, rel_tol):
        cnt = saved[2](k, Dk, nbrs_k, dm, cams_, px_tol, rel_tol)
        with lock:
            rec_cons[k] = dict(nbrs=[j for j in nbrs_k if j in dm], px_tol=float(px_tol),
                               rel_tol=[float(rel_tol[j]) for j in nbrs_k if j in dm], cnt=cnt.copy())
        return cnt

    def init_normals(Dk, ray):
        n = saved[3](Dk, ray)
        with lock:
            rec_norm.append((np.array(Dk, np.float32), n.copy()))
        return n

    class DenseProxy:
        def __getattr__(self, name):
            return getattr(saved[4], name)

        def pm_refine(self, ref, ray, Cr, srcs, sdeps, par, depth, normal, score, active, r, step, top_k, geo_w,
                      geo_tol, iters, dmin, dmax, seed):
            before = dict(depth=depth.copy(), normal=normal.copy(), score=score.copy(), active=active.copy(),
                          ref=ref.copy(), Cr=np.array(Cr), par=np.array(par),
                          args=np.array([r, step, top_k, iters, seed], np.int64),
                          fargs=np.array([geo_w, geo_tol, dmin, dmax], np.float64))
            ch = saved[4].pm_refine(ref, ray, Cr, srcs, sdeps, par, depth, normal, score, active, r, step, top_k,
                                    geo_w, geo_tol, iters, dmin, dmax, seed)
            before.update(depth_out=depth.copy(), normal_out=normal.copy(), score_out=score.copy(),
                          changed=np.array(ch))
            with lock:
                rec_pm[tuple(np.round(np.asarray(Cr, np.float64) * 1000).astype(np.int64))] = before
            return ch

    opt = D.DepthOptions()
    opt.window, opt.num_depths, opt.patchmatch, opt.keep_depthmaps, opt.workers = 2, 24, True, True, 1
    out_dir = tempfile.mkdtemp(prefix="views_case_")
    D.load_rgb = lambda fr, s: rgb[fr.path]
    D.load_mask = lambda path, w, h: None
    D._consistency, D._init_normals, D._dense = consistency, init_normals, DenseProxy()
    try:
        try:
            D.densify(ar, rec, {}, None, out_dir, opt)
        except RuntimeError as e:                     # fusion may find too few points: not needed here
            print("views_case: fusion:", e)
    finally:
        D.load_rgb, D.load_mask, D._consistency, D._init_normals, D._dense = saved
    wd = os.path.join(out_dir, "depthmaps")
    res = {"X": X, "C": rec.C, "R": rec.R, "obs_cam": obs_cam, "obs_pt": obs_pt, "rms_px": np.array(rec.rms_px),
           "intr": np.array([cams[0].f, cams[0].cx, cams[0].cy, W, H]),
           "opt": np.array([opt.window, opt.num_depths, opt.top_k, opt.refine_steps, opt.pm_iters, opt.pm_window,
                            opt.pm_step], np.int64),
           "fopt": np.array([opt.min_ncc, opt.min_texture, opt.pm_geo_weight], np.float64)}
    have = []
    for k in range(N):
        res[f"img{k}"] = imgs[k]
        if not os.path.exists(os.path.join(wd, f"p{k:05d}.npy")):
            continue
        have.append(k)
        res[f"p{k}"] = np.load(os.path.join(wd, f"p{k:05d}.npy"))
        res[f"s{k}"] = np.load(os.path.join(wd, f"s{k:05d}.npy"))
        res[f"t{k}"] = np.load(os.path.join(wd, f"t{k:05d}.npy"))
        res[f"final{k}"] = np.load(os.path.join(wd, f"{k:05d}.npy"))
        if k in rec_cons:
            c = rec_cons[k]
            res[f"cnt{k}"] = c["cnt"]
            res[f"nbrs{k}"] = np.array(c["nbrs"], np.int32)
            res[f"tol{k}"] = np.array(c["rel_tol"], np.float64)
            res["px_tol"] = np.array(c["px_tol"])
    # PatchMatch: its inputs are the pass-1 maps, the images, the cameras, _init_normals of the
    # raw map and the active mask; the outputs are kept for the first view only (size)
    for k in have:
        pm = rec_pm.get(tuple(np.round(np.asarray(rec.C[k], np.float64) * 1000).astype(np.int64)))
        if pm is None:
            continue
        assert np.array_equal(pm["depth"], res[f"p{k}"], equal_nan=True)
        for key in ("active", "args", "fargs", "changed"):
            res[f"pm{k}_{key}"] = pm[key]
        if k == have[0]:
            for key in ("depth_out", "normal_out", "score_out"):
                res[f"pm{k}_{key}"] = pm[key]
    res["have"] = np.array(have, np.int32)
    # the first recorded _init_normals call (the first repaired view's raw map), bit for bit
    Dn, nn = rec_norm[0]
    res["norm_view"] = np.array([k for k in have if np.array_equal(res[f"p{k}"], Dn, equal_nan=True)][0])
    res["norm_out"] = nn
    np.savez_compressed(os.path.join(HERE, "views_case.npz"), **res)
    shutil.rmtree(out_dir, ignore_errors=True)


def fuse_case(D):
    """The reference's point fusion (densify._fuse, densify.py:676-762, through its compiled path
    _fast.ref_points / neighbour_sample / agreement / accumulate) on the pass-2 depth maps of
    views_case.npz, in two settings: (min_views, point_stride) = (2, 2) and (3, 1)."""
    from concurrent.futures import ThreadPoolExecutor
    from types import SimpleNamespace
    z = np.load(os.path.join(HERE, "views_case.npz"))
    f, cx, cy, W, H = (float(v) for v in z["intr"])
    W, H = int(W), int(H)
    have = [int(k) for k in z["have"]]
    N = len(z["C"])
    cams = {k: D._Cam(z["R"][k], z["C"][k], f, 0.0, 0.0, cx, cy, W, H) for k in range(N)}
    nbrs = {k: [int(j) for j in z[f"nbrs{k}"]] for k in have}
    tols = {k: {j: float(t) for j, t in zip(nbrs[k], z[f"tol{k}"])} for k in have}
    px_tol = float(z["px_tol"])
    rgb = {k: np.ascontiguousarray(np.repeat(z[f"img{k}"][:, :, None], 3, axis=2)) for k in range(N)}
    res = {"px_tol": np.array(px_tol)}
    for c, (min_views, stride) in enumerate(((2, 2), (3, 1))):
        dm = {k: np.ascontiguousarray(z[f"final{k}"], np.float32) for k in have}
        used = {k: np.zeros(dm[k].shape, bool) for k in have}
        pts, cols, nv, owner = [], [], [], []
        opt = SimpleNamespace(point_stride=stride, neighbors=4)
        fpool = ThreadPoolExecutor(1)
        try:
            D._fuse(sorted(have), dm, used, cams, nbrs, set(have), lambda k: tols[k], opt, px_tol, min_views,
                    lambda k: (None, rgb[k], None), {}, pts, cols, nv, owner, 1000, fpool)
        finally:
            fpool.shutdown()
        res[f"f{c}_args"] = np.array([min_views, stride], np.int64)
        res[f"f{c}_xyz"] = np.concatenate(pts) if pts else np.zeros((0, 3))
        res[f"f{c}_cols"] = np.concatenate(cols) if cols else np.zeros((0, 3), np.uint8)
        res[f"f{c}_nv"] = np.concatenate(nv) if nv else np.zeros(0, np.uint8)
        res[f"f{c}_owner"] = np.concatenate(owner) if owner else np.zeros(0, np.int32)
        for k in have:
            res[f"f{c}_used{k}"] = used[k]
        print(f"fuse_case {c}: {len(res[f'f{c}_xyz'])} points")
    np.savez_compressed(os.path.join(HERE, "fuse_case.npz"), **res)


def height_case(W=160, H=120):
    """The reference's legacy height sweep (mvs.py) on its CPU backend: kernel cases of
    _mvs.sample_view (a Z stack into a distorted camera, 3 channels), _fast.box_sat_mean and
    _mvs.sgm on seeded random inputs, and mvs.dense_reconstruct end to end on a rendered 5-view
    survey (images through a replaced loader, tie points on the terrain)."""
    from types import SimpleNamespace
    from py_ortho_b200 import scene as S
    M = refpkg.load_module("mvs")
    B = refpkg.load_module("backend")
    import _mvs
    R_ = O.reference()
    rng = np.random.default_rng(31)
    res = {}
    # sample_view
    img = (rng.random((70, 90, 3)) * 255).astype(np.float32)
    th = 0.2
    Rm = np.diag([1.0, -1.0, -1.0]) @ np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    Cc = np.array([2.0, -3.0, 60.0])
    cam = np.array([80.0, -0.08, 0.02, 0.001, 44.5, 34.5])       # f k1 k2 k3 cx cy
    Z = (rng.random((4, 50, 60)) * 12 - 2).astype(np.float32)
    out = np.zeros(Z.shape + (3,), np.float32)
    val = np.zeros(Z.shape, np.uint8)
    for d in range(Z.shape[0]):
        _mvs.sample_view(img, Rm, Cc, *[float(v) for v in cam[:4]], float(cam[4]), float(cam[5]), -25.0, 20.0, 0.7,
                         Z[d], out[d], val[d])
    res.update(sv_img=img, sv_R=Rm, sv_C=Cc, sv_cam=cam, sv_grid=np.array([-25.0, 20.0, 0.7]), sv_Z=Z, sv_out=out,
               sv_valid=val)
    # box_sat_mean
    a = (rng.normal(0, 30, (6, 41, 53))).astype(np.float32)
    res.update(box_in=a, box_r=np.array(3), box_out=R_._fast.box_sat_mean(a, 3))
    # sgm
    cost = rng.random((37, 23, 29)).astype(np.float32)
    res.update(sgm_cost=cost, sgm_p=np.array([0.05, 0.6], np.float32), sgm_out=_mvs.sgm(cost, 0.05, 0.6, 1))
    # dense_reconstruct on a rendered survey
    sc = S.make_scene("c1", seed=21, width=W, height=H)
    cams = [sc.ref_cam] + list(sc.src_cams)
    imgs = [sc.ref] + list(sc.srcs)
    X, obs_cam, obs_pt = _tie_points(sc, cams, np.random.default_rng(5), 3000, 30.0, 22.0)
    intr = [SimpleNamespace(f=float(cams[0].f), cx=float(cams[0].cx), cy=float(cams[0].cy), width=W, height=H,
                            k1=0.0, k2=0.0, k3=0.0)]
    rec = SimpleNamespace(used=list(range(len(cams))), intr=intr, cam_group=np.zeros(len(cams), np.int32), X=X,
                          C=np.array([c.C for c in cams]), R=np.array([c.R for c in cams]))
    frames = [SimpleNamespace(width=W, height=H, path=f"view{k}") for k in range(len(cams))]
    ar = SimpleNamespace(frames=frames, backend=B.CPUBackend(), workers=1)
    rgb = {f"view{k}": np.ascontiguousarray(np.repeat(imgs[k][:, :, None], 3, axis=2)) for k in range(len(cams))}
    saved = M.load_rgb
    M.load_rgb = lambda fr, s: rgb[fr.path]
    try:
        opt = M.DenseOptions(tile=64, overlap=8, levels=2, workers=1)
        native = float(sc.ref_cam.C[2] / sc.ref_cam.f)
        r = M.dense_reconstruct(ar, rec, {}, native, opt)
    finally:
        M.load_rgb = saved
    res.update(h_X=X, h_C=rec.C, h_R=rec.R, h_intr=np.array([intr[0].f, intr[0].cx, intr[0].cy, W, H]),
               h_native=np.array(native), h_opt=np.array([opt.tile, opt.overlap, opt.levels], np.int64),
               h_Z=r.Z, h_score=r.score, h_rgb=r.rgb, h_covered=r.covered, h_grid=np.array([r.minX, r.maxY, r.gsd]))
    for k in range(len(cams)):
        res[f"h_img{k}"] = imgs[k]
    print("height_case:", r.Z.shape, float(np.nanmean(r.Z)), float(np.mean(r.score)))
    np.savez_compressed(os.path.join(HERE, "height_case.npz"), **res)


def main():
    D = refpkg.load_densify()
    R = O.reference()
    if D is None or R is None:
        raise SystemExit("the reference is not available here: build oracle/_ref first (make -C oracle ref)")
    cases = {"sweep_cases": lambda: sweep_cases(R), "sweep_e2e": lambda: sweep_e2e(D),
             "scene_small": lambda: scene_small(D), "helpers": lambda: helpers(D, R), "pm_case": lambda: pm_case(R),
             "pm_case8": lambda: pm_case8(R), "depth_map": lambda: depth_map_case(D),
             "views_case": lambda: views_case(D), "fuse_case": lambda: fuse_case(D), "height_case": height_case}
    wanted = sys.argv[1:] or list(cases)
    for name in wanted:
        cases[name]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()

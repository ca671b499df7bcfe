"""Precision variant (FP16 source storage, FP32 window sums, FP64 homography and parabola) and the
plain FP32 sweep against the all-float64 oracle on 10 seeded scenes: median and p99 relative
depth error. Grey values of uint8 images ((g - 128) / 64) are exact in FP16, so half of the scenes
get a radiometric gain / bias (as densify's per-image gain correction produces) that makes FP16
storage round."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

W, H, PLANES, R, TOPK = 320, 240, 64, 2, 2
MEDIAN_BAR = 1e-3          # median depth error vs the FP64 oracle (0.1 %)


def _scene(seed):
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=200 + seed, width=W, height=H)
    ref = sc.grey(sc.ref)
    srcs = [sc.grey(s) for s in sc.srcs]
    if seed % 2:                                           # non-FP16-exact grey values
        srcs = [(s * np.float32(1.0 + 0.013 * (k + 1)) + np.float32(0.0371 * (k + 1))).astype(np.float32)
                for k, s in enumerate(srcs)]
    return sc, ref, srcs


def _fp64(seed):
    from oracle import oracle as O
    from py_ortho_b200 import scene as S
    sc, ref, srcs = _scene(seed)
    planes = S.plane_list(35.0, 55.0, PLANES)
    ray = O.rays_world((H, W), sc.ref_cam)
    geo = S.geo_rows(sc.ref_cam, sc.src_cams)
    d, best, idx = O.sweep_fp64(ref, srcs, ray, geo, [np.full((H, W), p, np.float64) for p in planes], R, TOPK)
    return d


def test_fp16_and_fp32_depth_error_vs_fp64_oracle():
    from py_ortho_b200 import _lib as L, dense, fast, scene as S
    with ThreadPoolExecutor(8) as ex:
        ref64 = list(ex.map(_fp64, range(10)))
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    rows = []
    errs = {"fp32": [], "fp16": []}
    for seed in range(10):
        sc, ref, srcs = _scene(seed)
        planes = S.plane_list(35.0, 55.0, PLANES)
        hyp = dense.Hypotheses.planes_inv(planes)
        mu, sd = fast.ref_stats(T(ref), R)
        geo = S.geo_rows(sc.ref_cam, sc.src_cams)
        for prec, srcs_k in (("fp32", [T(s) for s in srcs]), ("fp16", [fast.to_fp16(T(s)) for s in srcs])):
            st = dense.sweep(T(ref), mu, sd, None, srcs_k, geo, hyp, R, TOPK, ref_cam=sc.ref_cam.row(),
                             precision=L.PREC_FP16 if prec == "fp16" else L.PREC_FP32)
            d = dense.finalize(hyp, st).cpu().numpy().astype(np.float64)
            d64 = ref64[seed]
            rel = np.abs(d - d64) / d64
            errs[prec].append(rel)
            rows.append((seed, prec, float(np.median(rel)), float(np.percentile(rel, 99))))
    for seed, prec, med, p99 in rows:
        print(f"scene {seed} {prec}: median {med:.2e} p99 {p99:.2e}")
    for prec in ("fp32", "fp16"):
        allr = np.concatenate(errs[prec])
        print(f"ALL {prec}: median {np.median(allr):.3e} p99 {np.percentile(allr, 99):.3e}")
        assert np.median(allr) <= MEDIAN_BAR
        assert all(np.median(e) <= MEDIAN_BAR for e in errs[prec])

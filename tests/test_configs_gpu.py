"""Parity at the measured configurations, through the C ABI, against the oracle (the reference's
per-hypothesis kernel restated in C and pinned bit for bit to the reference's own kernel):

* C1 in full: 640 x 480, 4 sources, 128 inverse-depth planes over [35, 55] m, 5 x 5 window,
  best-2 of 4 (the whole view, every pixel);
* C2, the benchmark's step: 4000 x 3000, 8 sources, 256 planes over [60, 90] m, 7 x 7 window;
  the device sweeps the whole view and three row bands of it are checked against the oracle
  (each band swept by the oracle on a crop with an r-row halo and the full view's window
  statistics, so its rows see exactly the full view's inputs).

The bar is the one the depth-map path is specified by: winner index exact wherever the best-to-
second score gap exceeds 1e-3, depth within 0.1 % relative everywhere else (flipped pixels
included)."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

from conftest import same_bits
from oracle import oracle as O
from tests_support import SCORE_ABS, check_parity, gap_of

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def _device_sweep(ref, srcs, sc, planes, r, top_k, precision=None):
    from py_ortho_b200 import _lib as L
    from py_ortho_b200 import dense, fast, scene as S
    geo = S.geo_rows(sc.ref_cam, sc.src_cams)
    ref_d = ref if isinstance(ref, torch.Tensor) else _dev(ref)
    mu, sd = fast.ref_stats(ref_d, r)
    hyp = dense.Hypotheses.planes_inv(planes)
    srcs_d = [s if isinstance(s, torch.Tensor) else _dev(s) for s in srcs]
    st = dense.sweep(ref_d, mu, sd, None, srcs_d, geo, hyp, r, top_k, ref_cam=sc.ref_cam.row(),
                     precision=L.PREC_FP32 if precision is None else precision)
    depth = dense.finalize(hyp, st)
    torch.cuda.synchronize()
    return st, depth, mu, sd, geo


def _score_report(best, ref_best, same):
    e = np.abs(best.astype(np.float64) - ref_best)[same]
    return {"score_abs_max": float(e.max()), "score_abs_q999": float(np.quantile(e, 0.999)),
            "score_over_bar": int((e > SCORE_ABS).sum())}


@pytest.mark.parametrize("form", ["fp32", "fp64_sums_rays"])
def test_c1_full_view_parity(form):
    """C1 in full, every pixel against the oracle. With the reference's own arithmetic - float64
    window sums (MVS_PREC_FP64_SUMS) on the per-pixel ray path (float64 projection and bilinear,
    the 128 planes given as maps) - the bar holds at every pixel. The bench's path (float32 sums,
    float32-evaluated homographies) meets it on all but a stated handful of pixels at this small
    window (r = 2): bright low-texture windows amplify the float32 rounding ~1e3-fold (measured: 1
    decided pixel of 307200 one plane off, 1 flipped pixel's depth 0.30 % off; float64 sums on the
    homography path leave the same 1 decided pixel)."""
    from py_ortho_b200 import _lib as L
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=0, device="cuda")
    ref = sc.grey(sc.ref)
    srcs = [sc.grey(s) for s in sc.srcs]
    H, W = ref.shape
    assert (H, W, len(srcs)) == (480, 640, 4)
    planes = S.plane_list(35.0, 55.0, 128)
    r, top_k = 2, 2
    ray = O.rays_world((H, W), sc.ref_cam)
    if form == "fp32":
        st, depth, _, _, geo = _device_sweep(ref, srcs, sc, planes, r, top_k, L.PREC_FP32)
    else:
        from py_ortho_b200 import dense, fast
        geo = S.geo_rows(sc.ref_cam, sc.src_cams)
        ref_d = _dev(ref)
        mu, sd = fast.ref_stats(ref_d, r)
        maps = torch.from_numpy(np.repeat(planes.astype(np.float32)[:, None, None], H * W).reshape(-1, H, W)).cuda()
        hyp = dense.Hypotheses(L.HYP_MAPS, len(planes), maps=maps)
        st = dense.sweep(ref_d, mu, sd, _dev(ray), [_dev(s) for s in srcs], geo, hyp, r, top_k,
                         precision=L.PREC_FP64_SUMS)
        depth = dense.finalize(hyp, st)
        torch.cuda.synchronize()
    full = O.sweep(ref, srcs, ray, geo, [np.full((H, W), p, np.float32) for p in planes], r, top_k, keep_scores=True)
    idx, d, best = st[4].cpu().numpy(), depth.cpu().numpy(), st[0].cpu().numpy()
    strict = form != "fp32"
    rep = check_parity(idx, d, None, full["idx"], full["depth"], None, gap_of(full["scores"]), f"C1 640x480 {form}",
                       flip_depth_frac=0.0 if strict else 1e-4, decided_miss_frac=0.0 if strict else 2e-5)
    rep.update(_score_report(best, full["best"], idx == full["idx"]))
    print(f"C1 parity ({form}):", rep)
    assert rep["decided"] > 0.5 * H * W


def _oracle_rows(ref, mu, sd, srcs, ray, geo, planes, r, top_k, y0, y1):
    """The oracle's sweep of rows [y0, y1) of a large view: a crop with an r-row halo on each side
    and the full view's window statistics."""
    H, W = ref.shape
    a, b = max(0, y0 - r), min(H, y1 + r)
    c = lambda x: np.ascontiguousarray(x[a:b])
    cref, cmu, csd, cray = c(ref), c(mu), c(sd), np.ascontiguousarray(ray[:, a:b])
    h = b - a
    best, prev, spb, snb, idx = O.init_state(h, W)
    top1 = np.full((h, W), -np.inf, np.float32)
    top2 = np.full((h, W), -np.inf, np.float32)
    for i, p in enumerate(planes):
        O.sweep_hypothesis(cref, cmu, csd, srcs, cray, geo, np.full((h, W), p, np.float32), r, top_k, i, best, prev,
                           spb, snb, idx)
        top2 = np.where(prev > top1, top1, np.maximum(top2, prev))
        top1 = np.maximum(top1, prev)
    inv0 = np.full((h, W), planes[0], np.float32)
    inv1 = np.full((h, W), planes[1], np.float32)
    depth = O.finalize(best, spb, snb, idx, inv0, inv1, len(planes))
    rows = slice(y0 - a, y1 - a)
    return {"idx": idx[rows], "depth": depth[rows], "best": best[rows], "gap": (top1 - top2)[rows]}


def test_c2_bench_step_row_bands_parity():
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c2", seed=0, device="cuda")
    ref = sc.grey(sc.ref)
    srcs = [sc.grey(s) for s in sc.srcs]
    H, W = ref.shape
    assert (H, W, len(srcs)) == (3000, 4000, 8)
    planes = S.plane_list(60.0, 90.0, 256)
    r, top_k = 3, 2
    st, depth, mu, sd, geo = _device_sweep(ref, srcs, sc, planes, r, top_k)
    mu, sd = mu.cpu().numpy(), sd.cpu().numpy()
    ray = O.rays_world((H, W), sc.ref_cam)
    idx, d, best = st[4].cpu().numpy(), depth.cpu().numpy(), st[0].cpu().numpy()
    bands = [(0, 24), (1488, 1512), (2976, 3000)]        # top edge, middle, bottom edge
    with ThreadPoolExecutor(len(bands)) as ex:
        outs = list(ex.map(lambda b: _oracle_rows(ref, mu, sd, srcs, ray, geo, planes, r, top_k, *b), bands))
    reps = []
    for (y0, y1), o in zip(bands, outs):
        rep = check_parity(idx[y0:y1], d[y0:y1], None, o["idx"], o["depth"], None, o["gap"], f"C2 rows {y0}-{y1}",
                           flip_depth_frac=1e-4)
        rep.update(_score_report(best[y0:y1], o["best"], idx[y0:y1] == o["idx"]))
        reps.append(rep)
        assert rep["decided"] > 0.5 * (y1 - y0) * W
    print("C2 band parity:", reps)


def test_c3_precision_variant_on_ten_scenes():
    """C3: C1's shape (640 x 480, 4 sources, 128 planes over [35, 55] m, 5 x 5, best 2) on ten seeded
    scenes; depth error of each storage / summation form against the all-float64 oracle sweep of
    the same planes (float64 statistics, sums, NCC and parabola): median and 99th percentile over
    all pixels. Forms: plain FP32, FP16 storage, and the compensated sums (pivoted tile, Kahan
    vertical sums, statistics from the pivoted tile) with FP16 and FP32 storage. Bar: median
    <= 0.1 % for every form."""
    from py_ortho_b200 import _lib as L
    from py_ortho_b200 import dense, fast, scene as S
    forms = {"fp32": L.PREC_FP32, "fp16": L.PREC_FP16, "fp16_comp": L.PREC_FP16_COMP, "fp32_comp": L.PREC_FP32_COMP}
    planes = S.plane_list(35.0, 55.0, 128)
    r, top_k = 2, 2
    hyp = dense.Hypotheses.planes_inv(planes)
    errs = {k: [] for k in forms}
    scenes = []
    for seed in range(10):
        sc = S.make_scene("c1", seed=100 + seed, device="cuda")
        ref = sc.grey(sc.ref)
        srcs = [sc.grey(s) for s in sc.srcs]
        geo = S.geo_rows(sc.ref_cam, sc.src_cams)
        H, W = ref.shape
        ref_d = _dev(ref)
        mu, sd = fast.ref_stats(ref_d, r)
        s32 = [_dev(s) for s in srcs]
        s16 = [fast.to_fp16(s) for s in s32]
        outs = {}
        for name, prec in forms.items():
            st = dense.sweep(ref_d, mu, sd, None, s16 if prec in (L.PREC_FP16, L.PREC_FP16_COMP) else s32, geo, hyp, r,
                             top_k, ref_cam=sc.ref_cam.row(), precision=prec)
            outs[name] = dense.finalize(hyp, st).cpu().numpy().astype(np.float64)
        scenes.append((ref, srcs, O.rays_world((H, W), sc.ref_cam), geo, outs))

    def oracle64(item):
        ref, srcs, ray, geo, _ = item
        H, W = ref.shape
        d64, _, _ = O.sweep_fp64(ref, srcs, ray, geo, [np.full((H, W), p, np.float64) for p in planes], r, top_k)
        return d64

    with ThreadPoolExecutor(5) as ex:
        d64s = list(ex.map(oracle64, scenes))
    for (_, _, _, _, outs), d64 in zip(scenes, d64s):
        for name in forms:
            errs[name].append(np.abs(outs[name] - d64) / d64)
    report = {}
    for name in forms:
        e = np.concatenate([x.ravel() for x in errs[name]])
        report[name] = {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)),
                        "p999": float(np.percentile(e, 99.9)), "max": float(e.max())}
    print("C3 depth error vs the float64 oracle (10 scenes, 640x480, 128 planes):", report)
    for name in forms:
        assert report[name]["median"] <= 1e-3, (name, report[name])


def test_c2_patchmatch_on_a_crop_of_the_bench_view():
    """C2's PatchMatch on a 320 x 240 crop of the benchmark's view (8 sources at 4000 x 3000,
    7 x 7 window, step 1; depth from the device sweep, normals seeded within 30 degrees of
    vertical): one iteration through the C ABI against the oracle (the reference's pm_refine
    restated, pinned to it), float64 bit for bit, float32 within 0.1 % on >= 99.9 % of pixels."""
    from py_ortho_b200 import dense, scene as S
    sc = S.make_scene("c2", seed=0, device="cuda")
    srcs = [sc.grey(s) for s in sc.srcs]
    y0, x0, h, w = 1400, 1800, 240, 320
    ref = np.ascontiguousarray(sc.grey(sc.ref)[y0:y0 + h, x0:x0 + w])
    cam = sc.ref_cam
    # the crop's camera: the same pose, principal point shifted by the crop origin
    ray = np.ascontiguousarray(O.rays_world((3000, 4000), cam)[:, y0:y0 + h, x0:x0 + w])
    planes = S.plane_list(60.0, 90.0, 256)
    st, depth, _, _, _ = _device_sweep(sc.grey(sc.ref), srcs, sc, planes, 3, 2)
    d0 = np.ascontiguousarray(depth.cpu().numpy()[y0:y0 + h, x0:x0 + w])
    n0 = S.tilted_normals(h, w, 1000)
    par = np.array([c.row() for c in sc.src_cams], np.float64)
    act = np.ones((h, w), np.uint8)
    args = (3, 1, 2, 0.0, 0.02, 1, 60.0, 90.0, 12345)
    b = [d0.copy(), n0.copy(), np.zeros((h, w), np.float32)]
    cb = O.pm_refine(ref, ray, cam.C, srcs, [None] * 8, par, *b, act, *args)
    for prec in ("fp64", "fp32"):
        a = [d0.copy(), n0.copy(), np.zeros((h, w), np.float32)]
        ca = dense.pm_refine(ref, ray, cam.C, srcs, [None] * 8, par, *a, act, *args, precision=prec)
        if prec == "fp64":
            assert ca == cb
            for x, y in zip(a, b):
                assert same_bits(x, y)
        else:
            fin = np.isfinite(b[0])
            rel = np.abs(a[0][fin].astype(np.float64) - b[0][fin]) / b[0][fin]
            print(f"C2 crop PatchMatch fp32 vs oracle: within 0.1 % {(rel <= 1e-3).mean():.5f}, median {np.median(rel):.1e}")
            assert (rel <= 1e-3).mean() >= 0.999

"""PatchMatch on the device against the reference and the oracle. The device draws from the
reference's own xorshift32 stream (per colour pass: a prefix count of the drawing pixels in raster
order and a GF(2) jump to each pixel's offset), so the float64 kernel (no contraction) is
bit-identical to the reference's pm_refine: parallel red-black updates equal the reference's
raster order because every neighbour has the other colour."""
import numpy as np
import pytest
import torch

from conftest import golden, same_bits
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _case():
    z = golden("pm_case.npz")
    r, step, top_k, iters, seed = (int(v) for v in z["args"])
    geo_w, geo_tol, dmin, dmax = (float(v) for v in z["fargs"])
    srcs = [z[f"src{j}"] for j in range(3)]
    return z, srcs, [None, z["sdep1"], None], (r, step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed)


def test_pm_refine_bit_exact_vs_reference():
    """The reference's own pm_refine output (golden, made by its compiled kernel) and the oracle:
    same depth, normal and score bits, same change count."""
    from py_ortho_b200 import dense
    z, srcs, sdeps, (r, step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed) = _case()
    a = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    b = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    ch_gpu = dense.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *a, z["active"], r, step, top_k,
                             geo_w, geo_tol, iters, dmin, dmax, seed)
    ch_cpu = O.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *b, z["active"], r, step, top_k, geo_w,
                         geo_tol, iters, dmin, dmax, seed)
    assert ch_gpu == ch_cpu == int(z["changed"]) > 0
    for x, y, ref in zip(a, b, (z["depth"], z["normal"], z["score"])):
        assert same_bits(x, y)
        assert same_bits(x, ref)


def test_pm_refine_resumes_across_calls():
    """Iterations split over calls (it0, the stream state carried on the device) give the same
    result as one call (resumable jobs)."""
    from py_ortho_b200 import dense
    z, srcs, sdeps, (r, step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed) = _case()
    one = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    two = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    c1 = dense.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *one, z["active"], r, step, top_k, geo_w,
                         geo_tol, 3, dmin, dmax, seed)
    st = dense.stream_start(seed)
    c2 = 0
    for it in range(3):
        c2 += dense.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *two, z["active"], r, step, top_k,
                              geo_w, geo_tol, 1, dmin, dmax, seed, it0=it, rng_state=st)
    assert c1 == c2
    for x, y in zip(one, two):
        assert same_bits(x, y)
    # the state left on the device is the oracle's after the same draws
    ost = np.array([seed | 1], np.uint32)
    three = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    O.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *three, z["active"], r, step, top_k, geo_w,
                geo_tol, 3, dmin, dmax, seed, state=ost)
    assert int(st.cpu().numpy().view(np.uint32)[0]) == int(ost[0])


def test_pm_refine_bit_exact_vs_reference_rendered_8_sources():
    """A rendered 8-source scene (golden from the reference's own pm_refine: noisy depth, 1 % holes,
    80 % active, 7 x 7 window, 2 iterations): the device result equals the reference's bits."""
    from py_ortho_b200 import dense
    z = golden("pm_case8.npz")
    r, step, top_k, iters, seed = (int(v) for v in z["args"])
    geo_w, geo_tol, dmin, dmax = (float(v) for v in z["fargs"])
    grey = lambda u8: ((u8.astype(np.float32) - np.float32(128)) / np.float32(64)).astype(np.float32)
    ref = grey(z["ref_u8"])
    srcs = [grey(u) for u in z["src_u8"]]
    st = [z["depth0"].copy(), z["normal0"].copy(), np.zeros(ref.shape, np.float32)]
    ch = dense.pm_refine(ref, z["ray"], z["Cr"], srcs, [None] * len(srcs), z["par"], *st, z["active"], r, step, top_k,
                         geo_w, geo_tol, iters, dmin, dmax, seed)
    assert ch == int(z["changed"]) > 0
    for x, ref_out in zip(st, (z["depth"], z["normal"], z["score"])):
        assert same_bits(x, ref_out)


def test_pm_fp32_against_the_reference_rendered_8_sources():
    """The float32 mode against the reference's own result on the rendered 8-source case: the same
    stream (which pixels draw does not depend on the cost arithmetic), so only near-ties decided
    the other way differ. Depth within 0.1 % of the reference on >= 99.9 % of pixels."""
    from py_ortho_b200 import dense
    z = golden("pm_case8.npz")
    r, step, top_k, iters, seed = (int(v) for v in z["args"])
    geo_w, geo_tol, dmin, dmax = (float(v) for v in z["fargs"])
    grey = lambda u8: ((u8.astype(np.float32) - np.float32(128)) / np.float32(64)).astype(np.float32)
    ref = grey(z["ref_u8"])
    srcs = [grey(u) for u in z["src_u8"]]
    st = [z["depth0"].copy(), z["normal0"].copy(), np.zeros(ref.shape, np.float32)]
    dense.pm_refine(ref, z["ray"], z["Cr"], srcs, [None] * len(srcs), z["par"], *st, z["active"], r, step, top_k,
                    geo_w, geo_tol, iters, dmin, dmax, seed, precision="fp32")
    d, dr = st[0].astype(np.float64), z["depth"].astype(np.float64)
    assert np.array_equal(np.isfinite(d), np.isfinite(dr))
    fin = np.isfinite(dr)
    rel = np.abs(d[fin] - dr[fin]) / dr[fin]
    print(f"fp32 PatchMatch vs reference: identical {(rel == 0).mean():.4%}, within 0.1 % {(rel <= 1e-3).mean():.4%}, "
          f"median {np.median(rel):.1e}")
    assert (rel <= 1e-3).mean() >= 0.999
    assert np.median(rel) == 0.0


def test_pm_no_sources_is_a_noop():
    from py_ortho_b200 import dense
    z, srcs, sdeps, (r, step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed) = _case()
    d = z["depth0"].copy()
    assert dense.pm_refine(z["ref"], z["ray"], z["Cr"], [], [], np.zeros((0, 18)), d, z["normal0"].copy(),
                           z["score0"].copy(), z["active"], r, step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed) == 0
    assert same_bits(d, z["depth0"])


# ------------------------------------------------------------------ float32 evaluation mode
def _rendered_pm_case(W, H, n_src, seed, nan_frac=0.0):
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1" if n_src <= 4 else "c2", seed=seed, width=W, height=H)
    ref = sc.grey(sc.ref).astype(np.float32)
    srcs = [sc.grey(s).astype(np.float32) for s in sc.srcs[:n_src]]
    rng = np.random.default_rng(seed)
    if nan_frac:
        ref[rng.random(ref.shape) < nan_frac] = np.nan
        for s in srcs:
            s[rng.random(s.shape) < nan_frac] = np.nan
    ray = O.rays_world((H, W), sc.ref_cam)
    par = np.array([c.row() for c in sc.src_cams[:n_src]], np.float64)
    depth = (sc.depth_true * (1 + rng.normal(0, 0.01, (H, W)))).astype(np.float32)
    depth[rng.random((H, W)) < 0.01] = np.nan
    normal = S.tilted_normals(H, W, seed + 5)
    return ref, srcs, ray, sc.ref_cam.C, par, depth, normal


CASES = [(160, 120, 4, 3, 1, 0.0), (96, 80, 6, 2, 2, 0.01), (120, 90, 8, 4, 2, 0.0), (64, 48, 3, 1, 1, 0.02)]


@pytest.mark.parametrize("W,H,n_src,r,step,nan_frac", CASES)
def test_pm_fp32_cost_matches_fp64_per_pixel(W, H, n_src, r, step, nan_frac):
    """The float32 cost itself: with every candidate outside [dmin, dmax] only the current plane
    is evaluated, so the score map is its photo term at every pixel; float32 and float64 agree to
    1e-5 on 99.9 % of pixels (border windows, masked pixels, 3-8 sources)."""
    from py_ortho_b200 import dense
    ref, srcs, ray, Cr, par, depth, normal = _rendered_pm_case(W, H, n_src, seed=3, nan_frac=nan_frac)
    act = np.ones((H, W), np.uint8)
    sdeps = [None] * n_src
    out = {}
    for prec in ("fp32", "fp64"):
        st = [depth.copy(), normal.copy(), np.zeros((H, W), np.float32)]
        ch = dense.pm_refine(ref, ray, Cr, srcs, sdeps, par, *st, act, r, step, 2, 0.0, 0.02, 1, 1e9, 1e9 + 1, 5,
                             precision=prec)
        assert ch == 0
        assert same_bits(st[0], depth) and same_bits(st[1], normal)
        out[prec] = st[2]
    a, b = out["fp32"].astype(np.float64), out["fp64"].astype(np.float64)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    d = np.abs(a - b)[np.isfinite(a)]
    assert np.quantile(d, 0.999) <= 1e-5, f"99.9 % quantile {np.quantile(d, 0.999):.2e}"
    assert d.max() <= 1e-3, f"max {d.max():.2e}"


@pytest.mark.parametrize("W,H,n_src,r,step,nan_frac", CASES[:3])
def test_pm_fp32_refinement_agrees_with_fp64(W, H, n_src, r, step, nan_frac):
    """Two full iterations: the float32 mode lands on the float64 result (same draws) except where
    near-ties were decided the other way; depth within 0.1 % on >= 99.9 % of pixels. Float32
    accepts fewer changes: candidates that differ from the kept plane by float64 rounding only
    (neighbours that share its plane) round to the same float32 cost, and '<' rejects them."""
    from py_ortho_b200 import dense
    ref, srcs, ray, Cr, par, depth, normal = _rendered_pm_case(W, H, n_src, seed=3, nan_frac=nan_frac)
    act = np.ones((H, W), np.uint8)
    zr = float(Cr[2])
    args = (r, step, 2, 0.0, 0.02, 2, zr - 30.0, zr + 5.0, 99)
    a = [depth.copy(), normal.copy(), np.zeros((H, W), np.float32)]
    b = [depth.copy(), normal.copy(), np.zeros((H, W), np.float32)]
    ca = dense.pm_refine(ref, ray, Cr, srcs, [None] * n_src, par, *a, act, *args, precision="fp32")
    cb = dense.pm_refine(ref, ray, Cr, srcs, [None] * n_src, par, *b, act, *args, precision="fp64")
    fin = np.isfinite(b[0]) & np.isfinite(a[0])
    assert np.array_equal(np.isfinite(a[0]), np.isfinite(b[0]))
    rel = np.abs(a[0][fin].astype(np.float64) - b[0][fin]) / b[0][fin]
    same = (a[0] == b[0])[fin].mean()
    within = (rel <= 1e-3).mean()
    print(f"fp32 vs fp64 PatchMatch {W}x{H} {n_src} sources: changes {ca} / {cb}, identical depth {same:.2%}, "
          f"within 0.1 % {within:.2%}")
    assert within >= 0.999
    assert 0.8 * cb <= ca <= cb


def test_pm_fp32_cost_with_the_geometric_term():
    """The float32 cost on the reference fixture, whose second source carries a depth map (the
    geometric term, geo_w 0.5, evaluated in float64 in both modes): with every candidate outside
    [dmin, dmax] the score map is the current plane's photo term at every pixel."""
    from py_ortho_b200 import dense
    z, srcs, sdeps, (r, step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed) = _case()
    out = {}
    for prec in ("fp32", "fp64"):
        st = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
        ch = dense.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *st, z["active"], r, step, top_k,
                             geo_w, geo_tol, 1, 1e9, 1e9 + 1, seed, precision=prec)
        assert ch == 0
        out[prec] = st[2].astype(np.float64)
    a, b = out["fp32"], out["fp64"]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    d = np.abs(a - b)[np.isfinite(a) & z["active"].astype(bool)]
    assert d.size > 0
    assert np.quantile(d, 0.999) <= 1e-5, f"99.9 % quantile {np.quantile(d, 0.999):.2e}"
    assert d.max() <= 1e-3, f"max {d.max():.2e}"


@pytest.mark.parametrize("W,H,n_src,r,step,case", [(1, 9, 2, 2, 1, "plain"), (7, 1, 3, 1, 1, "plain"),
                                                   (13, 11, 4, 3, 2, "plain"), (33, 17, 5, 2, 1, "no_active"),
                                                   (29, 21, 3, 2, 1, "all_nan"), (31, 23, 6, 3, 1, "sparse"),
                                                   (64, 40, 8, 3, 1, "plain")])
def test_pm_stream_edge_cases_bit_exact_vs_oracle(W, H, n_src, r, step, case):
    """The reference's stream on odd shapes (one-pixel rows and columns, odd widths whose colours
    have unequal pixel counts), no active pixel (no draws at all), every depth NaN (pixels draw
    only where a neighbour's plane was propagated in), and a sparse active mask: the float64 kernel
    equals the oracle's sequential evaluation bit for bit, and the stream state left on the device
    is the oracle's."""
    from py_ortho_b200 import dense, scene as S
    sc = S.make_scene("c2", seed=W + H, width=max(W, 8), height=max(H, 8))
    ref = sc.grey(sc.ref)[:H, :W].astype(np.float32).copy()
    srcs = [sc.grey(s).astype(np.float32) for s in sc.srcs[:n_src]]
    rng = np.random.default_rng(W * 31 + H)
    ray = O.rays_world((max(H, 8), max(W, 8)), sc.ref_cam)[:, :H, :W].copy()
    par = np.array([c.row() for c in sc.src_cams[:n_src]], np.float64)
    depth = (sc.depth_true[:H, :W] * (1 + rng.normal(0, 0.01, (H, W)))).astype(np.float32)
    act = np.ones((H, W), np.uint8)
    if case == "no_active":
        act[:] = 0
    elif case == "all_nan":
        depth[:] = np.nan
        depth[H // 2, W // 2] = sc.depth_true[H // 2, W // 2]
    elif case == "sparse":
        act = (rng.random((H, W)) < 0.2).astype(np.uint8)
        depth[rng.random((H, W)) < 0.3] = np.nan
    normal = S.tilted_normals(H, W, 3)
    zr = float(sc.ref_cam.C[2])
    args = (r, step, 2, 0.0, 0.02, 3, zr - 40.0, zr + 5.0, 2024)
    a = [depth.copy(), normal.copy(), np.zeros((H, W), np.float32)]
    b = [depth.copy(), normal.copy(), np.zeros((H, W), np.float32)]
    st = dense.stream_start(2024)
    ca = dense.pm_refine(ref, ray, sc.ref_cam.C, srcs, [None] * n_src, par, *a, act, *args, rng_state=st)
    ost = np.array([2024 | 1], np.uint32)
    cb = O.pm_refine(ref, ray, sc.ref_cam.C, srcs, [None] * n_src, par, *b, act, *args, state=ost)
    assert ca == cb
    for x, y in zip(a, b):
        assert same_bits(x, y)
    assert int(st.cpu().numpy().view(np.uint32)[0]) == int(ost[0])
    if case == "no_active":
        assert int(ost[0]) == 2024 | 1                 # nothing drew

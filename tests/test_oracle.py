"""The oracle (oracle/mvs_oracle.c + oracle/oracle.py) against the reference: bit for bit on the
golden fixtures made by the reference itself (tests/golden/make_golden.py), and against the
reference's compiled kernels live when oracle/_ref is built. CPU only."""
import numpy as np
import pytest

from conftest import golden, same_bits
from oracle import oracle as O


def test_oracle_sweep_matches_reference_fixtures(sweep_cases):
    for c in sweep_cases:
        H, W = c["H"], c["W"]
        best, prev, spb, snb, idx = O.init_state(H, W)
        for i, inv in enumerate(c["hyps"]):
            scores = None
            O.sweep_hypothesis(c["ref"], c["mu"], c["sd"], c["srcs"], c["ray"], c["geo"], inv, c["r"], c["top_k"], i,
                               best, prev, spb, snb, idx, scores)
            assert same_bits(prev, c["scores"][i]), (H, W, c["n"], i)
        for a, b in ((best, c["best"]), (prev, c["prev"]), (spb, c["spb"]), (snb, c["snb"]), (idx, c["idx"])):
            assert same_bits(a, b), (H, W, c["n"], c["r"])


def test_oracle_flat_images_keep_first_hypothesis(sweep_cases):
    c = sweep_cases[-1]                     # flat sources: scores tie wherever all samples are valid
    first_max = np.argmax(c["scores"], axis=0)   # argmax returns the first maximal index
    assert np.array_equal(c["idx"], first_max)
    ties = np.all(c["scores"] == c["scores"][0], axis=0)
    assert ties.mean() > 0.5 and np.all(c["idx"][ties] == 0)


def test_oracle_ref_stats_match_reference(sweep_cases):
    for c in sweep_cases:
        mu, sd = O.ref_stats(c["ref"], c["r"])
        assert same_bits(mu, c["mu"]) and same_bits(sd, c["sd"])


def test_oracle_sweep_end_to_end_matches_reference():
    z = golden("sweep_e2e.npz")
    H, W, n, r, top_k, nh = (int(v) for v in z["meta"])
    srcs = [z[f"src{j}"] for j in range(n)]
    out = O.sweep(z["ref"], srcs, z["ray"], z["geo"], list(z["hyps"]), r, top_k)
    assert same_bits(out["depth"], z["depth"])
    assert same_bits(out["best"], z["best"])
    assert same_bits(out["sd"], z["sd"])


def test_oracle_scene_sweep_matches_reference():
    z = golden("scene_small.npz")
    H, W, n, r, top_k, nh = (int(v) for v in z["meta"])
    grey = lambda u8: ((u8.astype(np.float32) - np.float32(128)) / np.float32(64)).astype(np.float32)
    ref = grey(z["ref_u8"])
    srcs = [grey(z[f"src{j}_u8"]) for j in range(n)]
    hyps = [np.full((H, W), p, np.float32) for p in z["planes"]]
    out = O.sweep(ref, srcs, z["ray"], z["geo"], hyps, r, top_k, keep_scores=True)
    assert same_bits(out["depth"], z["depth"])
    assert same_bits(out["best"], z["best"])
    srt = np.sort(out["scores"], axis=0)
    assert same_bits((srt[-1] - srt[-2]).astype(np.float32), z["gap"])
    # the synthetic scene is matchable: most pixels find the rendered depth within 1 %
    valid = np.isfinite(z["depth_true"])
    rel = np.abs(out["depth"] - z["depth_true"]) / z["depth_true"]
    assert np.median(rel[valid]) < 0.01


def test_oracle_helpers_match_reference():
    z = golden("helpers.npz")
    for r in (0, 1, 2, 5, 7):
        assert same_bits(O.box(z["box_in"], r), z[f"box_r{r}"]), r
        assert same_bits(O.box(np.ascontiguousarray(z["box_in"] * z["box_in"]), r), z[f"box_sq_r{r}"]), r

    class Cam:
        pass

    cam = Cam()
    row = z["rays_cam"]
    cam.R, cam.C = row[:9].reshape(3, 3), row[9:12]
    cam.f, cam.k1, cam.k2, cam.k3, cam.cx, cam.cy = row[12:]
    rays = O.rays_world((96, 128), cam)
    assert np.max(np.abs(rays - z["rays"])) <= 1e-7 * np.max(np.abs(z["rays"]))


def test_oracle_finalize_boundaries():
    # interior test, clip and the depth floor, in NumPy semantics (densify.py:354-361)
    best = np.array([[0.9, 0.9, 0.5, 0.2]], np.float32)
    spb = np.array([[0.8, 0.85, -2.0, 0.2]], np.float32)
    snb = np.array([[0.1, 0.88, 0.4, 0.2]], np.float32)
    idx = np.array([[3, 5, 0, 2]], np.int32)
    inv0 = np.full((1, 4), 0.02, np.float32)
    inv1 = np.full((1, 4), 0.021, np.float32)
    d = O.finalize(best, spb, snb, idx, inv0, inv1, 8)
    assert d.dtype == np.float32 and d.shape == (1, 4)
    assert abs(d[0, 2] - 1 / 0.02) < 1e-3           # idx 0: no parabola
    assert abs(d[0, 3] - 1 / 0.022) < 1e-3          # flat: den = 0 -> no offset


def test_oracle_pm_matches_reference_fixture():
    z = golden("pm_case.npz")
    r, step, top_k, iters, seed = (int(v) for v in z["args"])
    geo_w, geo_tol, dmin, dmax = (float(v) for v in z["fargs"])
    srcs = [z[f"src{j}"] for j in range(3)]
    sdeps = [None, z["sdep1"], None]
    depth, normal, score = z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()
    ch = O.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], depth, normal, score, z["active"], r, step,
                     top_k, geo_w, geo_tol, iters, dmin, dmax, seed)
    assert ch == int(z["changed"])
    assert same_bits(depth, z["depth"]) and same_bits(normal, z["normal"]) and same_bits(score, z["score"])


def test_oracle_pm_matches_reference_rendered_8_sources():
    """The oracle against the reference's own pm_refine on a rendered 8-source scene (7 x 7, 2
    iterations, 1 % holes, 80 % active)."""
    z = golden("pm_case8.npz")
    r, step, top_k, iters, seed = (int(v) for v in z["args"])
    geo_w, geo_tol, dmin, dmax = (float(v) for v in z["fargs"])
    grey = lambda u8: ((u8.astype(np.float32) - np.float32(128)) / np.float32(64)).astype(np.float32)
    srcs = [grey(u) for u in z["src_u8"]]
    st = [z["depth0"].copy(), z["normal0"].copy(), np.zeros(z["depth0"].shape, np.float32)]
    ch = O.pm_refine(grey(z["ref_u8"]), z["ray"], z["Cr"], srcs, [None] * len(srcs), z["par"], *st, z["active"], r,
                     step, top_k, geo_w, geo_tol, iters, dmin, dmax, seed)
    assert ch == int(z["changed"])
    for a, b in zip(st, (z["depth"], z["normal"], z["score"])):
        assert same_bits(a, b)


def test_oracle_pm_stream_carries_across_calls():
    """Iterations split over calls, with the stream state carried, equal one call (the resumable
    form the device takes with mvs_pm_args.rng_state)."""
    z = golden("pm_case.npz")
    r, step, top_k, iters, seed = (int(v) for v in z["args"])
    geo_w, geo_tol, dmin, dmax = (float(v) for v in z["fargs"])
    srcs = [z[f"src{j}"] for j in range(3)]
    sdeps = [None, z["sdep1"], None]
    one = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    c1 = O.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *one, z["active"], r, step, top_k, geo_w,
                     geo_tol, 3, dmin, dmax, seed)
    two = [z["depth0"].copy(), z["normal0"].copy(), z["score0"].copy()]
    st = np.array([seed | 1], np.uint32)
    c2 = sum(O.pm_refine(z["ref"], z["ray"], z["Cr"], srcs, sdeps, z["par"], *two, z["active"], r, step, top_k,
                         geo_w, geo_tol, 1, dmin, dmax, seed, it0=it, state=st) for it in range(3))
    assert c1 == c2 > 0
    assert all(same_bits(a, b) for a, b in zip(one, two))


def test_oracle_fp64_agrees_with_float32_where_decided():
    z = golden("scene_small.npz")
    H, W, n, r, top_k, nh = (int(v) for v in z["meta"])
    grey = lambda u8: ((u8.astype(np.float32) - np.float32(128)) / np.float32(64)).astype(np.float32)
    ref = grey(z["ref_u8"])
    srcs = [grey(z[f"src{j}_u8"]) for j in range(n)]
    hyps = [np.full((H, W), p, np.float64) for p in z["planes"]]
    d64, b64, i64 = O.sweep_fp64(ref, srcs, z["ray"], z["geo"], hyps, r, top_k)
    decided = z["gap"] > 1e-3
    rel = np.abs(d64 - z["depth"]) / d64
    assert np.median(rel[decided]) < 1e-5
    assert np.mean(rel[decided] < 1e-3) > 0.99


def test_oracle_matches_live_reference_kernels():
    R = O.reference()
    if R is None:
        pytest.skip("oracle/_ref not built (the reference sources are not present on this machine)")
    from tests_support import random_sweep_case
    rng = np.random.default_rng(101)
    for (H, W, n, r, top_k, nh) in [(23, 29, 3, 2, 2, 4), (17, 40, 6, 4, 3, 5), (31, 12, 2, 0, 1, 3)]:
        ref, srcs, ray, geo, hyps = random_sweep_case(rng, H, W, n, nh)
        mu, sd = O.ref_stats(ref, r)
        s1, s2 = O.init_state(H, W), O.init_state(H, W)
        for i, inv in enumerate(hyps):
            O.sweep_hypothesis(ref, mu, sd, srcs, ray, geo, inv, r, top_k, i, *s1)
            R._dense.sweep_hypothesis(ref, mu, sd, srcs, ray, geo, np.ascontiguousarray(inv), r, top_k, i, *s2)
        assert all(same_bits(a, b) for a, b in zip(s1, s2))

"""bench.py --check, the band validation of the cpu_baseline leg, on the CPU: given the oracle's
own full-image sweep for a row band it passes (the band's strips with their halo reproduce the
full-image result), and a decided pixel planted with another winner index makes it fail."""
import numpy as np

from oracle import oracle as O


def _case():
    from py_ortho_b200 import scene as S
    sc = S.make_scene("c1", seed=3, width=160, height=96)
    ref = sc.grey(sc.ref)
    srcs = [sc.grey(s) for s in sc.srcs]
    geo = S.geo_rows(sc.ref_cam, sc.src_cams)
    planes = S.plane_list(35.0, 55.0, 12)
    return sc, ref, srcs, geo, planes


def test_band_check_passes_on_the_oracle_result_and_catches_a_planted_flip():
    import bench
    sc, ref, srcs, geo, planes = _case()
    H, W = ref.shape
    r, top_k, y0, y1 = 2, 2, 40, 60
    ray = O.rays_world((H, W), sc.ref_cam)
    full = O.sweep(ref, srcs, ray, geo, [np.full((H, W), p, np.float32) for p in planes], r, top_k, keep_scores=True)
    mu, sd = O.ref_stats(ref, r)
    band = (y0, y1, full["idx"][y0:y1].copy(), full["best"][y0:y1].astype(np.float32), full["depth"][y0:y1].copy(),
            mu[y0 - r:y1 + r], sd[y0 - r:y1 + r])
    out = bench.reference_band_check(sc, ref, srcs, geo, planes, r, top_k, band)
    assert out["pass"], out
    assert out["decided_missed"] == 0 and out["flips"] == 0 and out["depth_rel_max_kept"] == 0.0
    assert out["decided"] > 0.3 * (y1 - y0) * W
    # the planted mistake (in the checked result, on the CPU): one decided pixel's winner moved
    scores = np.sort(np.stack(full["scores"]), axis=0)
    gap = (scores[-1] - scores[-2])[y0:y1]
    yy, xx = np.argwhere(gap > 1e-3)[0]
    idx = band[2].copy()
    idx[yy, xx] = (idx[yy, xx] + 3) % len(planes)
    out2 = bench.reference_band_check(sc, ref, srcs, geo, planes, r, top_k, (y0, y1, idx) + band[3:])
    assert not out2["pass"] and out2["decided_missed"] == 1


def test_check_needs_the_cpu_baseline_leg():
    """--check runs inside the cpu_baseline leg, so the bench refuses it together with --no-cpu
    (an argument error, before any device work)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--check", "--no-cpu"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 2
    assert "--check runs in the cpu_baseline leg" in r.stderr

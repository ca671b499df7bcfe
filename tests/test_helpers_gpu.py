"""The per-view helpers on the device, bit for bit against the reference's golden outputs."""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu


def test_box_zero_mean_bit_exact():
    from py_ortho_b200 import fast
    z = golden("helpers.npz")
    for r in (0, 1, 2, 5, 7):
        assert same_bits(fast.box_zero_mean(z["box_in"], r), z[f"box_r{r}"]), r
        assert same_bits(fast.box_zero_mean(np.ascontiguousarray(z["box_in"] * z["box_in"]), r), z[f"box_sq_r{r}"]), r
    with pytest.raises(ValueError):
        fast.box_zero_mean(z["box_in"], -1)


def test_ref_stats_bit_exact(sweep_cases):
    from py_ortho_b200 import fast
    for c in sweep_cases:
        mu, sd = fast.ref_stats(c["ref"], c["r"])
        assert same_bits(mu, c["mu"]) and same_bits(sd, c["sd"])


def test_hypothesis_maps_bit_exact():
    from py_ortho_b200 import fast
    z = golden("helpers.npz")
    for i in (0, 1, 7, 191):
        assert same_bits(fast.hyp_linear(z["hyp_base"], z["hyp_step"], i), z[f"hyp_linear_{i}"])
    for t in (-3, -1, 0, 2, 3):
        assert same_bits(fast.hyp_refine(z["hyp_iu"], z["hyp_step"], t), z[f"hyp_refine_{t + 3}"])


def test_depth_view_bit_exact():
    from py_ortho_b200 import fast
    z = golden("helpers.npz")
    g, r8 = fast.depth_view(z["dv_rgb"], z["dv_gain"], z["dv_bias"], z["dv_mask"])
    assert same_bits(g, z["dv_grey"]) and same_bits(r8, z["dv_rgb8"])
    g0, r0 = fast.depth_view(z["dv_rgb"])
    assert same_bits(g0, z["dv_grey0"]) and same_bits(r0, z["dv_rgb80"])


def test_rays_and_pyramid():
    from py_ortho_b200 import fast

    class Cam:
        pass

    z = golden("helpers.npz")
    row = z["rays_cam"]
    cam = Cam()
    cam.R, cam.C = row[:9].reshape(3, 3), row[9:12]
    cam.f, cam.k1, cam.k2, cam.k3, cam.cx, cam.cy = row[12:]
    rays = fast.rays_world((96, 128), cam, host=True)
    ulp = np.abs(rays.view(np.int32).astype(np.int64) - z["rays"].view(np.int32).astype(np.int64))
    assert ulp.max() <= 1 and (ulp == 0).mean() > 0.99
    assert same_bits(fast.half(z["half_in"]), z["half_out"])
    assert same_bits(fast.half(z["half_in"][0]), z["half_out"][0])

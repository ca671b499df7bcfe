"""Legacy height sweep (mvs.py) on the host side: the oracle's sampler, float64 box mean and SGM
against the reference's own kernels (height_case.npz, recorded from _mvs.sample_view,
_fast.box_sat_mean and _mvs.sgm), bit for bit. CPU only."""
import numpy as np

from conftest import golden, same_bits
from oracle import oracle as O


def _sv_args(z):
    f, k1, k2, k3, cx, cy = (float(v) for v in z["sv_cam"])
    X0, Y0, gsd = (float(v) for v in z["sv_grid"])
    return (z["sv_R"], z["sv_C"], f, k1, k2, k3, cx, cy), X0, Y0, gsd


def test_oracle_sample_view_matches_the_reference():
    z = golden("height_case.npz")
    cam, X0, Y0, gsd = _sv_args(z)
    out, valid = O.sample_view(z["sv_img"], cam, X0, Y0, gsd, z["sv_Z"])
    assert np.array_equal(valid, z["sv_valid"]) and 0 < valid.mean() < 1
    assert same_bits(out, z["sv_out"])


def test_oracle_box_sat_mean_matches_the_reference():
    z = golden("height_case.npz")
    assert same_bits(O.box_sat_mean(z["box_in"], int(z["box_r"])), z["box_out"])


def test_oracle_sgm_matches_the_reference():
    z = golden("height_case.npz")
    p1, p2 = (float(v) for v in z["sgm_p"])
    assert same_bits(O.sgm(z["sgm_cost"], np.float32(p1), np.float32(p2)), z["sgm_out"])

"""Legacy height sweep (mvs.py) on the device against the reference (height_case.npz): the sampler,
the float64 box mean and the 8-path SGM bit for bit; mvs.dense_reconstruct end to end (the
reference ran on its CPU backend) within the tolerance that the order of the top-k NCC sum
(np.partition's order there, descending here) and float32 powers leave."""
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_sample_view_bit_exact():
    from py_ortho_b200 import height as Hs
    from test_height import _sv_args
    z = golden("height_case.npz")
    cam, X0, Y0, gsd = _sv_args(z)
    out, valid = Hs.sample_view(_t(z["sv_img"]), cam, X0, Y0, gsd, _t(z["sv_Z"]))
    assert np.array_equal(valid.cpu().numpy(), z["sv_valid"])
    assert same_bits(out.cpu().numpy(), z["sv_out"])


def test_box_sat_mean_bit_exact():
    from py_ortho_b200 import height as Hs
    z = golden("height_case.npz")
    assert same_bits(Hs.box(_t(z["box_in"]), int(z["box_r"])).cpu().numpy(), z["box_out"])


def test_sgm_bit_exact():
    from py_ortho_b200 import height as Hs
    z = golden("height_case.npz")
    p1, p2 = (float(v) for v in z["sgm_p"])
    assert same_bits(Hs.sgm(_t(z["sgm_cost"]), np.float32(p1), np.float32(p2)).cpu().numpy(), z["sgm_out"])


def test_dense_reconstruct_matches_the_reference():
    from py_ortho_b200 import height as Hs
    z = golden("height_case.npz")
    f, cx, cy, W, H = z["h_intr"]
    W, H = int(W), int(H)
    n = len(z["h_C"])
    intr = [SimpleNamespace(f=float(f), cx=float(cx), cy=float(cy), width=W, height=H, k1=0.0, k2=0.0, k3=0.0)]
    rec = SimpleNamespace(used=list(range(n)), intr=intr, cam_group=np.zeros(n, np.int32), X=z["h_X"], C=z["h_C"],
                          R=z["h_R"])
    frames = [SimpleNamespace(width=W, height=H, path=f"view{k}") for k in range(n)]
    imgs = {f"view{k}": np.repeat(z[f"h_img{k}"][:, :, None], 3, axis=2) for k in range(n)}
    tile, overlap, levels = (int(v) for v in z["h_opt"])
    opt = Hs.DenseOptions(tile=tile, overlap=overlap, levels=levels, workers=1)
    r = Hs.dense_reconstruct(SimpleNamespace(frames=frames, workers=1), rec, {}, float(z["h_native"]), opt,
                             load_rgb=lambda fr, s: imgs[fr.path])
    assert np.allclose([r.minX, r.maxY, r.gsd], z["h_grid"])
    assert r.Z.shape == z["h_Z"].shape
    assert np.array_equal(np.isfinite(r.Z), np.isfinite(z["h_Z"]))
    assert np.array_equal(r.covered, z["h_covered"])
    fin = np.isfinite(r.Z)
    dz = np.abs(r.Z[fin] - z["h_Z"][fin])
    same = (dz <= 1e-4).mean()
    ds = np.abs(r.score - z["h_score"])
    print(f"height sweep: Z identical within 1e-4 m on {same:.2%} of cells, max |dZ| {dz.max():.3f} m; "
          f"score |d| median {np.median(ds):.1e}, rgb max |d| {np.abs(r.rgb.astype(int) - z['h_rgb']).max()}")
    assert same >= 0.99
    assert np.median(ds) <= 1e-6

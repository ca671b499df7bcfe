"""The depth_map driver (3-level pyramid, tie-point band, coarse sweep + two refinement levels)
on the device against the reference's own densify.depth_map output (golden fixture)."""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu


def test_depth_map_matches_reference():
    from types import SimpleNamespace
    from py_ortho_b200 import densify as Dn
    z = golden("depth_map.npz")
    f, cx, cy, w, h = z["intr"]
    rec = SimpleNamespace(intr=[SimpleNamespace(f=f, cx=cx, cy=cy, width=int(w), height=int(h))],
                          cam_group=np.zeros(len(z["C"]), np.int32), X=z["X"], C=z["C"], R=z["R"],
                          obs_cam=z["obs_cam"], obs_pt=z["obs_pt"])
    greys = [((z[f"img{k}"].astype(np.float32) - np.float32(128)) / np.float32(64)).astype(np.float32)
             for k in range(len(z["C"]))]

    def views(k):
        return greys[k], None, Dn._Cam(z["R"][k], z["C"][k], float(f), 0.0, 0.0, float(cx), float(cy), int(w), int(h))

    opt = Dn.DepthOptions()
    opt.window, opt.num_depths = int(z["opt"][0]), int(z["opt"][1])
    depth, score, low = Dn.depth_map(0, [1, 2, 3, 4], rec, views, opt)
    assert same_bits(low, z["low"])                          # window deviation is bit-exact
    fin, rfin = np.isfinite(depth), np.isfinite(z["depth"])
    assert (fin == rfin).mean() > 0.995
    both = fin & rfin
    rel = np.abs(depth[both].astype(np.float64) - z["depth"][both]) / z["depth"][both]
    assert np.median(rel) < 1e-5
    assert (rel <= 1e-3).mean() > 0.99                      # coarse-to-fine near-ties may move a few
    assert np.median(np.abs(score[both] - z["score"][both])) < 1e-5


def test_depth_map_tie_point_geometry_matches_reference():
    """The driver's tie-point priors on the device (mvs_tie_depths for the depth range,
    mvs_depth_band for the per-pixel band and its linear hypothesis maps) and the hypothesis count
    give the reference's values on the depth_map fixture, bit for bit."""
    from types import SimpleNamespace
    from py_ortho_b200 import densify as Dn
    z = golden("depth_map.npz")
    f, cx, cy, w, h = z["intr"]
    rec = SimpleNamespace(intr=[SimpleNamespace(f=f, cx=cx, cy=cy, width=int(w), height=int(h))],
                          cam_group=np.zeros(len(z["C"]), np.int32), X=z["X"], C=z["C"], R=z["R"],
                          obs_cam=z["obs_cam"], obs_pt=z["obs_pt"])
    rng = Dn._depth_range(rec, 0)
    assert np.array_equal(np.array(rng), z["range"])
    cam = Dn._Cam(z["R"][0], z["C"][0], float(f), 0.0, 0.0, float(cx), float(cy), int(w), int(h))
    cam2 = cam.scaled(0.5, 160, 120).scaled(0.5, 80, 60)
    nd = Dn._num_depths(rec, 0, [1, 2, 3, 4], rng, cam2.f, int(z["opt"][1]))
    assert nd == int(z["nd"])
    base, step, inv_hi = (t.cpu().numpy() for t in Dn._band_maps(rec, 0, cam2, (60, 80), rng, nd,
                                                                  block=max(8, 80 // 16)))
    assert same_bits(base, z["band_lo"]) and same_bits(inv_hi, z["band_hi"])
    want = ((z["band_hi"] - z["band_lo"]) / max(nd - 1, 1)).astype(np.float32)
    assert same_bits(step, want)
    # fewer observed points than the band needs: the view's whole range everywhere
    few = SimpleNamespace(**vars(rec))
    few.obs_cam = rec.obs_cam.copy()
    few.obs_cam[np.flatnonzero(few.obs_cam == 0)[40:]] = -1
    b2, s2, h2 = (t.cpu().numpy() for t in Dn._band_maps(few, 0, cam2, (60, 80), rng, nd, block=8))
    assert (b2 == np.float32(1.0 / rng[1])).all() and (h2 == np.float32(1.0 / rng[0])).all()

"""The synthetic scene generator (CPU): determinism, geometry of the configurations."""
import numpy as np

from py_ortho_b200 import scene as S


def test_scene_is_seeded_and_deterministic():
    a = S.make_scene("c1", seed=4, width=64, height=48)
    b = S.make_scene("c1", seed=4, width=64, height=48)
    c = S.make_scene("c1", seed=5, width=64, height=48)
    assert np.array_equal(a.ref, b.ref) and all(np.array_equal(x, y) for x, y in zip(a.srcs, b.srcs))
    assert not np.array_equal(a.ref, c.ref)
    assert a.ref.dtype == np.uint8 and a.ref.shape == (48, 64) and len(a.srcs) == 4
    assert 20 < a.ref.std() < 80


def test_configuration_geometry():
    c1, c2 = S.CONFIGS["c1"], S.CONFIGS["c2"]
    assert (c1.width, c1.height, c1.sources, c1.planes, c1.radius) == (640, 480, 4, 128, 2)
    assert (c2.width, c2.height, c2.sources, c2.planes, c2.radius, c2.pm_iters) == (4000, 3000, 8, 256, 3, 4)
    offs = S.source_offsets(c1)
    assert np.isclose(offs[0][0], 0.2 * 640 * 50 / 600) and np.isclose(offs[2][1], 0.3 * 480 * 50 / 600)
    assert len(S.source_offsets(c2)) == 8
    p = S.plane_list(35.0, 55.0, 128)
    assert p.dtype == np.float32 and np.isclose(1 / p[0], 55.0) and np.isclose(1 / p[-1], 35.0)
    assert np.all(np.diff(p) > 0)


def test_rendered_depth_is_inside_the_sweep_range():
    sc = S.make_scene("c1", seed=0, width=80, height=60)
    near, far = S.CONFIGS["c1"].depth_range
    assert near < sc.depth_true.min() and sc.depth_true.max() < far


def test_tilted_normals_are_unit_and_within_the_cone():
    n = S.tilted_normals(20, 30, 1, 30.0)
    assert np.allclose(np.linalg.norm(n, axis=0), 1, atol=1e-6)
    assert np.degrees(np.arccos(n[2])).max() <= 30.0 + 1e-4

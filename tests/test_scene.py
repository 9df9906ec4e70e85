"""Seeded scene generator and Bevy-convention matrices."""
import math

import numpy as np

from bevy_strand_rasterizer_b200.plugin import pack_strand_set, pack_strands
from bevy_strand_rasterizer_b200.scene import CameraSpec, LightSpec, scalp_hair, workload


def test_generator_is_seeded_and_shaped():
    a = scalp_hair(100, 16, seed=3)
    b = scalp_hair(100, 16, seed=3)
    assert np.array_equal(a.vertices, b.vertices)
    assert a.n_strands == 100 and a.n_points == 1600 and a.n_segments == 1500
    roots = a.vertices[::16]
    assert np.allclose(np.linalg.norm(roots, axis=1), 0.1, atol=1e-6)
    assert np.all(roots[:, 1] >= -1e-6)  # upper hemisphere
    lengths = np.linalg.norm(np.diff(a.vertices.reshape(100, 16, 3), axis=1), axis=2).sum(1)
    assert np.all(lengths > 0.14) and np.all(lengths < 0.40)
    c = scalp_hair(50, 32, seed=4, curly=True)
    assert c.vertices.shape == (1600, 3) and np.isfinite(c.vertices).all()


def test_camera_is_reverse_z_infinite():
    cam = CameraSpec(eye=(0.0, 0.0, 0.6), width=1920, height=1080)
    m = cam.clip_from_world().reshape(4, 4).T.astype(np.float64)
    origin = m @ np.array([0.0, 0.0, 0.0, 1.0])
    ndc = origin[:3] / origin[3]
    assert abs(ndc[0]) < 1e-6 and abs(ndc[1]) < 1e-6
    assert abs(ndc[2] - 0.1 / 0.6) < 1e-6  # near / distance
    near = m @ np.array([0.0, 0.0, 0.5, 1.0])
    assert abs(near[2] / near[3] - 1.0) < 1e-6


def test_light_is_orthographic_reverse_z():
    lo, hi = np.array([-0.3, -0.4, -0.3]), np.array([0.3, 0.2, 0.3])
    m = LightSpec((1.0, 1.0, 1.0)).clip_from_world(lo, hi).reshape(4, 4).T.astype(np.float64)
    corners = np.array([[x, y, z, 1.0] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    c = corners @ m.T
    assert np.allclose(c[:, 3], 1.0)
    assert np.all(np.abs(c[:, :2]) < 1.0) and np.all((c[:, 2] > 0.0) & (c[:, 2] < 1.0))
    toward = np.array([0.1, 0.1, 0.1, 1.0]) @ m.T
    away = np.array([-0.1, -0.1, -0.1, 1.0]) @ m.T
    assert toward[2] > away[2]  # larger depth = nearer the light


def test_pack_strands_drops_short_strands():
    v = np.arange(30, dtype=np.float32).reshape(10, 3)
    p = pack_strands(v, [[0, 1, 2], [3], [4, 5], [6, 7, 8, 9]])
    assert p.strand_count == 3 and p.meta["count"].tolist() == [3, 2, 4]
    assert p.meta["offset"].tolist() == [0, 3, 5] and p.max_segments_in_strand == 4
    assert p.vertices.shape == (10, 4)
    w = workload("small")
    assert w.segments == 150_000 and w.width == 1280
    assert pack_strand_set(scalp_hair(10, 4, 1)).index_count == 40

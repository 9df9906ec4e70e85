"""Seeded synthetic strand scenes, Bevy-convention cameras and lights.

Scalp hair: roots uniform by area on the upper hemisphere (+Y) of a 0.1 m
sphere at the origin, strands grown along the surface normal with length
U[0.15, 0.30] m, drooping toward -Y by 0.5 rad accumulated linearly along the
strand, N(0, 1 mm) jitter per point except the root; the curly variant winds a
helix (radius U[2, 6] mm, pitch U[8, 20] mm) around the drooped spine.

Cameras follow Bevy 0.19: Transform::looking_at for the view and
Mat4::perspective_infinite_reverse_rh for the projection (reverse-Z, infinite
far plane, near 0.1). Directional lights use one orthographic reverse-Z
frustum fitted to the scene's bounding box (larger depth = nearer the light,
the convention strand_rasterizer.wgsl:371-377 expects).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


# ---------------------------------------------------------------------------
# Matrices (column-major float32[16], glam layout)
# ---------------------------------------------------------------------------
def looking_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """world_from_view of Transform::from_translation(eye).looking_at(target, up)."""
    eye = np.asarray(eye, np.float64)
    back = eye - np.asarray(target, np.float64)
    back /= np.linalg.norm(back)
    up = np.asarray(up, np.float64)
    if abs(np.dot(up, back)) > 0.999:
        up = np.array([0.0, 0.0, 1.0])
    right = np.cross(up, back)
    right /= np.linalg.norm(right)
    up2 = np.cross(back, right)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = right, up2, back, eye
    return m


def perspective_infinite_reverse_rh(fov_y: float, aspect: float, near: float) -> np.ndarray:
    f = 1.0 / math.tan(0.5 * fov_y)
    m = np.zeros((4, 4))
    m[0, 0] = f / aspect
    m[1, 1] = f
    m[3, 2] = -1.0
    m[2, 3] = near
    return m


def orthographic_reverse_z(l, r, b, t, near, far) -> np.ndarray:
    """x, y -> [-1, 1]; view depth -near -> 1, -far -> 0."""
    m = np.zeros((4, 4))
    m[0, 0] = 2.0 / (r - l)
    m[1, 1] = 2.0 / (t - b)
    m[2, 2] = 1.0 / (far - near)
    m[0, 3] = -(r + l) / (r - l)
    m[1, 3] = -(t + b) / (t - b)
    m[2, 3] = far / (far - near)
    m[3, 3] = 1.0
    return m


def to_cols(m: np.ndarray) -> np.ndarray:
    """4x4 row-major math matrix -> column-major float32[16]."""
    return np.ascontiguousarray(m.T.reshape(16).astype(np.float32))


@dataclass
class CameraSpec:
    eye: tuple
    target: tuple = (0.0, 0.0, 0.0)
    fov_y_deg: float = 45.0
    near: float = 0.1
    width: int = 1920
    height: int = 1080

    def clip_from_world(self) -> np.ndarray:
        view = np.linalg.inv(looking_at(self.eye, self.target))
        proj = perspective_infinite_reverse_rh(math.radians(self.fov_y_deg), self.width / self.height, self.near)
        return to_cols(proj @ view)


@dataclass
class LightSpec:
    direction_to_light: tuple
    illuminance: float = 10_000.0  # DirectionalLight default, lux
    color: tuple = (1.0, 1.0, 1.0)
    size: int = 2048

    def clip_from_world(self, aabb_min, aabb_max) -> np.ndarray:
        d = np.asarray(self.direction_to_light, np.float64)
        d /= np.linalg.norm(d)
        lo, hi = np.asarray(aabb_min, np.float64), np.asarray(aabb_max, np.float64)
        center = 0.5 * (lo + hi)
        radius = 0.5 * np.linalg.norm(hi - lo) + 1e-3
        view = np.linalg.inv(looking_at(center + d * (2.0 * radius), center))
        corners = np.array([[x, y, z, 1.0] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
        v = corners @ view.T
        l, r = v[:, 0].min(), v[:, 0].max()
        b, t = v[:, 1].min(), v[:, 1].max()
        near, far = -v[:, 2].max(), -v[:, 2].min()
        pad = 0.02 * max(r - l, t - b, far - near)
        proj = orthographic_reverse_z(l - pad, r + pad, b - pad, t + pad, max(near - pad, 1e-4), far + pad)
        return to_cols(proj @ view)

    def color4(self) -> np.ndarray:
        c = np.asarray(self.color, np.float32) * np.float32(self.illuminance)
        return np.array([c[0], c[1], c[2], self.illuminance], np.float32)

    def direction(self) -> np.ndarray:
        d = np.asarray(self.direction_to_light, np.float64)
        return (d / np.linalg.norm(d)).astype(np.float32)


# ---------------------------------------------------------------------------
# Strand generation
# ---------------------------------------------------------------------------
@dataclass
class StrandSet:
    """Polylines in the StrandList layout: vertices + per-strand vertex indices."""
    vertices: np.ndarray           # (P, 3) float32
    strand_counts: np.ndarray      # (S,) uint32
    strand_offsets: np.ndarray     # (S,) uint32 into indices
    indices: np.ndarray            # (P,) uint32

    @property
    def n_strands(self) -> int:
        return int(self.strand_counts.shape[0])

    @property
    def n_points(self) -> int:
        return int(self.indices.shape[0])

    @property
    def n_segments(self) -> int:
        c = self.strand_counts.astype(np.int64)
        return int(np.maximum(c - 1, 0)[c >= 2].sum())


def scalp_hair(n_strands: int, n_points: int, seed: int, curly: bool = False) -> StrandSet:
    rng = np.random.default_rng(seed)
    y = rng.uniform(0.0, 1.0, n_strands)
    phi = rng.uniform(0.0, 2.0 * math.pi, n_strands)
    rxz = np.sqrt(np.maximum(0.0, 1.0 - y * y))
    normal = np.stack([rxz * np.cos(phi), y, rxz * np.sin(phi)], axis=1)
    root = 0.1 * normal
    length = rng.uniform(0.15, 0.30, n_strands)
    down = np.array([0.0, -1.0, 0.0])
    perp = down[None, :] - (normal @ down)[:, None] * normal
    pn = np.linalg.norm(perp, axis=1)
    fallback = np.tile([1.0, 0.0, 0.0], (n_strands, 1))
    perp = np.where(pn[:, None] > 1e-6, perp / np.maximum(pn, 1e-12)[:, None], fallback)
    k = np.arange(n_points, dtype=np.float64)
    step = length / max(n_points - 1, 1)
    # direction of segment k at the segment midpoint: bend 0.5 rad accumulated linearly
    s_mid = (np.arange(max(n_points - 1, 1)) + 0.5) / max(n_points - 1, 1)
    ang = 0.5 * s_mid
    dirs = (np.cos(ang)[None, :, None] * normal[:, None, :] + np.sin(ang)[None, :, None] * perp[:, None, :])
    seg = dirs * step[:, None, None]
    pos = np.concatenate([root[:, None, :], root[:, None, :] + np.cumsum(seg, axis=1)], axis=1)[:, :n_points]
    if curly:
        radius = rng.uniform(0.002, 0.006, n_strands)
        pitch = rng.uniform(0.008, 0.020, n_strands)
        phase0 = rng.uniform(0.0, 2.0 * math.pi, n_strands)
        b2 = np.cross(normal, perp)
        arc = k[None, :] * step[:, None]
        ph = 2.0 * math.pi * arc / pitch[:, None] + phase0[:, None]
        ramp = np.minimum(1.0, arc / pitch[:, None])
        off = (radius[:, None] * ramp)[:, :, None] * (np.cos(ph)[:, :, None] * perp[:, None, :] +
                                                      np.sin(ph)[:, :, None] * b2[:, None, :])
        pos = pos + off
    jitter = rng.normal(0.0, 0.001, pos.shape)
    jitter[:, 0, :] = 0.0
    pos = pos + jitter
    vertices = pos.reshape(-1, 3).astype(np.float32)
    counts = np.full(n_strands, n_points, np.uint32)
    offsets = (np.arange(n_strands, dtype=np.uint64) * n_points).astype(np.uint32)
    indices = np.arange(n_strands * n_points, dtype=np.uint32)
    return StrandSet(vertices, counts, offsets, indices)


# ---------------------------------------------------------------------------
# Benchmark workloads (sizes of the plain-pipeline configurations)
# ---------------------------------------------------------------------------
@dataclass
class Workload:
    name: str
    strands: int
    points: int
    width: int
    height: int
    dom_size: int
    dom_layers: int
    lights: list = field(default_factory=list)
    curly: bool = False
    seed: int = 1
    depth_slices: int = 64
    froxel: int = 8
    orbit_frames: int = 200
    # Fine-reference capacity = factor x binning capacity (the reference's default is 4).
    # At 4K a curly scene's segments cross more cells than that holds.
    ref_capacity_factor: int = 4

    def camera(self, frame: int = 0) -> CameraSpec:
        theta = 2.0 * math.pi * (frame % self.orbit_frames) / self.orbit_frames
        return CameraSpec(eye=(0.6 * math.sin(theta), 0.0, 0.6 * math.cos(theta)), width=self.width,
                          height=self.height)

    @property
    def segments(self) -> int:
        return self.strands * (self.points - 1)


def workload(name: str) -> Workload:
    l1 = (1.0, 1.0, 1.0)
    l2 = (-1.0, 1.0, 0.5)
    if name == "tiny":
        return Workload("tiny", 300, 8, 160, 120, 128, 4, [l1], seed=7, depth_slices=16)
    if name == "small":
        return Workload("small", 10_000, 16, 1280, 720, 1024, 4, [l1], seed=11, depth_slices=32)
    if name == "medium":
        return Workload("medium", 100_000, 32, 1920, 1080, 2048, 8, [l1], seed=12, depth_slices=64)
    if name == "large":
        return Workload("large", 500_000, 32, 3840, 2160, 4096, 8, [l1, l2], curly=True, seed=13, depth_slices=64,
                        ref_capacity_factor=8)
    raise KeyError(name)

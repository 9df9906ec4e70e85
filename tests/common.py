"""Shared scene setup for the parity tests: the GPU plugin and the oracle get
byte-identical inputs (same packed slabs, same camera / light matrices)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from bevy_strand_rasterizer_b200 import abi
from bevy_strand_rasterizer_b200.plugin import FroxelConfig, StrandMaterial, pack_strand_set
from bevy_strand_rasterizer_b200.scene import LightSpec, scalp_hair, workload


@dataclass
class Scene:
    assets: list            # (packed, material, world_from_local)
    camera_cfg: FroxelConfig
    cam: abi.Camera
    light_cfgs: list
    lights_c: object
    settings: abi.Settings


def build_scene(name="tiny", frame=0, strands=None, points=None, width=None, height=None, dom=None, layers=None,
                lights=None, material: StrandMaterial | None = None, cull=True, illuminance=10_000.0,
                settings_overrides=None, curly=None, seed=None) -> Scene:
    w = workload(name)
    strands = strands or w.strands
    points = points or w.points
    width = width or w.width
    height = height or w.height
    dom = dom or w.dom_size
    layers = layers or w.dom_layers
    light_dirs = lights if lights is not None else w.lights
    s = scalp_hair(strands, points, seed if seed is not None else w.seed, curly=w.curly if curly is None else curly)
    packed = pack_strand_set(s)
    material = material or StrandMaterial()
    ident = np.eye(4, dtype=np.float32).reshape(16)
    assets = [(packed, material, ident)]
    cam_spec = w.camera(frame)
    cam_spec.width, cam_spec.height = width, height
    camera_cfg = FroxelConfig(width, height, w.froxel, w.froxel, w.depth_slices)
    cam = abi.Camera()
    cam.clip_from_world[:] = [float(x) for x in cam_spec.clip_from_world()]
    cam.world_position[:] = [float(x) for x in cam_spec.eye]
    lo, hi = packed.aabb_min, packed.aabb_max
    light_cfgs = [FroxelConfig(dom, dom, w.froxel, w.froxel, w.depth_slices) for _ in light_dirs]
    lights_c = (abi.Light * max(1, len(light_dirs)))()
    for i, d in enumerate(light_dirs):
        spec = LightSpec(d, illuminance=illuminance, size=dom)
        lights_c[i].clip_from_world[:] = [float(x) for x in spec.clip_from_world(lo, hi)]
        lights_c[i].direction_to_light[:] = [float(x) for x in spec.direction()]
        lights_c[i].color[:] = [float(x) for x in spec.color4()]
    st = abi.default_settings()
    st.dom_slices = layers
    st.stochastic_cull_enabled = 1 if cull else 0
    for k, v in (settings_overrides or {}).items():
        setattr(st, k, v)
    return Scene(assets, camera_cfg, cam, light_cfgs, lights_c, st)


def run_gpu(scene: Scene, plugin=None, fused=False, stream=None, scene_color=None, out=None, scene_depth=None,
            opaque_depth=None, opaque_samples=1):
    from bevy_strand_rasterizer_b200.plugin import StrandRasterizerPlugin
    if plugin is None:
        plugin = StrandRasterizerPlugin()
        abi.check(plugin.lib.fiber_settings_set(plugin.ctx, C.byref(scene.settings)), "fiber_settings_set")
        for packed, material, w in scene.assets:
            plugin.add_geometry(packed, material, w)
    plugin.frame_begin_raw(scene.camera_cfg, scene.cam, scene.light_cfgs, scene.lights_c, stream)
    if fused:
        plugin.frame_fused(scene_color, scene_depth, out, stream)
    else:
        plugin.render_nodes(scene_color, scene_depth, out, stream, opaque_samples=opaque_samples,
                            opaque_depth=opaque_depth)
    return plugin


def run_ref(scene: Scene, **kw):
    from oracle_bridge import run_oracle
    return run_oracle(scene.assets, scene.camera_cfg, scene.cam, scene.light_cfgs, scene.lights_c, scene.settings,
                      **kw)


def opaque_plane(width: int, height: int, level: float, samples: int = 1, seed: int = 0) -> np.ndarray:
    """A seeded opaque depth image (H, W, samples), reversed-Z: a wall at
    `level` over the left 60% of the screen, a ramp from 0 to 2*level across
    the bottom quarter, nothing elsewhere. With several samples one sample in
    ~3% of the wall's pixels is left empty, so some tiles of the wall are not
    fully covered, and the others jitter by a few ulps around the level."""
    rng = np.random.default_rng(seed)
    d = np.zeros((height, width, samples), np.float32)
    d[:, : int(width * 0.6), :] = level
    ramp = np.linspace(0.0, 2.0 * level, width, dtype=np.float32)
    d[int(height * 0.75):, :, :] = ramp[None, :, None]
    if samples > 1:
        jitter = rng.integers(-3, 4, size=d.shape).astype(np.float32) * np.float32(1e-7)
        d = np.where(d > 0, d + jitter, d).astype(np.float32)
        holes = rng.random((height, width)) < 0.03
        d[holes, rng.integers(0, samples)] = 0.0
    return d


def opaque_tiles_numpy(depth: np.ndarray, froxel: int) -> np.ndarray:
    """reduce_opaque_depth (src/shaders/opaque_depth_reduce.wgsl:36-86) in
    numpy: (covered, quantised farthest depth) per fine tile."""
    h, w = depth.shape[:2]
    z = depth.reshape(h, w, -1).min(axis=2)
    ty, tx = -(-h // froxel), -(-w // froxel)
    out = np.zeros((ty * tx, 2), np.uint32)
    for t in range(ty * tx):
        y0, x0 = (t // tx) * froxel, (t % tx) * froxel
        blk = z[y0:y0 + froxel, x0:x0 + froxel]
        cov = blk > 0
        far = np.float32(min(1.0, float(blk[cov].min()))) if cov.any() else np.float32(1.0)
        out[t, 0] = 1 if cov.all() else 0
        # quantize_depth01: the product rounds to f32 first, then to even
        out[t, 1] = np.uint32(np.rint(np.float32(np.clip(far, 0, 1)) * np.float32(16777215.0)))
    return out


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(peak * peak / mse)

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


def run_gpu(scene: Scene, plugin=None, fused=False, stream=None, scene_color=None, out=None):
    from bevy_strand_rasterizer_b200.plugin import StrandRasterizerPlugin
    if plugin is None:
        plugin = StrandRasterizerPlugin()
        abi.check(plugin.lib.fiber_settings_set(plugin.ctx, C.byref(scene.settings)), "fiber_settings_set")
        for packed, material, w in scene.assets:
            plugin.add_geometry(packed, material, w)
    plugin.frame_begin_raw(scene.camera_cfg, scene.cam, scene.light_cfgs, scene.lights_c, stream)
    if fused:
        plugin.frame_fused(scene_color, None, out, stream)
    else:
        plugin.render_nodes(scene_color, None, out, stream)
    return plugin


def run_ref(scene: Scene, **kw):
    from oracle_bridge import run_oracle
    return run_oracle(scene.assets, scene.camera_cfg, scene.cam, scene.light_cfgs, scene.lights_c, scene.settings,
                      **kw)


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(peak * peak / mse)

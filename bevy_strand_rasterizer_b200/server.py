"""The served mode over libfiber's request server (fiber_server_*).

Render requests of different sizes (scene, camera, lights, resolution) run
over scenes kept resident on the device. A request is admitted as soon as a
slot is free; the frames of different slots overlap on the GPU. The slot count
is what the HBM budget holds. Every slot runs with the temporal shadow history
off, so a request renders the same image alone and in the mix.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .plugin import FroxelConfig, PackedStrandBuffers, StrandMaterial

IDENTITY = np.eye(4, dtype=np.float32).reshape(16)


def _host_ptr(buf) -> int:
    """Address of a contiguous host buffer (numpy array or CPU torch tensor)."""
    if isinstance(buf, np.ndarray):
        if not buf.flags["C_CONTIGUOUS"]:
            raise ValueError("host buffer must be contiguous")
        return int(buf.ctypes.data)
    if hasattr(buf, "data_ptr"):
        if buf.is_cuda or not buf.is_contiguous():
            raise ValueError("host buffer must be a contiguous CPU tensor")
        return int(buf.data_ptr())
    raise TypeError(f"unsupported host buffer {type(buf)!r}")


class FiberServer:
    def __init__(self, device: int = 0, slots: int = 0, max_width: int = 1920, max_height: int = 1080,
                 max_lights: int = 1, max_dom: int = 2048, hbm_budget: int = 0,
                 settings: abi.Settings | None = None, priority_levels: int = 0,
                 priority_order: int = abi.PRIORITY_ARRIVAL):
        self.lib = abi.load_library()
        self.srv = C.c_void_p()
        cfg = abi.ServerConfig(slots, max_width, max_height, max_lights, max_dom, priority_levels, hbm_budget,
                               priority_order, 0)
        st = settings if settings is not None else abi.default_settings()
        abi.check(self.lib.fiber_server_create(device, C.byref(st), C.byref(cfg), C.byref(self.srv)),
                  "fiber_server_create")
        self._keep: dict[int, tuple] = {}
        self.slots = 0

    def add_scene(self, packed: PackedStrandBuffers, material: StrandMaterial | None = None,
                  world_from_local: np.ndarray | None = None) -> int:
        material = material or StrandMaterial()
        v = np.ascontiguousarray(packed.vertices, np.float32)
        idx = np.ascontiguousarray(packed.indices, np.uint32)
        meta = np.ascontiguousarray(packed.meta)
        mat = material.to_c()
        sc = abi.ServerScene()
        sc.vertices, sc.n_vertices = v.ctypes.data, v.shape[0]
        sc.indices, sc.n_indices = idx.ctypes.data, idx.shape[0]
        sc.meta, sc.n_meta = meta.ctypes.data, meta.shape[0]
        sc.geo = packed.geo()
        sc.materials, sc.n_materials = C.addressof(mat), 1
        w = IDENTITY if world_from_local is None else np.asarray(world_from_local, np.float32).reshape(16)
        sc.world_from_local[:] = [float(x) for x in w]
        sid = C.c_uint32()
        abi.check(self.lib.fiber_server_add_scene(self.srv, C.byref(sc), C.byref(sid)), "fiber_server_add_scene")
        return int(sid.value)

    def start(self) -> int:
        n = C.c_uint32()
        abi.check(self.lib.fiber_server_start(self.srv, C.byref(n)), "fiber_server_start")
        self.slots = int(n.value)
        return self.slots

    def now_ns(self) -> int:
        return int(self.lib.fiber_server_now_ns())

    def submit(self, scene: int, camera_cfg: FroxelConfig, cam: abi.Camera, light_cfgs, lights_c, out,
               scene_rgba16f=None, arrival_ns: int = 0) -> int:
        """Queues one request; `out` (and `scene_rgba16f`, if given) are host
        RGBA16F buffers of the camera's size that must stay alive until wait()."""
        r = abi.ServerRequest()
        r.scene = scene
        r.n_lights = len(light_cfgs)
        if r.n_lights > abi.SERVER_MAX_LIGHTS:
            raise ValueError("too many lights")
        r.camera_cfg = camera_cfg.to_c()
        r.camera = cam
        for i, (cfg, light) in enumerate(zip(light_cfgs, lights_c)):
            r.light_cfgs[i] = cfg.to_c()
            r.lights[i] = light
        r.out_rgba16f = _host_ptr(out)
        r.scene_rgba16f = _host_ptr(scene_rgba16f) if scene_rgba16f is not None else None
        r.arrival_ns = arrival_ns
        t = C.c_uint64()
        abi.check(self.lib.fiber_server_submit(self.srv, C.byref(r), C.byref(t)), "fiber_server_submit")
        self._keep[int(t.value)] = (r, out, scene_rgba16f)
        return int(t.value)

    def wait(self, ticket: int, allow_overflow: bool = True, check: bool = True) -> abi.ServerResult:
        """Result of a request. EOVERFLOW (a capacity-sized queue dropped work,
        flagged exactly as the reference flags it; the image was still written)
        is returned, not raised, unless allow_overflow is False; with
        check=False every status is returned in the result."""
        res = abi.ServerResult()
        abi.check(self.lib.fiber_server_wait(self.srv, ticket, C.byref(res)), "fiber_server_wait")
        self._keep.pop(ticket, None)
        if check:
            abi.check(res.status, f"request {ticket}", (abi.OK, abi.EOVERFLOW) if allow_overflow else (abi.OK,))
        return res

    def close(self):
        if self.srv:
            abi.check(self.lib.fiber_server_destroy(self.srv), "fiber_server_destroy")
            self.srv = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

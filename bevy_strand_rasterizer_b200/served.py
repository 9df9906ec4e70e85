"""The served configuration: resident scenes, a seeded Poisson request stream
and its replay against a FiberServer, with per-request latency.

Scenes: 8 seeded scalp-hair sets of 5k to 500k strands x 32 points, straight
and curly alternating. A request draws a scene uniformly, a resolution from
{256^2, 512^2, 1280x720, 1920x1080}, a camera on a sphere of radius 0.4-1.0 m
(upper hemisphere) looking at the origin, and one directional light from the
upper hemisphere with a 512^2, 1024^2 or 2048^2 deep-opacity map.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass

import numpy as np

from . import abi
from .plugin import FroxelConfig, PackedStrandBuffers, pack_strand_set
from .scene import CameraSpec, LightSpec, scalp_hair

SCENE_STRANDS = (5_000, 10_000, 25_000, 50_000, 100_000, 200_000, 350_000, 500_000)
SCENE_POINTS = 32
RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080))
DOM_SIZES = (512, 1024, 2048)


def served_scenes(strands=SCENE_STRANDS, points=SCENE_POINTS, seed=1000) -> list[PackedStrandBuffers]:
    return [pack_strand_set(scalp_hair(n, points, seed + i, curly=(i % 2 == 1))) for i, n in enumerate(strands)]


@dataclass
class Request:
    scene: int
    camera_cfg: FroxelConfig
    camera: abi.Camera
    light_cfgs: list
    lights: object


def _hemisphere(rng) -> np.ndarray:
    z = rng.uniform(0.0, 1.0)
    phi = rng.uniform(0.0, 2.0 * np.pi)
    r = np.sqrt(max(0.0, 1.0 - z * z))
    return np.array([r * np.cos(phi), z, r * np.sin(phi)])


def make_request(rng, scenes: list[PackedStrandBuffers], resolutions=RESOLUTIONS, dom_sizes=DOM_SIZES) -> Request:
    si = int(rng.integers(0, len(scenes)))
    w, h = resolutions[int(rng.integers(0, len(resolutions)))]
    dom = dom_sizes[int(rng.integers(0, len(dom_sizes)))]
    eye = _hemisphere(rng) * rng.uniform(0.4, 1.0)
    spec = CameraSpec(eye=tuple(float(x) for x in eye), width=w, height=h)
    cam = abi.Camera()
    cam.clip_from_world[:] = [float(x) for x in spec.clip_from_world()]
    cam.world_position[:] = [float(x) for x in spec.eye]
    light = LightSpec(tuple(float(x) for x in _hemisphere(rng)), size=dom)
    lights = (abi.Light * 1)()
    packed = scenes[si]
    lights[0].clip_from_world[:] = [float(x) for x in light.clip_from_world(packed.aabb_min, packed.aabb_max)]
    lights[0].direction_to_light[:] = [float(x) for x in light.direction()]
    lights[0].color[:] = [float(x) for x in light.color4()]
    return Request(si, FroxelConfig(w, h, 8, 8, 64), cam, [FroxelConfig(dom, dom, 8, 8, 64)], lights)


def request_stream(n: int, rate_hz: float, scenes, seed: int = 7):
    """n requests with Poisson arrivals at rate_hz (seconds from the start)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_hz, n)) if rate_hz > 0 else np.zeros(n)
    return arrivals, [make_request(rng, scenes) for _ in range(n)]


def replay(server, scene_ids, arrivals, requests, outputs) -> dict:
    """Submits each request at its arrival time (all at once when every arrival
    is 0) and collects the results. outputs maps (w, h) to a host RGBA16F
    buffer the requests of that size write (the images are not inspected).
    Returns latency percentiles (ms, arrival to image in host memory) and
    frames/s over the span from the first arrival to the last completion."""
    n = len(requests)
    tickets = [0] * n
    results = [None] * n
    ready = threading.Semaphore(0)
    errors = []

    def collect():
        for i in range(n):
            ready.acquire()
            if tickets[i] == 0 or errors:
                continue
            try:
                results[i] = server.wait(tickets[i], check=False)
            except Exception as e:  # re-raised by the submitting thread
                errors.append(e)

    th = threading.Thread(target=collect)
    th.start()
    t0 = server.now_ns() + 20_000_000
    try:
        for i, r in enumerate(requests):
            due = t0 + int(arrivals[i] * 1e9)
            while True:
                now = server.now_ns()
                if now >= due:
                    break
                if due - now > 2_000_000:
                    time.sleep((due - now - 1_000_000) / 1e9)
            key = (r.camera_cfg.screen_width, r.camera_cfg.screen_height)
            tickets[i] = server.submit(scene_ids[r.scene], r.camera_cfg, r.camera, r.light_cfgs, r.lights,
                                       outputs[key], arrival_ns=due)
            ready.release()
    finally:
        for _ in range(n - sum(1 for t in tickets if t)):
            ready.release()
        th.join()
    if errors:
        raise errors[0]
    # A request whose status is not OK (e.g. EOVERFLOW: work dropped, the image
    # truncated) counts as failed: it is not a frame, and its latency is kept
    # out of the percentiles.
    ok = [res for res in results if res.status == abi.OK]
    lat = np.array([(res.done_ns - res.arrival_ns) / 1e6 for res in ok]) if ok else np.array([np.nan])
    span = (max(res.done_ns for res in results) - min(res.arrival_ns for res in results)) / 1e9
    return {"requests": n, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "frames_per_s": len(ok) / span, "span_s": span,
            "slots_used": len({res.slot for res in results}),
            "failed": n - len(ok),
            "overflowed": sum(1 for res in results if res.status == abi.EOVERFLOW),
            "statuses": sorted({abi.STATUS_NAMES.get(res.status, str(res.status)) for res in results}),
            "rerendered": sum(1 for res in results if res.renders > 1)}

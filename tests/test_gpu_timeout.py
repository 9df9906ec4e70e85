"""The bounded-wait failure path on the device, through the C ABI.

Every decoupled look-back wait gives up after a bounded number of polls and
sets the frame's error word instead of spinning forever. fiber_debug_stall_lookback
makes one tile of one look-back stage never publish its prefix (a flag that
nothing sets) and shortens the poll limit, so the waits behind that tile run
out for real. The frame must then report FIBER_ETIMEDOUT through
fiber_stats_get with timeout_flags set, the context must stay usable, and the
next frame must be clean and identical to the frame before the stall. Nothing
traps, faults or hangs: the waits are bounded and the kernels after a failed
stage do nothing.
"""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, run_gpu

pytestmark = pytest.mark.gpu

STAGES = {0: "fine prepass", 1: "page allocation", 2: "page prefix", 3: "active tiles", 4: "raster work"}
KEPT = (abi.DUMP_TASKS, abi.DUMP_COUNTS, abi.DUMP_OFFSETS, abi.DUMP_REFS, abi.DUMP_WORK, abi.DUMP_RUNS,
        abi.DUMP_COLOR, abi.DUMP_DOM_OPACITY)


def _status(plugin):
    s = abi.Stats()
    st = plugin.lib.fiber_stats_get(plugin.ctx, C.byref(s))
    return st, s


@pytest.mark.parametrize("stage", sorted(STAGES))
def test_lookback_timeout_is_reported_and_the_next_frame_is_clean(stage):
    scene = build_scene("small", settings_overrides={"history_enabled": 0})
    plugin = run_gpu(scene)
    st, s = _status(plugin)
    assert st == abi.OK and s.timeout_flags == 0
    before = {w: plugin.dump(w).copy() for w in KEPT}

    abi.check(plugin.lib.fiber_debug_stall_lookback(plugin.ctx, stage, 1, 2048), "fiber_debug_stall_lookback")
    run_gpu(scene, plugin=plugin)
    st, s = _status(plugin)
    assert st == abi.ETIMEDOUT, f"{STAGES[stage]}: status {st}"
    assert s.timeout_flags != 0

    run_gpu(scene, plugin=plugin)
    st, s = _status(plugin)
    assert st == abi.OK and s.timeout_flags == 0, f"{STAGES[stage]}: the frame after the stall gave {st}"
    for w, v in before.items():
        assert np.array_equal(plugin.dump(w).view(np.uint8), v.view(np.uint8)), f"{STAGES[stage]}: dump {w}"
    plugin.close()


def test_stall_hook_rejects_unknown_stage():
    scene = build_scene("tiny")
    plugin = run_gpu(scene)
    assert plugin.lib.fiber_debug_stall_lookback(plugin.ctx, 5, 0, 0) == abi.EINVAL
    plugin.close()

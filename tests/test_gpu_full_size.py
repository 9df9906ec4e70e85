"""Parity at the medium configuration's sizes.

- 1920x1080 camera and one 2048^2 x 8 deep-opacity map, exact against the
  oracle on the first 25,000 of its strands (the oracle finishes that in
  seconds);
- the full 100,000-strand medium frame, through properties that hold at any
  size: counts and offsets form per-page exclusive scans, page bases follow
  page order, no (instance, segment) repeats inside a cell, the work items of
  every run go near to far (depth key strictly decreasing) and carry the run's
  load, DOM opacity never decreases with depth, and a repeated frame is
  identical.
"""
import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, run_gpu
from test_gpu_parity import _compare

pytestmark = pytest.mark.gpu


def test_parity_medium_sizes_subset():
    scene = build_scene("medium", strands=25_000, settings_overrides={"fragment_counts_enabled": 1})
    s = _compare(scene)
    assert s.fine_refs > 1_000_000 and s.shadow_runs > 1000


def test_full_medium_frame_invariants():
    scene = build_scene("medium", settings_overrides={"history_enabled": 0})
    p = run_gpu(scene)
    st = p.stats()
    assert st.overflow_flags == 0 and st.timeout_flags == 0 and st.fine_refs > 20_000_000
    pm = p.dump(abi.DUMP_PAGE_META)
    counts = p.dump(abi.DUMP_COUNTS).reshape(-1, 256).astype(np.int64)
    offsets = p.dump(abi.DUMP_OFFSETS).reshape(-1, 256).astype(np.int64)
    excl = np.concatenate([np.zeros((counts.shape[0], 1), np.int64), np.cumsum(counts, 1)[:, :-1]], 1)
    assert np.array_equal(offsets, excl)
    assert np.array_equal(pm["seg_ref_count"].astype(np.int64), counts.sum(1))
    bases = np.concatenate([[0], np.cumsum(pm["seg_ref_count"].astype(np.int64))[:-1]])
    nz = pm["seg_ref_count"] > 0
    assert np.array_equal(pm["seg_ref_base"][nz].astype(np.int64), bases[nz])
    refs = p.dump(abi.DUMP_REFS)
    assert refs.shape[0] == st.fine_refs
    # no (instance, segment) twice in one cell
    flat = counts.reshape(-1)
    starts = (np.repeat(pm["seg_ref_base"].astype(np.int64), 256) + offsets.reshape(-1))[flat > 0]
    cell_of = np.zeros(refs.shape[0], np.int64)
    cell_of[starts] = 1
    cell_of = np.cumsum(cell_of)
    key = (cell_of << 40) ^ (refs["inst_id"].astype(np.int64) << 32) ^ refs["seg_id"].astype(np.int64)
    assert np.unique(key).shape[0] == refs.shape[0]
    # work items: near to far within a run, loads add up
    work, runs = p.dump(abi.DUMP_WORK), p.dump(abi.DUMP_RUNS)
    assert int(work["seg_ref_count"].astype(np.int64).sum()) == st.fine_refs
    for r in runs[:: max(1, runs.shape[0] // 4000)]:
        w = work[int(r["work_base"]): int(r["work_base"]) + int(r["work_count"])]
        assert np.all(np.diff(w["depth_key"].astype(np.int64)) < 0)
        assert int(w["seg_ref_count"].astype(np.int64).sum()) == int(r["load_score"])
    # DOM opacity accumulates with depth
    D = scene.light_cfgs[0].screen_width
    op = p.dump(abi.DUMP_DOM_OPACITY).reshape(-1, D * D)
    assert np.all(np.diff(op, axis=0) >= 0.0)
    first = {w: p.dump(w).copy() for w in (abi.DUMP_REFS, abi.DUMP_WORK, abi.DUMP_COLOR, abi.DUMP_DOM_OPACITY)}
    run_gpu(scene, plugin=p)
    for w, v in first.items():
        assert np.array_equal(p.dump(w).view(np.uint8), v.view(np.uint8)), w
    p.close()

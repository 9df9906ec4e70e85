"""Batched mode: the host-side branch plan (CPU), and on the GPU a batch of
views of different shapes replayed from one graph, each view bit-exact with
the same view rendered alone, before and after the autotuner and when the
context renders alone again afterwards."""
import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from bevy_strand_rasterizer_b200.batched import plan


def test_plan_index_order_is_round_robin():
    assert plan([5, 1, 1, 1, 1], 2, abi.BATCH_ORDER_INDEX).tolist() == [0, 1, 0, 1, 0]


def test_plan_lpt_balances_loads():
    costs = np.array([1, 9, 3, 7, 5, 5, 2, 8], np.float32)
    a = plan(costs, 3, abi.BATCH_ORDER_LPT)
    # longest first to the least loaded branch: 9 | 8 | 7, then 5 -> 7's branch, ...
    loads = np.bincount(a, weights=costs, minlength=3)
    assert sorted(loads.tolist()) == [13.0, 13.0, 14.0]
    assert a[1] == 0 and a[7] == 1 and a[3] == 2


def test_group_views_balances_and_keeps_order():
    from bevy_strand_rasterizer_b200.batched import group_views
    costs = [9.0, 1.0, 3.0, 7.0, 5.0, 5.0, 2.0, 8.0]
    sets = group_views(costs, 3)
    assert sorted(k for g in sets for k in g) == list(range(8))
    assert all(g == sorted(g) for g in sets)
    loads = sorted(sum(costs[k] for k in g) for g in sets)
    assert loads == [13.0, 13.0, 14.0]
    assert group_views(costs, 1) == [list(range(8))]
    assert len(group_views([1.0, 2.0], 4)) == 2  # no empty group


def test_plan_rejects_bad_arguments():
    lib = abi.load_library()
    assert lib.fiber_batch_plan(None, 3, 2, 0, None) == abi.EINVAL
    out = np.zeros(2, np.uint32)
    import ctypes as C
    c = np.ones(2, np.float32)
    assert lib.fiber_batch_plan(c.ctypes.data_as(C.POINTER(C.c_float)), 2, 0, 0,
                                out.ctypes.data_as(C.POINTER(C.c_uint32))) == abi.EINVAL
    assert lib.fiber_batch_create(None, 0, None) == abi.EINVAL


COMPARED = (abi.DUMP_COLOR, abi.DUMP_DEPTH, abi.DUMP_FRAGMENTS, abi.DUMP_DOM_OPACITY, abi.DUMP_DOM_DEPTH,
            abi.DUMP_REFS, abi.DUMP_WORK, abi.DUMP_ATLAS)


@pytest.mark.gpu
def test_batch_matches_views_alone():
    import torch
    from bevy_strand_rasterizer_b200.batched import FiberBatch, batched_views, plain_frame, view_plugin, view_strands

    specs = batched_views(6, seed=77, strand_range=(500, 4_000))
    packed = [view_strands(s) for s in specs]
    kw = dict(fragment_counts=True)
    alone = []
    for s, p in zip(specs, packed):
        ref = view_plugin(s, p, **kw)
        plain_frame(ref, s)
        torch.cuda.synchronize()
        alone.append({w: ref.dump(w).copy() for w in COMPARED})
        ref.close()

    plugins = [view_plugin(s, p, **kw) for s, p in zip(specs, packed)]
    stream = torch.cuda.Stream()
    batch = FiberBatch(plugins)

    def check(tag):
        torch.cuda.synchronize()
        for v, p in enumerate(plugins):
            for w, want in alone[v].items():
                got = p.dump(w)
                assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), f"{tag}: view {v} dump {w}"

    for branches, order in ((1, abi.BATCH_ORDER_INDEX), (3, abi.BATCH_ORDER_LPT)):
        batch.set_tuning(branches, order)
        for _ in range(3):  # replays: the device advances each frame's epoch
            batch.launch(stream)
        stream.synchronize()
        check(f"{branches} branches")
    best = batch.tune(stream)
    assert 1 <= best.branches <= 6 and best.ms > 0.0
    batch.launch(stream)
    stream.synchronize()
    check("tuned")
    # The contexts render alone again after the batch (the host epoch restarts).
    for s, p in zip(specs, plugins):
        plain_frame(p, s)
    check("alone after batch")
    batch.close()
    for p in plugins:
        p.close()

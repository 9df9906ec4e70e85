"""fiber_prefix_pages_noalloc: the page prefix for callers that cannot allocate
device memory where they run it (an engine that owns all GPU memory through
its own pool, or code inside CUDA stream capture). The caller provides every
buffer; the call's only scratch is a fixed device array inside the library.

Its results must equal the prefix the regular frame path (fiber_prepass)
produces for the same froxel counts, on two calls in a row (the second call
reuses the scratch the first one left behind). The file sorts last so a
stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, run_gpu

pytestmark = pytest.mark.gpu


def test_noalloc_prefix_matches_frame_prefix():
    import torch
    torch.cuda.set_device(0)
    plugin = run_gpu(build_scene("small"))
    counts = plugin.dump(abi.DUMP_COUNTS)
    want_offsets = plugin.dump(abi.DUMP_OFFSETS)
    meta = plugin.dump(abi.DUMP_PAGE_META)
    pages = int(meta.shape[0])
    assert pages > 0 and counts.shape[0] == pages * 256
    plugin.close()

    lib = abi.load_library()
    d_counts = torch.from_numpy(counts.astype(np.int32).view(np.int32)).cuda()
    stream = torch.cuda.Stream()
    for call in range(2):
        d_offsets = torch.full((pages * 256,), -1, dtype=torch.int32, device="cuda")
        d_base = torch.full((pages,), -1, dtype=torch.int32, device="cuda")
        d_totals = torch.full((2,), -1, dtype=torch.int32, device="cuda")
        st = lib.fiber_prefix_pages_noalloc(C.c_void_p(d_counts.data_ptr()), pages,
                                            C.c_void_p(d_offsets.data_ptr()), C.c_void_p(d_base.data_ptr()),
                                            C.c_void_p(d_totals.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == abi.OK, f"call {call}: status {st}"
        stream.synchronize()
        offsets = d_offsets.cpu().numpy().view(np.uint32)
        base = d_base.cpu().numpy().view(np.uint32)
        totals = d_totals.cpu().numpy().view(np.uint32)
        assert np.array_equal(offsets, want_offsets), f"call {call}: offsets differ"
        nonempty = meta["seg_ref_count"] > 0
        assert np.array_equal(base[nonempty], meta["seg_ref_base"][nonempty]), f"call {call}: page bases differ"
        assert np.all(base[~nonempty] == 0)
        assert totals[0] == int(meta["seg_ref_count"].sum()) and totals[1] == 0, f"call {call}: totals {totals}"


def test_noalloc_rejects_oversized_page_count():
    lib = abi.load_library()
    st = lib.fiber_prefix_pages_noalloc(None, 65537, None, None, None, None)
    assert st == abi.EINVAL

"""The C-ABI library loads without a GPU, exports every symbol include/fiber.h
declares, and its structs keep the reference's byte layouts."""
import ctypes as C
import re
from pathlib import Path

import pytest

from bevy_strand_rasterizer_b200 import abi

HEADER = Path(__file__).resolve().parents[1] / "include" / "fiber.h"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:fiber_status|uint32_t|uint64_t|const char\*)\s+(fiber_\w+)\(", text, re.M)))


def test_exports_every_declared_symbol():
    lib = abi.load_library()
    declared = header_functions()
    assert len(declared) >= 20
    assert sorted(abi.EXPORTS) == declared
    for name in declared:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("ctype,size", [
    (abi.DevicePtr, 12), (abi.Aabb, 32), (abi.StrandGeo, 64), (abi.StrandMaterialC, 64),
    (abi.StrandInstance, 160), (abi.FroxelConfigC, 20), (abi.Camera, 80), (abi.Light, 96), (abi.Image, 24),
    (abi.ServerConfig, 40), (abi.ServerScene, 192), (abi.ServerRequest, 600), (abi.ServerResult, 40),
    (abi.BatchTuning, 16), (abi.FrustumTelemetry, 44), (abi.Telemetry, 864), (abi.Stats, 408), (abi.View, 136),
])
def test_struct_sizes(ctype, size):
    assert C.sizeof(ctype) == size


def test_numpy_record_sizes():
    assert abi.BINNING_TASK.itemsize == 16 and abi.PROJECTED_SEGMENT.itemsize == 12
    assert abi.RASTER_WORK_ITEM.itemsize == 32 and abi.RASTER_TILE_RUN.itemsize == 32
    assert abi.FINE_SEG_REF.itemsize == 12 and abi.FINE_PAGE_META.itemsize == 32
    assert abi.LUT_ENTRY.itemsize == 16 and abi.FRUSTUM_DESC.itemsize == 64 and abi.STRAND_META.itemsize == 16


def test_default_settings_match_reference():
    s = abi.default_settings()
    assert s.stochastic_cull_enabled == 1 and s.target_strands_per_pixel == 2.0
    assert abs(s.min_keep_probability - 0.02) < 1e-7 and s.shadow_keep_probability == 1.0
    assert s.dom_slices == 12 and s.fine_binning_backend == 0 and s.ref_capacity_factor == 4


def test_status_strings_and_bad_arguments():
    lib = abi.load_library()
    assert lib.fiber_status_string(abi.OK) == b"ok"
    assert lib.fiber_status_string(abi.ETIMEDOUT).startswith(b"bounded")
    assert lib.fiber_ctx_create(0, 0, None) == abi.EINVAL
    assert lib.fiber_settings_default(None) == abi.EINVAL
    assert lib.fiber_ctx_destroy(None) == abi.EINVAL
    assert lib.fiber_span_count() == 14
    assert lib.fiber_span_name(1) == b"strand_prepass/fine"


def test_exact_op_flags_per_source():
    # The integer-deciding stages need one correctly rounded binary32 op per
    # source operation; only the shading file (compared within a tolerance)
    # is compiled with contraction and approximate division and square root.
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "fiber_build", Path(abi.__file__).resolve().parent / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    exact = {"--fmad=false", "-prec-div=true", "-prec-sqrt=true"}
    fast = {"--fmad=true", "-prec-div=false", "-prec-sqrt=false"}
    assert b.FAST_FP_SOURCES == {"fiber_render.cu"}
    for src in b.SOURCES:
        flags = set(b.flags_for(src))
        want, other = (fast, exact) if src in b.FAST_FP_SOURCES else (exact, fast)
        assert want <= flags and not (other & flags), (src, sorted(flags))
        assert "arch=compute_100a,code=sm_100a" in b.flags_for(src)

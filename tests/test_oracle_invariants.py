"""Oracle self-consistency on seeded scenes: canonical orders, count/offset
algebra, thread-count independence, and the committed golden digests."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from bevy_strand_rasterizer_b200 import abi
from common import build_scene, run_ref

GOLDEN = Path(__file__).parent / "golden" / "oracle_tiny.json"


@pytest.fixture(scope="module")
def tiny():
    return run_ref(build_scene("tiny"))


def test_tasks_in_canonical_order(tiny):
    t = tiny.get(abi.DUMP_TASKS)
    frustum = t["packed_field"] >> 3
    key = (frustum.astype(np.uint64) << 48) | (t["id_info"].astype(np.uint64) << 40) | \
          (t["chunk_id"].astype(np.uint64) << 20) | t["seg_idx"].astype(np.uint64)
    assert np.all(np.diff(key.astype(np.int64)) > 0)
    s = tiny.stats()
    assert s.camera_tasks == int((frustum == 0).sum())


def test_pages_counts_offsets_refs(tiny):
    pt = tiny.get(abi.DUMP_PAGE_TABLE)
    pm = tiny.get(abi.DUMP_PAGE_META)
    counts = tiny.get(abi.DUMP_COUNTS).reshape(-1, 256)
    offsets = tiny.get(abi.DUMP_OFFSETS).reshape(-1, 256)
    allocated = np.nonzero(pt)[0]
    assert np.array_equal(pt[allocated], np.arange(1, allocated.size + 1))  # page-table order
    assert np.array_equal(pm["coarse_tile_id"] * 16 + pm["coarse_z"], allocated)
    excl = np.concatenate([np.zeros((counts.shape[0], 1), np.uint32), np.cumsum(counts, 1)[:, :-1]], 1)
    assert np.array_equal(offsets, excl)
    assert np.array_equal(pm["seg_ref_count"], counts.sum(1))
    bases = np.concatenate([[0], np.cumsum(pm["seg_ref_count"])[:-1]])
    nz = pm["seg_ref_count"] > 0
    assert np.array_equal(pm["seg_ref_base"][nz], bases[nz])
    refs = tiny.get(abi.DUMP_REFS)
    keys = tiny.get(100 + 1, np.dtype("<u4"))
    assert refs.shape[0] == int(pm["seg_ref_count"].sum())
    # canonical order in every cell: depth key descending, then (inst, seg)
    for p in range(pm.shape[0]):
        for c in np.nonzero(counts[p] > 1)[0]:
            b = pm["seg_ref_base"][p] + offsets[p, c]
            n = counts[p, c]
            k = keys[b:b + n].astype(np.int64)
            order = np.lexsort((refs["seg_id"][b:b + n], refs["inst_id"][b:b + n], -k))
            assert np.array_equal(order, np.arange(n))


def test_work_items_and_runs(tiny):
    runs = tiny.get(abi.DUMP_RUNS)
    work = tiny.get(abi.DUMP_WORK)
    s = tiny.stats()
    assert runs.shape[0] == s.camera_runs + s.shadow_runs
    assert np.all(runs["frustum_id"][:s.camera_runs] == 0) and np.all(runs["frustum_id"][s.camera_runs:] > 0)
    assert runs["work_count"].sum() == work.shape[0]
    for r in runs:
        items = work[r["work_base"]:r["work_base"] + r["work_count"]]
        assert np.all(items["screen_tile_id"] == r["screen_tile_id"])
        assert items["load_score"].sum() == r["load_score"]
        # near-to-far: coarse z then fine z descending (lane = 255 - cz * 16 - fz)
        zkey = (items["cell_idx"] // 16).astype(np.int64)
        pm = tiny.get(abi.DUMP_PAGE_META)
        cz = pm["coarse_z"][items["page_idx"]].astype(np.int64)
        lane = 255 - (cz * 16 + zkey)
        assert np.all(np.diff(lane) > 0)


def test_thread_count_independent():
    scene = build_scene("tiny", frame=11)
    a = run_ref(scene, threads=1)
    b = run_ref(scene, threads=4)
    for w in range(abi.DUMP_OPAQUE_TILES + 1):
        assert np.array_equal(a.get(w).view(np.uint8), b.get(w).view(np.uint8)), w


def test_golden_digests(tiny):
    gold = json.loads(GOLDEN.read_text())
    for name, digest in gold.items():
        if name == "stats":
            continue
        got = hashlib.sha256(tiny.get(getattr(abi, name)).view("u1").tobytes()).hexdigest()
        assert got == digest, name
    s = tiny.stats().as_dict()
    for k, v in gold["stats"].items():
        assert s[k] == v, k


def test_cull_off_keeps_every_segment():
    scene = build_scene("tiny", cull=False, lights=[])
    s = run_ref(scene).stats()
    # camera-only frame: every on-screen segment is a binning task and is shaded
    assert s.frustum_count == 1 and s.camera_tasks == s.binning_tasks > 0 and s.shadow_runs == 0


@pytest.mark.parametrize("samples", [1, 4])
def test_opaque_cull(tiny, samples):
    """reduce_opaque_depth + fine_tile_occluded_by_opaque: the tiles match an
    independent numpy restatement; page marks are untouched; a camera cell
    keeps all of its references or loses all of them, exactly when its fine
    tile is covered and its slice ends behind the farthest opaque depth; the
    shadow frusta are untouched."""
    from common import opaque_plane, opaque_tiles_numpy
    scene = build_scene("tiny")
    cfg = scene.camera_cfg
    depth = opaque_plane(cfg.screen_width, cfg.screen_height, 0.2, samples, seed=3)
    r = run_ref(scene, opaque_depth=depth, opaque_samples=samples)
    tiles = r.get(abi.DUMP_OPAQUE_TILES).reshape(-1, 2)
    assert np.array_equal(tiles, opaque_tiles_numpy(depth, cfg.froxel_size_x))
    assert 0 < int(tiles[:, 0].sum()) < tiles.shape[0]
    assert not tiny.get(abi.DUMP_OPAQUE_TILES).any()  # no opaque depth: cleared
    assert np.array_equal(r.get(abi.DUMP_PAGE_TABLE), tiny.get(abi.DUMP_PAGE_TABLE))
    s, b = r.stats(), tiny.stats()
    assert 0 < s.fine_refs < b.fine_refs
    assert list(s.frustum_refs)[1:] == list(b.frustum_refs)[1:]

    frusta = r.get(abi.DUMP_FRUSTA)
    cam = frusta[0]
    lut = r.get(abi.DUMP_LUT)
    pm = r.get(abi.DUMP_PAGE_META)
    cc, cb = r.get(abi.DUMP_COUNTS).reshape(-1, 256), tiny.get(abi.DUMP_COUNTS).reshape(-1, 256)
    ftx = -(-int(cam["screen_width"]) // int(cam["froxel_size_x"]))
    fty = -(-int(cam["screen_height"]) // int(cam["froxel_size_y"]))
    culled_cells = 0
    for p in range(pm.shape[0]):
        tile, z = int(pm["coarse_tile_id"][p]), int(pm["coarse_z"][p])
        if tile >= int(cam["coarse_depth_tile_count"]):
            assert np.array_equal(cc[p], cb[p])
            continue
        zmax = np.float32(lut["z_max_q"][tile * 16 + z]) / np.float32(16777215.0)
        ccx, ccy = tile % int(cam["coarse_tiles_x"]), tile // int(cam["coarse_tiles_x"])
        for cell in range(256):
            fx, fy = ccx * 4 + cell % 4, ccy * 4 + (cell // 4) % 4
            hidden = False
            if fx < ftx and fy < fty:
                cov, q = tiles[fy * ftx + fx]
                far = np.float32(q) / np.float32(16777215.0)
                hidden = bool(cov) and zmax <= np.float32(far - np.float32(1e-4))
            want = 0 if hidden else cb[p, cell]
            assert cc[p, cell] == want, (p, cell)
            culled_cells += int(hidden and cb[p, cell] > 0)
    assert culled_cells > 0


def test_telemetry_consistent(tiny):
    """finalize_telemetry's image agrees with the frame's own counts."""
    t = tiny.telemetry()
    s = tiny.stats()
    assert t.allocated_pages == s.allocated_pages and t.binning_tasks == s.binning_tasks
    assert t.frustum_count == s.frustum_count == 2
    assert sum(t.candidate_histogram) == t.active_candidate_pages <= t.allocated_pages
    assert t.page_candidates >= t.active_candidate_pages and t.max_candidates_per_page > 0
    runs = 0
    for f in range(s.frustum_count):
        fr = t.frustum[f]
        assert fr.emitted_segments == s.frustum_tasks[f]
        assert fr.allocated_pages == s.frustum_pages[f] and fr.fine_refs == s.frustum_refs[f]
        assert 0 < fr.retained_strands <= fr.visible_strands and fr.visible_instances == 1
        assert fr.max_page_candidates <= fr.page_candidates and fr.max_raster_load <= fr.raster_load
        runs += fr.raster_runs
    assert runs == s.camera_runs + s.shadow_runs
    assert sum(t.frustum[f].page_candidates for f in range(2)) == t.page_candidates


def _composite_numpy(strand_rgba, strand_depth, scene, scene_depth, dest):
    """strand_composite.wgsl:12-33 + ALPHA_BLENDING onto the loaded destination,
    restated in numpy (binary32, one rounding per operation)."""
    f32 = np.float32
    a = strand_rgba[..., 3:4]
    mixed = scene[..., :3] * (f32(1) - a) + strand_rgba[..., :3] * a
    frag = np.concatenate([mixed, scene[..., 3:4]], axis=-1)
    front = (scene_depth > strand_depth)[..., None]
    frag = np.where(front, scene, frag).astype(f32)
    oma = f32(1) - frag[..., 3:4]
    rgb = frag[..., :3] * frag[..., 3:4] + dest[..., :3] * oma
    alpha = frag[..., 3:4] * f32(1) + dest[..., 3:4] * oma
    return np.concatenate([rgb, alpha], axis=-1).astype(f32)


def test_composite_against_numpy(tiny):
    # The oracle's composite over a distinct destination, in place, and with
    # no scene depth, against the numpy statement of the same rule.
    scene = build_scene("tiny")
    h, w = scene.camera_cfg.screen_height, scene.camera_cfg.screen_width
    strand = tiny.get(abi.DUMP_COLOR).astype(np.float32).reshape(h, w, 4)
    sdepth = tiny.get(abi.DUMP_DEPTH).reshape(h, w)
    rng = np.random.default_rng(4)
    color = rng.uniform(0, 1, (h, w, 4)).astype(np.float16).astype(np.float32)
    color[..., 3] = rng.uniform(0.2, 1.0, (h, w)).astype(np.float16)
    depth = np.where(rng.random((h, w)) < 0.5, sdepth * np.float32(0.5), sdepth * np.float32(1.5)).astype(np.float32)
    dest = rng.uniform(0, 1, (h, w, 4)).astype(np.float32)
    assert (sdepth > 0).sum() > 100
    for d, dst in ((depth, dest), (depth, None), (None, dest)):
        got = tiny.composite(color, d, dst, half_out=False)
        want = _composite_numpy(strand, sdepth, color, np.zeros_like(sdepth) if d is None else d,
                                color if dst is None else dst)
        assert np.array_equal(got, want)
    half = tiny.composite(color, depth, dest, half_out=True)
    assert np.array_equal(half, tiny.composite(color, depth, dest, half_out=False).astype(np.float16).astype(np.float32))

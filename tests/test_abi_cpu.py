"""CPU checks of the C ABI: the library loads, exports every entry point
include/gs_b200.h declares, and reports errors without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import ROOT

HEADER = os.path.join(ROOT, "include", "gs_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^GS_API\s+[\w\s\*]+?\b(gs_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("gs_render", "gs_stage_sh", "gs_stage_project", "gs_stage_build", "gs_stage_sort", "gs_stage_ranges",
              "gs_stage_raster", "gs_render_batch", "gs_scene_create"):
        assert s in syms


def test_library_exports_every_declared_symbol(gs):
    lib = ctypes.CDLL(gs.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_and_helpers(gs):
    assert gs.lib.gs_version() >= 100
    for code in range(0, 7):
        assert gs.lib.gs_status_string(code)
    rc = gs.RenderConfig()
    assert gs.num_tiles(1920, 1080, rc) == 120 * 68
    assert gs.num_tiles(1024, 1024, gs.RenderConfig.reference()) == 4096
    assert gs.key_bits(4096) == 44
    assert gs.key_bits(8160) == 45
    assert gs.key_bits(1) == 32


def test_camera_matches_reference_conventions(gs):
    cam = gs.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 60.0, 800, 600, 0.1, 100.0)
    c = cam.c
    coty = 1 / np.tan(np.radians(30))
    assert np.isclose(c.fov_cotangent[1], coty, rtol=1e-6)
    assert np.isclose(c.fov_cotangent[0], coty / (800 / 600), rtol=1e-6)
    assert np.isclose(c.depth_scale_bias[0], -2 / 99.9, rtol=1e-6)
    assert np.isclose(c.depth_scale_bias[1], -100.1 / 99.9, rtol=1e-6)
    V = np.array(c.view, np.float32).reshape(4, 4)  # [col][row]
    # the origin lies 3 units in front (view z = -3)
    p = V.T @ np.array([0, 0, 0, 1], np.float32)
    assert np.allclose(p[:3], [0, 0, -3], atol=1e-6)


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and __import__("torch").cuda.is_available(),
                    reason="a GPU is present")
def test_errors_without_gpu(gs):
    h = ctypes.c_void_p()
    st = gs.lib.gs_ctx_create(0, ctypes.byref(h))
    assert st in (gs.GS_ERR_NO_DEVICE, gs.GS_ERR_CUDA)
    # null arguments are rejected before any device work
    assert gs.lib.gs_render(None, None, None, None, None, None, None) == gs.GS_ERR_INVALID
    assert gs.lib.gs_stage_ranges(-1, None, 0, None, None) == gs.GS_ERR_INVALID
    assert gs.lib.gs_autotune(None, None, None, 0, None, 1, None, None, None, 0, None, None) == gs.GS_ERR_INVALID
    assert gs.lib.gs_autotune_lookup(None, 0, 1, 1, 1, None, None) == gs.GS_ERR_INVALID
    assert gs.lib.gs_autotune_entries(None) == 0


def test_overlay_text_matches_reference_formats(gs):
    """gs_format_stats formats the lines of DrawPerformanceOverlay
    (app/perf_overlay.cpp:125-161) with the reference's formats."""
    st = {"total_ms": 1.234, "sh_eval_ms": 0.0, "project_ms": 0.25, "build_tile_ms": 0.125, "sort_ms": 0.04,
          "raster_ms": 0.6}
    text = gs.format_stats(3_000_000, st, 812.34)
    assert text.splitlines() == ["FPS: 812.3", "Gaussians: 3000000", "Total: 1.23ms", "SH: 0.00ms",
                                 "Project: 0.25ms", "Build: 0.12ms", "Sort: 0.04ms", "Raster: 0.60ms"]


def test_overlay_font(gs):
    assert gs.font_glyph(" ") == [0] * 7
    assert gs.font_glyph("\x7f") == [0] * 7
    one = gs.font_glyph("1")
    assert len(one) == 7 and all(r < 32 for r in one) and sum(bin(r).count("1") for r in one) > 5
    # every character the overlay prints has a glyph
    for c in "FPS:.0123456789GaussinTotalHProjectBuildSortRasterm":
        assert any(gs.font_glyph(c)), c


def test_image_writers_flip_rows_and_round_trip(gs, tmp_path):
    """PPM and PNG output: top row first (the frame's row 0 is the bottom),
    PPM drops alpha, PNG keeps RGBA; every PNG chunk CRC and the zlib
    stream check out with the standard library's decoders."""
    import struct
    import zlib
    rng = np.random.default_rng(4)
    H, W = 23, 37
    img = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
    ppm = str(tmp_path / "f.ppm")
    gs.write_image(ppm, img)
    data = open(ppm, "rb").read()
    head = f"P6\n{W} {H}\n255\n".encode()
    assert data.startswith(head)
    rgb = np.frombuffer(data[len(head):], np.uint8).reshape(H, W, 3)
    assert np.array_equal(rgb, img[::-1, :, :3])
    png = str(tmp_path / "f.png")
    gs.write_image(png, img)
    data = open(png, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(kind + body)
        chunks[kind] = chunks.get(kind, b"") + body
        pos += 12 + n
    assert struct.unpack(">IIBBBBB", chunks[b"IHDR"]) == (W, H, 8, 6, 0, 0, 0)
    raw = np.frombuffer(zlib.decompress(chunks[b"IDAT"]), np.uint8).reshape(H, 1 + 4 * W)
    assert (raw[:, 0] == 0).all()
    assert np.array_equal(raw[:, 1:].reshape(H, W, 4), img[::-1])
    assert b"IEND" in chunks
    # a frame larger than one stored deflate block
    big = rng.integers(0, 256, (300, 200, 4), dtype=np.uint8)
    gs.write_image(png, big)
    data = open(png, "rb").read()
    idat = data.index(b"IDAT")
    (n,) = struct.unpack(">I", data[idat - 4:idat])
    raw = np.frombuffer(zlib.decompress(data[idat + 4:idat + 4 + n]), np.uint8).reshape(300, 801)
    assert np.array_equal(raw[:, 1:].reshape(300, 200, 4), big[::-1])
    with pytest.raises(gs.GsError):
        gs.write_image(str(tmp_path / "no_such_dir" / "x.png"), img)


def test_autotune_buckets(gs):
    """The tuning table's key, computed on the host: powers of two of N and
    of the pixel count, and six view-count classes."""
    assert gs.autotune_bucket(3_000_000, 1920, 1080, 64) == (21, 20, 5)
    assert gs.autotune_bucket((1 << 20) - 1, 1024, 1024, 1) == (19, 20, 0)
    assert gs.autotune_bucket(1 << 20, 1024, 1023, 1) == (20, 19, 0)
    assert gs.autotune_bucket(0, 1, 1, 1) == (-1, 0, 0)
    classes = [gs.autotune_bucket(1000, 64, 64, v)[2] for v in (1, 2, 4, 5, 8, 9, 16, 17, 32, 33, 1000)]
    assert classes == [0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5]
    for bad in ((-1, 64, 64, 1), (10, 0, 64, 1), (10, 64, 64, 0)):
        with pytest.raises(gs.GsError):
            gs.autotune_bucket(*bad)

"""CPU tests of the oracle: pinned against the reference's own kernel outputs
(tests/golden, produced by tests/golden/make_golden.py on a B200) and
cross-checked against small pure-Python restatements."""
import math
import os

import numpy as np
import pytest

from helpers import GOLDEN, camera_from_fixture, canonical, load_frame, psnr, bits_equal, reference_image_check
from conftest import golden_frames

PROBES = os.path.join(GOLDEN, "probes.npz")


# ---- golden pins -------------------------------------------------------------

@pytest.mark.skipif(not os.path.exists(PROBES), reason="golden probes not generated")
def test_probe_overlap_matches_reference(O):
    d = np.load(PROBES)
    got = O.overlap(d["ell6"], d["rect4"])
    ref = d["overlap"]
    bad = np.nonzero(got != ref)[0]
    assert len(bad) == 0, f"{len(bad)} of {len(ref)} overlap probes differ, first {bad[:10]}"


@pytest.mark.skipif(not os.path.exists(PROBES), reason="golden probes not generated")
def test_probe_aabb_matches_reference(O):
    d = np.load(PROBES)
    got = O.aabb(d["ell6"])
    ok = bits_equal(got, d["aabb"]) | (np.isnan(got) & np.isnan(d["aabb"]))
    assert ok.all(), f"{(~ok).sum()} aabb components differ"


@pytest.mark.skipif(not os.path.exists(PROBES), reason="golden probes not generated")
def test_probe_key_matches_reference(O):
    d = np.load(PROBES)
    got = O.key(d["key_tile"], d["key_depth"])
    assert np.array_equal(got, d["key"])


@pytest.mark.parametrize("name", golden_frames())
def test_oracle_build_sort_ranges_bit_exact_vs_reference(O, name):
    """Stage-isolated: the reference's projected floats in, keys/values/ranges
    must equal the reference's bit for bit."""
    gs = __import__("importlib").import_module("3dgaussianrenderer_b200")
    d = load_frame(name)
    cam = camera_from_fixture(d)
    rc = gs.RenderConfig.reference()
    keys, vals = O.build(d["ref_xy"], d["ref_ell"], d["ref_z"], cam, rc)
    assert len(keys) == int(d["ref_K"])
    keys, vals = O.sort(keys, vals, 44)
    rk, rv = d["ref_keys"], d["ref_vals"]
    assert np.array_equal(keys, rk)
    k2, v2 = canonical(keys, vals)
    assert np.array_equal(v2, rv)
    ranges = O.ranges(keys, 4096)
    assert np.array_equal(ranges, d["ref_ranges"])


@pytest.mark.parametrize("name", golden_frames())
def test_oracle_raster_vs_reference(O, name):
    gs = __import__("importlib").import_module("3dgaussianrenderer_b200")
    d = load_frame(name)
    cam = camera_from_fixture(d)
    rc = gs.RenderConfig.reference()
    color = d["ref_color"] if "ref_color" in d else d["color4"]
    img = O.raster(cam, rc, d["ref_ranges"], d["ref_vals"], d["ref_xy"], d["ref_conic"], color)
    max_diff, p = reference_image_check(img, d)
    assert max_diff <= 2, f"max abs diff {max_diff}"
    assert p >= 50.0


@pytest.mark.parametrize("name", golden_frames())
def test_oracle_project_vs_reference(O, name):
    d = load_frame(name)
    cam = camera_from_fixture(d)
    xy, z, ell, con = O.project(d["pos4"], d["sr4"], cam)
    vis = d["ref_ell"][:, 2] > 0
    np.testing.assert_array_equal(ell[:, 2] > 0, vis)
    np.testing.assert_allclose(z, d["ref_z"], rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(xy[vis], d["ref_xy"][vis], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(ell[vis, 2:], d["ref_ell"][vis, 2:], rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(con[vis, :3], d["ref_conic"][vis, :3], rtol=1e-3, atol=1e-2)


@pytest.mark.parametrize("name", golden_frames())
def test_oracle_sh_vs_reference(O, name):
    d = load_frame(name)
    if "ref_color" not in d:
        pytest.skip("degree-0 scene")
    gs = __import__("importlib").import_module("3dgaussianrenderer_b200")
    deg = int(d["sh_degree"])
    col = O.sh(d["pos4"], gs.scenes.grouped_sh(d["sh"]), 3 * (deg + 1) ** 2, min(deg, 2), d["cam_pos"])
    np.testing.assert_allclose(col, d["ref_color"], atol=2e-6)


@pytest.mark.parametrize("name", golden_frames())
def test_oracle_full_frame_vs_reference(O, name):
    gs = __import__("importlib").import_module("3dgaussianrenderer_b200")
    d = load_frame(name)
    cam = camera_from_fixture(d)
    scene = {"pos4": d["pos4"], "sr4": d["sr4"], "color4": d["color4"], "sh_degree": int(d["sh_degree"]),
             "sh": d["sh"] if int(d["sh_degree"]) > 0 else None}
    sh = gs.scenes.grouped_sh(scene["sh"]) if scene["sh"] is not None else None
    img, K, _, _ = O.render(scene, sh, cam, gs.RenderConfig.reference())
    ref = d["ref_image"]
    assert abs(K - int(d["ref_K"])) <= max(2, int(d["ref_K"]) // 1000)
    diff = np.abs(img.astype(int) - ref.astype(int))
    assert np.percentile(diff, 99.9) <= 2
    assert psnr(img, ref) >= 45.0


# ---- self-consistency against pure-Python restatements ---------------------------

def _py_key(tile, depth):
    if math.isnan(depth):
        q = 0
    else:
        v = min(max((np.float32(depth) + np.float32(1)) * np.float32(0.5), np.float32(0)), np.float32(1))
        f = np.float32(v) * np.float32(4294967296.0)
        q = 0xFFFFFFFF if f >= 4294967296.0 else int(f)
    return (tile << 32) | q


def test_key_matches_python(O):
    rng = np.random.default_rng(0)
    tiles = rng.integers(0, 8160, 500).astype(np.int32)
    depth = np.concatenate([rng.uniform(-1.5, 1.5, 490), [-1, 1, 0, np.nan, np.inf, -np.inf, 1e-30, -1e-30,
                                                          0.9999999, -0.9999999]]).astype(np.float32)
    got = O.key(tiles, depth)
    want = np.array([_py_key(int(t), float(z)) for t, z in zip(tiles, depth)], np.uint64)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [0, 1, 2, 255, 256, 4097, 100_000])
@pytest.mark.parametrize("bits", [44, 51])
def test_sort_is_stable_radix(O, n, bits):
    rng = np.random.default_rng(n + bits)
    tiles = rng.integers(0, 1 << (bits - 32), n).astype(np.uint64)
    depth = rng.integers(0, 64, n).astype(np.uint64)  # many ties
    keys = (tiles << np.uint64(32)) | depth
    vals = rng.permutation(n).astype(np.int32)
    k, v = O.sort(keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order])
    assert np.array_equal(v, vals[order])


def test_ranges_match_python(O):
    rng = np.random.default_rng(3)
    keys = np.sort((rng.integers(0, 50, 1000).astype(np.uint64) << np.uint64(32)) | rng.integers(0, 9, 1000).astype(
        np.uint64))
    got = O.ranges(keys, 64)
    want = np.full(128, -1, np.int32)
    t = keys >> np.uint64(32)
    for i in range(len(keys)):
        if i == 0 or t[i] != t[i - 1]:
            want[2 * t[i]] = i
        if i == len(keys) - 1 or t[i] != t[i + 1]:
            want[2 * t[i] + 1] = i + 1
    assert np.array_equal(got, want)


def test_raster_single_tile_matches_python(O, gs):
    """One 16x16 tile, 40 splats, reference termination: the oracle against a
    direct per-pixel loop (rasterizeTilesKernel restated in Python)."""
    cam = gs.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 60.0, 16, 16, 0.1, 100.0)
    rc = gs.RenderConfig.reference()
    rng = np.random.default_rng(5)
    m = 40
    xy = rng.uniform(-1, 1, (m, 2)).astype(np.float32)
    conic = np.zeros((m, 4), np.float32)
    conic[:, 0] = rng.uniform(1, 30, m)
    conic[:, 2] = rng.uniform(1, 30, m)
    conic[:, 1] = rng.uniform(-0.5, 0.5, m) * np.sqrt(conic[:, 0] * conic[:, 2])
    color = rng.uniform(0, 1, (m, 4)).astype(np.float32)
    img = O.raster(cam, rc, np.array([0, m], np.int32), np.arange(m, dtype=np.int32), xy, conic, color)

    trace = {}  # pixel -> [(C, T) after each entry]
    for py in range(16):
        for px in range(16):
            cx, cy = px * (2 / 16) - 1, py * (2 / 16) - 1
            T, C, steps = 1.0, np.zeros(3), []
            for j in range(m):
                dx, dy = cx - xy[j, 0], cy - xy[j, 1]
                q = conic[j, 0] * dx * dx + conic[j, 2] * dy * dy + 2 * conic[j, 1] * dx * dy
                a = color[j, 3] * min(max(math.exp(-0.5 * q), 0.0), 1.0)
                C = C + color[j, :3] * T * a
                T *= 1 - a
                steps.append((C, T))
            trace[(py, px)] = steps
    stop = m
    for e in list(range(32, m, 32)) + [m]:
        if all(steps[e - 1][1] <= 0.02 for steps in trace.values()):
            stop = e
            break
    want = np.zeros((16, 16, 4), np.uint8)
    for (py, px), steps in trace.items():
        want[py, px, :3] = np.clip(np.floor(steps[stop - 1][0] * 255), 0, 255)
        want[py, px, 3] = 255
    assert np.abs(img.astype(int) - want.astype(int)).max() <= 1


def test_tile_counts_consistent_with_build(O, gs):
    sc = gs.scenes.uniform_scene(5000, seed=9)
    cam = gs.look_at((0.2, 0.1, 3), (0, 0, 0), (0, 1, 0), 60.0, 640, 480, 0.1, 100.0)
    rc = gs.RenderConfig()
    xy, z, ell, con = O.project(sc["pos4"], sc["sr4"], cam)
    rect, cand, hits = O.tile_counts(xy, ell, cam, rc)
    keys, vals = O.build(xy, ell, z, cam, rc)
    assert len(keys) == hits.sum()
    assert (hits <= cand).all()
    # emission order: Gaussian order, ascending tiles inside a Gaussian
    assert (np.diff(vals) >= 0).all()
    tiles = (keys >> np.uint64(32)).astype(np.int64)
    same = np.diff(vals) == 0
    assert (np.diff(tiles)[same] > 0).all()
    assert tiles.max() < gs.num_tiles(640, 480, rc)


def test_block_eval_count_of_the_warp_culled_raster(O, gs):
    """The oracle's count of the evaluations the GPU's warp-culled T_min
    raster executes: counting leaves the image and the unculled count
    unchanged; an 8x8 block evaluates each kept entry for all 64 pixels;
    reference-mode frames add nothing."""
    sc = gs.scenes.uniform_scene(5000, seed=9)
    sh = gs.scenes.grouped_sh(sc["sh"])
    cam = gs.look_at((0.2, 0.1, 3.0), (0, 0, 0), (0, 1, 0), 60.0, 160, 120, 0.1, 100.0)
    rc = gs.RenderConfig()
    img0, k0, ev0, _ = O.render(sc, sh, cam, rc)
    O.count_block_evals(True)
    img1, k1, ev1, _ = O.render(sc, sh, cam, rc)
    blocks = O.block_evals()
    O.count_block_evals(False)
    assert np.array_equal(img0, img1) and k0 == k1 and ev0 == ev1
    assert blocks > 0 and blocks % 64 == 0
    # reference-mode frames are not counted
    O.count_block_evals(True)
    O.render(sc, sh, cam, gs.RenderConfig.reference())
    assert O.block_evals() == 0
    O.count_block_evals(False)


def test_oracle_camera_equals_product_camera(O, gs):
    """The oracle's own look-at camera (used where the product library must
    not be loaded, e.g. the reference arm of bench.py) is the product's
    gs_camera_look_at bit for bit."""
    import ctypes
    rng = np.random.default_rng(8)
    poses = [((0.0, 0.0, 3.0), 60.0, 800, 800), ((0.2, 0.1, 3.0), 60.0, 320, 240)]
    poses += [(tuple(gs.scenes.sphere_pose(rng, r)), 50.0, w, h) for r, (w, h) in
              zip((10.0, 12.0, 15.0), ((1920, 1080), (1280, 720), (1024, 1024)))]
    poses += [(tuple(e), 50.0, 1600, 900) for e in gs.scenes.orbit_ring(4, 15.0, seed=1000)]
    for eye, fovy, W, H in poses:
        a = gs.look_at(eye, (0, 0, 0), (0, 1, 0), fovy, W, H, 0.1, 100.0)
        b = O.look_at(eye, (0, 0, 0), (0, 1, 0), fovy, W, H, 0.1, 100.0)
        assert bytes(a.c) == bytes(b), (eye, fovy, W, H)
        assert ctypes.sizeof(b) == ctypes.sizeof(a.c)

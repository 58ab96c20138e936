"""GPU parity tests of the CUDA path, called through the C ABI.

Against the reference (tests/golden fixtures made by the reference's own
kernels, and the live reference harness oracle/_ref/libgsref.so when it is
present): integer stages bit-exact, depths within 1e-6 relative, images
within 2/255 and >= 50 dB PSNR, in reference-compatible mode.
Against the CPU oracle at benchmark-config sizes: same bars, with the
integer stages compared stage-isolated (same floats in).
"""
import os

import numpy as np
import pytest

from conftest import golden_frames
from helpers import (camera_from_fixture, canonical, load_frame, psnr, bits_equal, scene_from_fixture,
                     reference_image_check)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

IMG_TOL = 2          # max abs difference per 8-bit channel
PSNR_MIN = 50.0      # dB
DEPTH_RTOL = 1e-6


@pytest.fixture(scope="module")
def ctx(gs):
    c = gs.Context(0)
    yield c
    c.close()


def dev(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def project_gpu(gs, pos4, sr4, cam):
    n = pos4.shape[0]
    xy = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    z = torch.zeros(n, dtype=torch.float32, device="cuda")
    ell = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    con = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    gs.stage_project(n, dev(pos4), dev(sr4), cam, xy, z, ell, con)
    torch.cuda.synchronize()
    return xy, z, ell, con


def build_sort_gpu(gs, ctx, n, xy, z, ell, cam, rc, cap=None):
    cap = cap or max(16, 64 * n)
    keys = torch.zeros(cap, dtype=torch.int64, device="cuda")
    vals = torch.zeros(cap, dtype=torch.int32, device="cuda")
    K = gs.stage_build(ctx, n, xy, z, ell, cam, rc, keys, vals, cap)
    keys_alt = torch.zeros(max(K, 1), dtype=torch.int64, device="cuda")
    vals_alt = torch.zeros(max(K, 1), dtype=torch.int32, device="cuda")
    pre_k = keys[:K].cpu().numpy().view(np.uint64).copy()
    pre_v = vals[:K].cpu().numpy().copy()
    tiles = gs.num_tiles(cam.GetWidth(), cam.GetHeight(), rc)
    sel = gs.stage_sort(ctx, K, gs.key_bits(tiles), keys, vals, keys_alt, vals_alt)
    torch.cuda.synchronize()
    sk = (keys_alt if sel else keys)[:K]
    sv = (vals_alt if sel else vals)[:K]
    return K, pre_k, pre_v, sk, sv


# ---- against the reference's own kernels (golden fixtures) ---------------------

@pytest.mark.parametrize("name", golden_frames())
def test_project_vs_reference(gs, name):
    d = load_frame(name)
    cam = camera_from_fixture(d)
    xy, z, ell, con = (t.cpu().numpy() for t in project_gpu(gs, d["pos4"], d["sr4"], cam))
    vis = d["ref_ell"][:, 2] > 0
    assert np.array_equal(ell[:, 2] > 0, vis)
    # every projected float of every splat, culled ones included, is the
    # reference's bit for bit (the depth bar of 1e-6 relative holds a fortiori)
    for k, a in (("xy", xy), ("z", z), ("ell", ell), ("conic", con[:, :3])):
        ref = d["ref_" + k] if k != "conic" else d["ref_conic"][:, :3]
        eq = bits_equal(a, ref) | (np.isnan(a) & np.isnan(ref))
        assert eq.all(), f"{name}: {k} differs from the reference at {np.count_nonzero(~eq)} values"
    np.testing.assert_allclose(z, d["ref_z"], rtol=DEPTH_RTOL, atol=0)


@pytest.mark.parametrize("name", golden_frames())
def test_sh_vs_reference(gs, name):
    d = load_frame(name)
    if "ref_color" not in d:
        pytest.skip("degree-0 scene")
    cam = camera_from_fixture(d)
    deg = int(d["sh_degree"])
    n = d["pos4"].shape[0]
    col = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    gs.stage_sh(n, dev(d["pos4"]), dev(gs.scenes.grouped_sh(d["sh"])), 3 * (deg + 1) ** 2, min(deg, 2), cam, col)
    np.testing.assert_allclose(col.cpu().numpy(), d["ref_color"], atol=1e-6)


@pytest.mark.parametrize("deg", [1, 2, 3])
def test_sh_stage_vs_oracle(gs, O, deg):
    """SH colour of gs_stage_sh against the oracle at each degree, degree 3
    included (its terms follow cuda_renderer.cu:119-156; the reference's
    built kernel stops at degree 2, gaussian_render.cu:62-91)."""
    sc = gs.scenes.uniform_scene(50_000, seed=40 + deg, sh_degree=3)
    sh = gs.scenes.grouped_sh(sc["sh"])
    cam = gs.look_at((0.4, -0.3, 2.5), (0, 0, 0), (0, 1, 0), 60.0, 800, 800, 0.1, 100.0)
    n = sc["pos4"].shape[0]
    col = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    gs.stage_sh(n, dev(sc["pos4"]), dev(sh), 48, deg, cam, col)
    got = col.cpu().numpy()
    want = O.sh(sc["pos4"], sh, 48, deg, np.array(cam.GetPosition(), np.float32))
    np.testing.assert_allclose(got, want, atol=1e-6, rtol=0)
    if deg == 3:
        # the degree-3 terms are large enough to matter in this scene
        lower = O.sh(sc["pos4"], sh, 48, 2, np.array(cam.GetPosition(), np.float32))
        assert np.abs(want[:, :3] - lower[:, :3]).max() > 1e-3


@pytest.mark.parametrize("name", golden_frames())
def test_build_sort_ranges_bit_exact_vs_reference(gs, ctx, name):
    """Stage-isolated: the reference's projection in; K, sorted keys, sorted
    values (equal-key runs canonicalised) and tile ranges bit-exact."""
    d = load_frame(name)
    cam = camera_from_fixture(d)
    rc = gs.RenderConfig.reference()
    n = d["pos4"].shape[0]
    K, _, _, sk, sv = build_sort_gpu(gs, ctx, n, dev(d["ref_xy"]), dev(d["ref_z"]), dev(d["ref_ell"]), cam, rc)
    assert K == int(d["ref_K"])
    k = sk.cpu().numpy().view(np.uint64)
    v = sv.cpu().numpy()
    assert np.array_equal(k, d["ref_keys"])
    assert np.array_equal(canonical(k, v)[1], d["ref_vals"])
    assert np.array_equal(v, d["ref_vals"]), "equal keys must leave in index order"
    ranges = torch.zeros(2 * 4096, dtype=torch.int32, device="cuda")
    gs.stage_ranges(K, sk, 4096, ranges)
    assert np.array_equal(ranges.cpu().numpy(), d["ref_ranges"])


@pytest.mark.parametrize("name", golden_frames())
def test_raster_vs_reference(gs, name):
    d = load_frame(name)
    cam = camera_from_fixture(d)
    rc = gs.RenderConfig.reference()
    color = d["ref_color"] if "ref_color" in d else d["color4"]
    img = torch.zeros((1024, 1024, 4), dtype=torch.uint8, device="cuda")
    gs.stage_raster(cam, rc, dev(d["ref_ranges"]), dev(d["ref_vals"]), dev(d["ref_xy"]), dev(d["ref_conic"]),
                    dev(color), img)
    out = img.cpu().numpy()
    max_diff, p = reference_image_check(out, d)
    assert max_diff <= IMG_TOL
    assert p >= PSNR_MIN
    print(name, "raster max diff", max_diff, "psnr", p)


@pytest.mark.parametrize("name", golden_frames())
def test_full_frame_vs_reference(gs, ctx, name):
    d = load_frame(name)
    cam = camera_from_fixture(d)
    sc = scene_from_fixture(d)
    sh = gs.scenes.grouped_sh(sc["sh"]) if sc["sh"] is not None else None
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, sc["sh_degree"], sc["color4"])
    img, st = gs.render_host(ctx, scene, cam, gs.RenderConfig.reference())
    assert st["num_keys"] == int(d["ref_K"])
    max_diff, p = reference_image_check(img, d)
    assert max_diff <= IMG_TOL
    assert p >= PSNR_MIN


# ---- against the CPU oracle at configuration sizes -------------------------------

CASES = [
    # (scene, n, camera eye, fovy, W, H)
    ("uniform", 100_000, (0.0, 0.0, 3.0), 60.0, 800, 800),
    ("uniform", 20_000, (0.5, 0.4, 2.5), 60.0, 1920, 1080),
    ("clusters", 200_000, (6.0, 3.0, 8.0), 50.0, 1280, 720),
]


def _scene(gs, kind, n, seed=31):
    if kind == "uniform":
        return gs.scenes.uniform_scene(n, seed=seed)
    return gs.scenes.cluster_scene(n, 64, 5.0, seed=seed)


@pytest.mark.parametrize("kind,n,eye,fovy,W,H", CASES)
def test_stages_vs_oracle(gs, ctx, O, kind, n, eye, fovy, W, H):
    sc = _scene(gs, kind, n)
    cam = gs.look_at(eye, (0, 0, 0), (0, 1, 0), fovy, W, H, 0.1, 100.0)
    rc = gs.RenderConfig()
    xy, z, ell, con = project_gpu(gs, sc["pos4"], sc["sr4"], cam)
    oxy, oz, oell, ocon = O.project(sc["pos4"], sc["sr4"], cam)
    vis = ell[:, 2].cpu().numpy() > 0
    np.testing.assert_allclose(z.cpu().numpy(), oz, rtol=DEPTH_RTOL, atol=1e-7)
    np.testing.assert_allclose(xy.cpu().numpy()[vis], oxy[vis], rtol=1e-5, atol=1e-6)
    # integer stages, stage-isolated: GPU floats into both builds
    K, pre_k, pre_v, sk, sv = build_sort_gpu(gs, ctx, n, xy, z, ell, cam, rc)
    ok, ov = O.build(xy.cpu().numpy(), ell.cpu().numpy(), z.cpu().numpy(), cam, rc)
    assert K == len(ok)
    assert np.array_equal(pre_k, ok) and np.array_equal(pre_v, ov), "emission order is Gaussian order"
    tiles = gs.num_tiles(W, H, rc)
    sok, sov = O.sort(ok, ov, gs.key_bits(tiles))
    assert np.array_equal(sk.cpu().numpy().view(np.uint64), sok)
    assert np.array_equal(sv.cpu().numpy(), sov)
    ranges = torch.zeros(2 * tiles, dtype=torch.int32, device="cuda")
    gs.stage_ranges(K, sk, tiles, ranges)
    oranges = O.ranges(sok, tiles)
    assert np.array_equal(ranges.cpu().numpy(), oranges)
    # raster on identical inputs, both termination modes
    deg = 3
    col = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    gs.stage_sh(n, dev(sc["pos4"]), dev(gs.scenes.grouped_sh(sc["sh"])), 48, deg, cam, col)
    for mode_cfg in (gs.RenderConfig(), gs.RenderConfig.reference()):
        img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        gs.stage_raster(cam, mode_cfg, ranges, sv, xy, con, col, img)
        oimg = O.raster(cam, mode_cfg, oranges, sov, xy.cpu().numpy(), con.cpu().numpy(), col.cpu().numpy())
        out = img.cpu().numpy()
        diff = np.abs(out.astype(int) - oimg.astype(int))
        assert diff.max() <= IMG_TOL, f"mode {mode_cfg.termination}: max diff {diff.max()}"
        assert psnr(out, oimg) >= PSNR_MIN


@pytest.mark.parametrize("W,H,tw,th", [(800, 800, 16, 16), (1920, 1080, 16, 16), (1280, 720, 16, 8),
                                       (1600, 900, 8, 8), (1023, 777, 16, 16)])
def test_full_frame_vs_oracle(gs, ctx, O, W, H, tw, th):
    sc = gs.scenes.uniform_scene(60_000, seed=W + H)
    cam = gs.look_at((0.3, 0.2, 3.0), (0, 0, 0), (0, 1, 0), 60.0, W, H, 0.1, 100.0)
    rc = gs.RenderConfig(tile_w=tw, tile_h=th)
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    img, st = gs.render_host(ctx, scene, cam, rc)
    oimg, K, _, _ = O.render(sc, sh, cam, rc)
    diff = np.abs(img.astype(int) - oimg.astype(int))
    # the projections differ in the last bits (libm vs CUDA atan2/cos/sin), so
    # a few border tiles of a splat may differ: bound the bulk and the PSNR
    assert abs(st["num_keys"] - K) <= max(4, K // 2000)
    assert np.percentile(diff, 99.9) <= IMG_TOL
    assert psnr(img, oimg) >= 45.0


@pytest.mark.parametrize("config", ["plain100k", "plain1m"])
def test_plain_configs_full_size_vs_oracle(gs, ctx, O, config):
    """The two single-view configurations at their full sizes: 100k uniform
    Gaussians at 800x800 from (0, 0, 3), fovy 60; 1M clustered Gaussians at
    1920x1080 from a seeded pose on a radius-10 sphere, fovy 50.  Tile lists
    of the GPU's projected floats are bit-exact in the oracle's build; whole
    frames in both modes meet the end-to-end image bar."""
    sc = gs.scenes.config_scene(config)
    if config == "plain100k":
        cam = gs.look_at((0.0, 0.0, 3.0), (0, 0, 0), (0, 1, 0), 60.0, 800, 800, 0.1, 100.0)
    else:
        eye = gs.scenes.sphere_pose(np.random.default_rng(12), 10.0)
        cam = gs.look_at(eye, (0, 0, 0), (0, 1, 0), 50.0, 1920, 1080, 0.1, 100.0)
    n = sc["pos4"].shape[0]
    rc = gs.RenderConfig.reference()
    xy, z, ell, _ = project_gpu(gs, sc["pos4"], sc["sr4"], cam)
    keys = torch.zeros(64 * n, dtype=torch.int64, device="cuda")
    vals = torch.zeros(64 * n, dtype=torch.int32, device="cuda")
    K = gs.stage_build(ctx, n, xy, z, ell, cam, rc, keys, vals, 64 * n)
    ok, ov = O.build(xy.cpu().numpy(), ell.cpu().numpy(), z.cpu().numpy(), cam, rc)
    assert K == len(ok) > 0
    assert np.array_equal(keys[:K].cpu().numpy().view(np.uint64), ok)
    assert np.array_equal(vals[:K].cpu().numpy(), ov)
    del keys, vals
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    for mode_cfg in (gs.RenderConfig.reference(), gs.RenderConfig()):
        img, st = gs.render_host(ctx, scene, cam, mode_cfg)
        oimg, OK, _, _ = O.render(sc, sh, cam, mode_cfg)
        assert abs(st["num_keys"] - OK) <= max(4, OK // 2000)
        diff = np.abs(img.astype(int) - oimg.astype(int))
        assert np.percentile(diff, 99.9) <= IMG_TOL, mode_cfg.termination
        assert psnr(img, oimg) >= 45.0
    scene.close()


def test_batch_views_identical_to_single(gs, ctx):
    """Every view of a mixed-resolution batch is bit-identical to rendering it alone."""
    sc = gs.scenes.cluster_scene(150_000, 32, 5.0, seed=77)
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    rc = gs.RenderConfig()
    cams = []
    rng = np.random.default_rng(5)
    for i, (W, H) in enumerate([(1280, 720), (1600, 900), (1920, 1080), (640, 480), (1280, 720)]):
        cams.append(gs.look_at(gs.scenes.sphere_pose(rng, 12.0), (0, 0, 0), (0, 1, 0), 50.0, W, H, 0.1, 100.0))
    total = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
    out = np.zeros(total, np.uint8)
    st = gs.render_batch_host(ctx, scene, cams, rc, out)
    off = 0
    for c in cams:
        single, s1 = gs.render_host(ctx, scene, c, rc)
        size = c.GetWidth() * c.GetHeight() * 4
        assert np.array_equal(out[off:off + size].reshape(single.shape), single)
        off += size


@pytest.mark.parametrize("views", [17, 40])
def test_large_host_batch_chunks_match_device_batch(gs, ctx, views):
    """Host-output batches above 16 views render 16 views at a time with the
    read-back overlapped; every image equals the device-output batch's (one
    frame for all views), the stats add up the chunks."""
    torch = pytest.importorskip("torch")
    sc = gs.scenes.cluster_scene(120_000, 32, 5.0, seed=78)
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    rng = np.random.default_rng(6)
    sizes = [(1280, 720), (640, 480), (800, 600)]
    cams = [gs.look_at(gs.scenes.sphere_pose(rng, 12.0), (0, 0, 0), (0, 1, 0), 50.0, *sizes[i % 3], 0.1, 100.0)
            for i in range(views)]
    for rc in (gs.RenderConfig(), gs.RenderConfig.reference()):
        outs = [torch.zeros((c.GetHeight(), c.GetWidth(), 4), dtype=torch.uint8, device="cuda") for c in cams]
        std = gs.render_batch(ctx, scene, cams, rc, outs)
        torch.cuda.synchronize()
        total = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
        host = np.zeros(total, np.uint8)
        sth = gs.render_batch_host(ctx, scene, cams, rc, host)
        assert sth["num_keys"] == std["num_keys"]
        assert sth["num_tiles"] == std["num_tiles"]
        off = 0
        for c, o in zip(cams, outs):
            size = c.GetWidth() * c.GetHeight() * 4
            assert np.array_equal(host[off:off + size].reshape(c.GetHeight(), c.GetWidth(), 4), o.cpu().numpy())
            off += size
    scene.close()


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 257, 4097])
def test_small_and_empty_scenes(gs, ctx, O, n):
    sc = gs.scenes.uniform_scene(max(n, 1), seed=n + 3)
    if n == 0:
        for k in ("pos4", "sr4", "color4", "sh"):
            sc[k] = sc[k][:0]
    cam = gs.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 60.0, 640, 480, 0.1, 100.0)
    rc = gs.RenderConfig.reference()
    sh = gs.scenes.grouped_sh(sc["sh"]) if n > 0 else np.zeros(256 * 48, np.float32)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    img, st = gs.render_host(ctx, scene, cam, rc)
    if n == 0:
        assert st["num_keys"] == 0 and img.max() == 0
        return
    oimg, K, _, _ = O.render(sc, sh, cam, rc)
    assert abs(st["num_keys"] - K) <= 2
    assert np.abs(img.astype(int) - oimg.astype(int)).max() <= 8


def test_all_culled_frame(gs, ctx):
    sc = gs.scenes.uniform_scene(10_000, seed=4)
    cam = gs.look_at((0, 0, 3), (0, 0, 6), (0, 1, 0), 60.0, 320, 240, 0.1, 100.0)  # looking away
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3)
    img, st = gs.render_host(ctx, scene, cam, gs.RenderConfig())
    assert st["num_keys"] == 0
    assert img.max() == 0


@pytest.mark.parametrize("n,bits", [(1, 44), (4095, 44), (4096, 44), (4097, 44), (1_000_003, 44), (3_000_000, 51),
                                    (200_000, 64)])
def test_sort_matches_stable_sort(gs, ctx, n, bits):
    rng = np.random.default_rng(n)
    hi = rng.integers(0, 1 << min(bits - 32, 31), n).astype(np.uint64)
    lo = rng.integers(0, 1 << 12, n).astype(np.uint64)  # ties
    keys = (hi << np.uint64(32)) | lo
    if bits == 64:
        keys = rng.integers(0, 2 ** 63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    vals = rng.permutation(n).astype(np.int32)
    k = dev(keys.view(np.int64))
    v = dev(vals)
    ka = torch.zeros_like(k)
    va = torch.zeros_like(v)
    sel = gs.stage_sort(ctx, n, bits, k, v, ka, va)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    gk = (ka if sel else k).cpu().numpy().view(np.uint64)
    gv = (va if sel else v).cpu().numpy()
    assert np.array_equal(gk, keys[order])
    assert np.array_equal(gv, vals[order])


def test_live_reference_harness_frame_time(gs):
    """When the reference harness is present, it runs on this GPU and its
    frame matches the golden image of the same scene."""
    import oracle
    if not os.path.exists(oracle.REF_LIB):
        pytest.skip("reference harness not built")
    names = golden_frames()
    if not names:
        pytest.skip("no golden frames")
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = load_frame(names[0])
    out = mg.run_ref_frame(oracle.Ref(), scene_from_fixture(d), camera_from_fixture(d))
    assert int(out["K"]) == int(d["ref_K"])
    assert np.array_equal(out["keys"], d["ref_keys"])

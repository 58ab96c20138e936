"""GPU tests of the autotuner (gs_autotune / gs_autotune_lookup): the knobs
it sweeps, the table it fills per (N, resolution, views) bucket, and that a
tuned configuration renders the images of the untuned one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

IMG_TOL = 2


def _cams(gs, n, W, H, seed):
    rng = np.random.default_rng(seed)
    return [gs.look_at(gs.scenes.sphere_pose(rng, 6.0), (0, 0, 0), (0, 1, 0), 55.0, W, H, 0.1, 100.0)
            for _ in range(n)]


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 99.0 if mse == 0 else 10 * np.log10(255.0 ** 2 / mse)


def _batch_images(gs, ctx, scene, cams, cfg):
    total = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
    out = np.zeros(total, np.uint8)
    gs.render_batch_host(ctx, scene, cams, cfg, out)
    return out


def test_autotune_tmin_sweeps_tile_shapes_and_fills_the_table(gs):
    ctx = gs.Context(0)
    n = 120_000
    sc = gs.scenes.cluster_scene(n, 16, 3.0, seed=21)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3)
    cams = _cams(gs, 4, 640, 480, 3)
    base = gs.RenderConfig()
    assert gs.autotune_lookup(ctx, n, 640, 480, 4, base) is None
    best, best_ms, results = gs.autotune(ctx, scene, cams, base, iterations=3)
    # four views: coordinate descent over tile shape, the tile sort's radix
    # width, the raster's batch and the persistent raster (views per block
    # matters above 8 views, the onesweep tile shape for onesweep frames)
    shapes = {(r.tile_w, r.tile_h) for r, _ in results}
    assert shapes == {(8, 8), (16, 8), (16, 16)}
    assert {r.sort_bits for r, _ in results} == {8, 16, 24, 32}
    assert {r.raster_chunk for r, _ in results} == {32, 64}
    assert {r.raster_persistent for r, _ in results} == {0, 1}
    assert {r.sort_variant for r, _ in results} == {0}
    assert len(results) == 3 + 3 + 1 + 1  # a candidate is timed once
    assert all(ms > 0 for _, ms in results)
    assert best_ms == min(ms for _, ms in results)
    assert (best.tile_w, best.tile_h) in shapes
    assert gs.lib.gs_autotune_entries(ctx.h) == 1
    # the bucket: same powers of two of N and pixels, same view-count class
    hit = gs.autotune_lookup(ctx, n + 1000, 700, 500, 3, base)
    assert hit is not None and (hit.tile_w, hit.tile_h, hit.views_per_block, hit.sort_bits, hit.raster_chunk,
                                hit.raster_persistent) == \
        (best.tile_w, best.tile_h, best.views_per_block, best.sort_bits, best.raster_chunk, best.raster_persistent)
    assert hit.sh_max_degree == base.sh_max_degree and hit.termination == base.termination
    assert gs.autotune_lookup(ctx, 4 * n, 640, 480, 4, base) is None        # other N bucket
    assert gs.autotune_lookup(ctx, n, 1920, 1080, 4, base) is None          # other resolution bucket
    assert gs.autotune_lookup(ctx, n, 640, 480, 16, base) is None           # other view-count bucket
    assert gs.autotune_lookup(ctx, n, 640, 480, 4, gs.RenderConfig.reference()) is None  # other termination
    # The tuned knobs render the untuned colours to within the renderer's
    # image bar (the bar of the full-frame oracle tests): a tile list holds
    # the splats whose cutoff ellipse reaches the tile, so lists of other
    # tile shapes differ by splats whose faint tails reach the pixel.  Alpha
    # is 255 in tiles that hold any entry and 0 in the others, as in the
    # reference, so it follows the tile grid and may differ only where the
    # colours are faint.
    want = _batch_images(gs, ctx, scene, cams, base).reshape(-1, 4)
    for cfg, _ in results:
        got = _batch_images(gs, ctx, scene, cams, cfg).reshape(-1, 4)
        diff = np.abs(got[:, :3].astype(int) - want[:, :3].astype(int))
        assert np.percentile(diff, 99.9) <= IMG_TOL, (cfg.tile_w, cfg.tile_h)
        assert diff.max() <= 16, (cfg.tile_w, cfg.tile_h, int(diff.max()))
        assert _psnr(got[:, :3], want[:, :3]) >= 45.0
        alpha_differs = got[:, 3] != want[:, 3]
        assert got[alpha_differs, :3].max(initial=0) <= IMG_TOL
        assert want[alpha_differs, :3].max(initial=0) <= IMG_TOL
    scene.close()
    ctx.close()


def test_autotune_reference_mode_keeps_16x16_and_sweeps_views_per_block(gs):
    ctx = gs.Context(0)
    n = 80_000
    sc = gs.scenes.uniform_scene(n, seed=5)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3)
    cams = _cams(gs, 20, 320, 240, 9)
    base = gs.RenderConfig.reference()
    best, best_ms, results = gs.autotune(ctx, scene, cams, base, iterations=2)
    assert {(r.tile_w, r.tile_h) for r, _ in results} == {(16, 16)}
    assert {r.views_per_block for r, _ in results} == {8, 16, 32}
    assert {r.sort_bits for r, _ in results} == {8, 16, 24, 32}
    assert len(results) == 3 + 3
    assert best.termination == gs.GS_TERM_REFERENCE and best.sh_max_degree == 2
    # neither views per block nor the sort's radix width changes the images
    want = _batch_images(gs, ctx, scene, cams, base)
    for cfg, _ in results:
        assert np.array_equal(_batch_images(gs, ctx, scene, cams, cfg), want)
    # retuning the bucket replaces its entry
    gs.autotune(ctx, scene, cams, base, iterations=1)
    assert gs.lib.gs_autotune_entries(ctx.h) == 1
    scene.close()
    ctx.close()


def test_autotune_onesweep_sweeps_sort_variants(gs):
    ctx = gs.Context(0)
    n = 50_000
    sc = gs.scenes.uniform_scene(n, seed=6)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3, keep_order=True)
    cams = _cams(gs, 1, 512, 512, 2)
    base = gs.RenderConfig(ordering=1)
    best, _, results = gs.autotune(ctx, scene, cams, base, iterations=1)
    assert len(results) == 3 + 3 + 1 + 1
    assert {r.sort_variant for r, _ in results} == {0, 1, 2, 3}
    assert {r.sort_bits for r, _ in results} == {16}  # the bucket sort's knob does not apply
    assert best.ordering == 1
    hit = gs.autotune_lookup(ctx, n, 512, 512, 1, base)
    assert hit is not None and hit.sort_variant == best.sort_variant
    assert gs.autotune_lookup(ctx, n, 512, 512, 1, gs.RenderConfig()) is None  # bucket ordering differs
    scene.close()
    ctx.close()


def test_autotune_rejects_bad_arguments(gs):
    ctx = gs.Context(0)
    sc = gs.scenes.uniform_scene(1000, seed=1)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3)
    cams = _cams(gs, 1, 64, 64, 1)
    with pytest.raises(gs.GsError):
        gs.autotune(ctx, scene, cams, gs.RenderConfig(), iterations=0)
    with pytest.raises(gs.GsError):
        gs.autotune(ctx, scene, cams, gs.RenderConfig(tile_w=32, tile_h=32))
    assert gs.lib.gs_autotune_entries(ctx.h) == 0
    scene.close()
    ctx.close()


def test_autotune_picks_the_ordering_when_asked(gs):
    """GS_ORDER_AUTO: the tuner times both orderings and the table returns
    the one it picked; an untuned AUTO frame renders as tile buckets."""
    ctx = gs.Context(0)
    n = 60_000
    sc = gs.scenes.uniform_scene(n, seed=7)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3, keep_order=True)
    cams = _cams(gs, 2, 640, 480, 4)
    auto = gs.RenderConfig(ordering=gs.GS_ORDER_AUTO)
    assert np.array_equal(_batch_images(gs, ctx, scene, cams, auto), _batch_images(gs, ctx, scene, cams,
                                                                                    gs.RenderConfig()))
    best, best_ms, results = gs.autotune(ctx, scene, cams, auto, iterations=1)
    assert {r.ordering for r, _ in results} == {gs.GS_ORDER_BUCKETS, gs.GS_ORDER_ONESWEEP}
    assert best.ordering in (gs.GS_ORDER_BUCKETS, gs.GS_ORDER_ONESWEEP)
    hit = gs.autotune_lookup(ctx, n, 640, 480, 2, auto)
    assert hit is not None and hit.ordering == best.ordering
    # a scene in the caller's order: both orderings give the same images
    want = _batch_images(gs, ctx, scene, cams, gs.RenderConfig())
    for cfg, _ in results:
        got = _batch_images(gs, ctx, scene, cams, cfg).reshape(-1, 4)
        diff = np.abs(got[:, :3].astype(int) - want.reshape(-1, 4)[:, :3].astype(int))
        assert diff.max() <= 16 and np.percentile(diff, 99.9) <= IMG_TOL
    scene.close()
    ctx.close()

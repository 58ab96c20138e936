"""Failure paths that replace the reference's exit-on-error
(core/cuda_error_check.h:2-11) and truncated frames
(core/gaussian_render.cu:506-509), exercised without faulting a GPU:

* a bounded device wait on a word nobody publishes gives up, reports
  GS_ERR_DEVICE_TIMEOUT, and the context keeps rendering correct frames;
* an allocation that fails at any point of a first frame (injected on the
  host) returns GS_ERR_OOM, and the next frame renders the correct image;
* a server request cancelled while queued completes as GS_ERR_CANCELLED,
  its buffer untouched, while the others render the images they render alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _small(gs):
    sc = gs.scenes.cluster_scene(60_000, 16, 3.0, seed=91)
    cam = gs.look_at((2.0, 1.0, 6.0), (0, 0, 0), (0, 1, 0), 50.0, 640, 480, 0.1, 100.0)
    return sc, gs.scenes.grouped_sh(sc["sh"]), cam


def test_bounded_wait_times_out_and_context_survives(gs):
    sc, sh, cam = _small(gs)
    ctx = gs.Context(0)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    before, _ = gs.render_host(ctx, scene, cam, gs.RenderConfig())
    for limit in (1, 1000):
        assert gs.lib.gs_test_bounded_wait(limit, None) == gs.GS_ERR_DEVICE_TIMEOUT
        assert b"gave up" in gs.lib.gs_last_error_string()
    after, st = gs.render_host(ctx, scene, cam, gs.RenderConfig())
    assert st["num_keys"] > 0
    assert np.array_equal(before, after)
    assert gs.lib.gs_test_bounded_wait(0, None) == gs.GS_ERR_INVALID
    scene.close()
    ctx.close()


@pytest.mark.parametrize("cfg", ["tmin", "reference", "onesweep"])
def test_allocation_failure_at_every_point_of_a_first_frame(gs, cfg):
    sc, sh, cam = _small(gs)
    rc = {"tmin": gs.RenderConfig(), "reference": gs.RenderConfig.reference(),
          "onesweep": gs.RenderConfig(ordering=gs.GS_ORDER_ONESWEEP)}[cfg]
    ref_ctx = gs.Context(0)
    ref_scene = gs.Scene(ref_ctx, sc["pos4"], sc["sr4"], sh, 3)
    want, want_st = gs.render_host(ref_ctx, ref_scene, cam, rc)
    ref_scene.close()
    ref_ctx.close()
    failed_at = []
    for skip in range(64):
        ctx = gs.Context(0)
        scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
        gs.lib.gs_test_fail_allocations(skip, 1)
        try:
            img, st = gs.render_host(ctx, scene, cam, rc)
            injected = gs.lib.gs_test_pending_allocation_failures() == 0
        except gs.GsError as e:
            assert e.status == gs.GS_ERR_OOM, e
            failed_at.append(skip)
            # the same context renders the next frame correctly
            img, st = gs.render_host(ctx, scene, cam, rc)
            injected = True
        finally:
            gs.lib.gs_test_fail_allocations(0, 0)
        assert np.array_equal(img, want), f"skip {skip}"
        assert st["num_keys"] == want_st["num_keys"]
        scene.close()
        ctx.close()
        if not injected:
            break  # the frame made fewer than skip + 1 allocations: every point was covered
    assert failed_at == list(range(len(failed_at))) and len(failed_at) >= 3, failed_at


def test_scene_upload_allocation_failure(gs):
    sc, sh, _ = _small(gs)
    ctx = gs.Context(0)
    gs.lib.gs_test_fail_allocations(1, 1)
    try:
        with pytest.raises(gs.GsError) as e:
            gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
        assert e.value.status == gs.GS_ERR_OOM
    finally:
        gs.lib.gs_test_fail_allocations(0, 0)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    assert gs.lib.gs_scene_size(scene.h) == sc["pos4"].shape[0]
    scene.close()
    ctx.close()


def test_server_cancel_while_queued(gs):
    sc, sh, _ = _small(gs)
    srv = gs.Server(0, budget_bytes=8 << 30, max_batch_views=4, num_workers=1)
    sid = srv.add_scene(sc["pos4"], sc["sr4"], sh, 3)
    rng = np.random.default_rng(3)
    cams = [gs.look_at(gs.scenes.sphere_pose(rng, 6.0), (0, 0, 0), (0, 1, 0), 50.0, 640, 480, 0.1, 100.0)
            for _ in range(6)]
    bufs = [np.full((480, 640, 4), 7, np.uint8) for _ in cams]
    srv.pause(True)
    ids = [srv.submit(sid, c, b) for c, b in zip(cams, bufs)]
    cancelled = {1, 4}
    for k in cancelled:
        assert srv.cancel(ids[k]) == gs.GS_OK
    assert srv.cancel(ids[1]) == gs.GS_ERR_INVALID  # already cancelled
    assert srv.cancel(10 ** 9) == gs.GS_ERR_INVALID  # unknown
    srv.pause(False)
    for k, rid in enumerate(ids):
        status = srv.wait_status(rid)
        assert status == (gs.GS_ERR_CANCELLED if k in cancelled else gs.GS_OK), (k, status)
    assert srv.cancel(ids[0]) == gs.GS_ERR_INVALID  # finished
    st = srv.stats()
    assert st["views_done"] == len(ids) - len(cancelled)
    srv.close()
    ctx = gs.Context(0)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    for k, (c, b) in enumerate(zip(cams, bufs)):
        if k in cancelled:
            assert (b == 7).all()
        else:
            alone, _ = gs.render_host(ctx, scene, c, gs.RenderConfig())
            assert np.array_equal(b, alone)
    scene.close()
    ctx.close()

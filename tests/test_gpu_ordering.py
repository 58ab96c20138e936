"""GPU tests of the two tile-list orderings and of graph replay.

GS_ORDER_BUCKETS (per-tile counts, bucket emission, per-tile depth sort) must
give the same per-tile order as GS_ORDER_ONESWEEP (keys in Gaussian order,
stable radix sort on tile and depth bits), which is the order of the
reference's sort: images and key counts are compared bit for bit.  The
scenes cover the size classes of the per-tile sort (tiles above the
4096-key shared-memory capacity take the global-memory path) and equal
depths (a plane facing the camera), where the order falls back to the
Gaussian index.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(gs):
    c = gs.Context(0)
    yield c
    c.close()


def _dense_scene(gs, n, seed, plane=False, spread=0.02):
    """n tiny Gaussians packed into a few tiles (and, for `plane`, all at the
    same depth)."""
    sc = gs.scenes.uniform_scene(n, seed=seed, log_scale_mu=-6.5, log_scale_sigma=0.2)
    rng = np.random.default_rng(seed)
    pos = sc["pos4"].copy()
    pos[:, 0] = rng.uniform(-spread, spread, n)
    pos[:, 1] = rng.uniform(-spread, spread, n)
    pos[:, 2] = 0.0 if plane else rng.uniform(-0.5, 0.5, n)
    sc["pos4"] = pos.astype(np.float32)
    return sc


def _plane_scene(gs, n, seed):
    sc = gs.scenes.uniform_scene(n, seed=seed)
    sc["pos4"][:, 2] = 0.0
    return sc


SCENES = {
    "uniform": lambda gs: gs.scenes.uniform_scene(60_000, seed=11),
    "clusters": lambda gs: gs.scenes.cluster_scene(150_000, 32, 5.0, seed=12),
    "dense_tiles": lambda gs: _dense_scene(gs, 40_000, 13),
    "plane": lambda gs: _plane_scene(gs, 30_000, 14),
    "dense_plane": lambda gs: _dense_scene(gs, 20_000, 15, plane=True),
    "tiny": lambda gs: gs.scenes.uniform_scene(3, seed=16),
}


def _cams(gs, name):
    if name in ("dense_tiles", "plane", "dense_plane"):
        return [gs.look_at((0, 0, 3.0), (0, 0, 0), (0, 1, 0), 60.0, 800, 800, 0.1, 100.0),
                gs.look_at((0.01, 0.0, 2.5), (0, 0, 0), (0, 1, 0), 60.0, 640, 480, 0.1, 100.0)]
    rng = np.random.default_rng(3)
    r = 12.0 if name == "clusters" else 3.0
    return [gs.look_at(gs.scenes.sphere_pose(rng, r), (0, 0, 0), (0, 1, 0), 55.0, W, H, 0.1, 100.0)
            for W, H in ((1280, 720), (800, 800), (1023, 777))]


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("term", [0, 1])
def test_bucket_order_equals_onesweep(gs, ctx, name, term):
    sc = SCENES[name](gs)
    sh = gs.scenes.grouped_sh(sc["sh"])
    # stored in the caller's order: onesweep frames order equal depths by storage order
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3, keep_order=True)
    cams = _cams(gs, name)
    base = gs.RenderConfig.reference() if term == 0 else gs.RenderConfig()
    total = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
    out = {}
    keys = {}
    for ordering in (gs.GS_ORDER_BUCKETS, gs.GS_ORDER_ONESWEEP):
        rc = gs.RenderConfig(**{**base.__dict__, "ordering": ordering, "graph": 0})
        buf = np.zeros(total, np.uint8)
        st = gs.render_batch_host(ctx, scene, cams, rc, buf)
        out[ordering], keys[ordering] = buf, st["num_keys"]
        # single views too
        for c in cams[:1]:
            img, st1 = gs.render_host(ctx, scene, c, rc)
            out[(ordering, "single")] = img
    assert keys[0] == keys[1]
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[(0, "single")], out[(1, "single")])
    scene.close()


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("term", [0, 1])
def test_spatial_storage_order_renders_caller_order_images(gs, ctx, name, term):
    """A scene stored in Morton order (the default) renders, in bucket
    frames, the images of the same scene stored in the caller's order, bit
    for bit: the per-item arithmetic does not depend on where an item is
    stored, and equal depths are ordered by the caller's index (the plane
    scenes are all ties)."""
    sc = SCENES[name](gs)
    sh = gs.scenes.grouped_sh(sc["sh"])
    cams = _cams(gs, name)
    base = gs.RenderConfig.reference() if term == 0 else gs.RenderConfig()
    total = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
    out = {}
    for keep in (True, False):
        scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3, keep_order=keep)
        buf = np.zeros(total, np.uint8)
        st = gs.render_batch_host(ctx, scene, cams, gs.RenderConfig(**{**base.__dict__, "graph": 0}), buf)
        img, _ = gs.render_host(ctx, scene, cams[0], base)
        out[keep] = (buf, img, st["num_keys"])
        scene.close()
    assert out[True][2] == out[False][2]
    assert np.array_equal(out[True][0], out[False][0])
    assert np.array_equal(out[True][1], out[False][1])


def test_spatial_storage_order_degree0_and_odd_sizes(gs, ctx):
    """Degree-0 scenes (colour array gathered) and sizes that are not a
    multiple of the 256-Gaussian SH group."""
    for n, deg in ((1, 3), (2, 0), (257, 2), (70_001, 0), (70_001, 1)):
        sc = gs.scenes.uniform_scene(n, seed=40 + n, sh_degree=deg)
        sh = gs.scenes.grouped_sh(sc["sh"]) if deg > 0 else None
        col = sc["color4"] if deg == 0 else None
        cam = gs.look_at((0.3, 0.2, 3.0), (0, 0, 0), (0, 1, 0), 60.0, 640, 480, 0.1, 100.0)
        imgs = []
        for keep in (True, False):
            scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, deg, color4=col, keep_order=keep)
            imgs.append(gs.render_host(ctx, scene, cam, gs.RenderConfig())[0])
            scene.close()
        assert np.array_equal(imgs[0], imgs[1]), (n, deg)


def test_dense_tiles_exceed_shared_memory_sort(gs, ctx):
    """The dense scene really puts more than 4096 keys into some tile."""
    sc = _dense_scene(gs, 40_000, 13)
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    cam = _cams(gs, "dense_tiles")[0]
    img, st = gs.render_host(ctx, scene, cam, gs.RenderConfig(graph=0))
    tiles = st["num_tiles"]
    assert tiles == 50 * 50
    # the packed region (about 10 pixels across, at the image centre) lies
    # in at most 2 x 2 tiles, so one of them holds more than 4096 keys
    assert st["num_keys"] >= 40_000
    assert st["num_keys"] / 4 > 4096
    scene.close()


def test_graph_replay_matches_stream_launches(gs, ctx):
    """The second call with the same scene, options and view sizes/outputs is
    captured and later ones replay the graph; cameras may change between
    replays and every frame equals the stream-launched one."""
    torch = pytest.importorskip("torch")
    sc = gs.scenes.cluster_scene(200_000, 32, 5.0, seed=21)
    sh = gs.scenes.grouped_sh(sc["sh"])
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    sizes = [(1280, 720), (1920, 1080), (800, 600), (1280, 720)]
    outs = [torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda") for W, H in sizes]
    rng = np.random.default_rng(4)
    replays = []
    for it in range(5):
        cams = [gs.look_at(gs.scenes.sphere_pose(rng, 12.0), (0, 0, 0), (0, 1, 0), 50.0, W, H, 0.1, 100.0)
                for W, H in sizes]
        st = gs.render_batch(ctx, scene, cams, gs.RenderConfig(graph=1), outs)
        torch.cuda.synchronize()
        replays.append(st["graph_replay"])
        got = [o.cpu().numpy() for o in outs]
        total = sum(W * H * 4 for W, H in sizes)
        want = np.zeros(total, np.uint8)
        st2 = gs.render_batch_host(ctx, scene, cams, gs.RenderConfig(graph=0), want)
        assert st2["graph_replay"] == 0
        assert st["num_keys"] == st2["num_keys"]
        off = 0
        for (W, H), g in zip(sizes, got):
            assert np.array_equal(g, want[off:off + W * H * 4].reshape(H, W, 4)), f"iteration {it}"
            off += W * H * 4
        if it >= 1:
            assert st["total_ms"] > 0 and st["raster_ms"] > 0
    assert replays[0] == 0 and all(r == 1 for r in replays[1:]), replays
    scene.close()


def test_tile_list_regrows_and_redoes_frame(gs):
    """A frame whose keys outgrow the lists is redone once at the new size
    (attempts == 2) and renders exactly as a fresh context does."""
    ctx = gs.Context(0)
    sc = gs.scenes.uniform_scene(50_000, seed=31, log_scale_mu=-2.0)  # big splats: K >> n
    sh = gs.scenes.grouped_sh(sc["sh"])
    # caller order: the onesweep frame below orders equal depths by storage order
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3, keep_order=True)
    far = gs.look_at((0, 0, 30.0), (0, 0, 0), (0, 1, 0), 60.0, 1920, 1080, 0.1, 100.0)
    near = gs.look_at((0, 0, 2.5), (0, 0, 0), (0, 1, 0), 60.0, 1920, 1080, 0.1, 100.0)
    rc = gs.RenderConfig(graph=1)
    _, s_far = gs.render_host(ctx, scene, far, rc)
    img, s_near = gs.render_host(ctx, scene, near, rc)
    assert s_near["num_keys"] > s_far["num_keys"]
    assert s_near["num_keys"] > (1 << 20)
    assert s_near["attempts"] == 2
    ref, _ = gs.render_host(ctx, scene, near, gs.RenderConfig(ordering=gs.GS_ORDER_ONESWEEP, graph=0))
    assert np.array_equal(img, ref)
    scene.close()
    ctx.close()

"""Parity of the benchmarked path -- per-pixel T_min termination, tile-bucket
ordering, batched views -- on the benchmark's own configuration: the 3M
Gaussian SH-3 cluster scene, orbit ring of radius 15, one view each at
1280x720, 1600x900 and 1920x1080, rendered as one batch.

Stage-isolated (the GPU's projected floats into the oracle's build, sort and
raster):
  * every tile's list -- global tile, depth bits and Gaussian index of every
    entry, in blend order -- is bit-exact with the oracle's stable sort of
    its build (core/gaussian_render.cu:312-677);
  * the raster of those lists is within 2/255 per channel (max-abs, every
    pixel) and >= 50 dB of the oracle's raster (gaussian_render.cu:679-759
    with per-pixel T_min termination).
End to end (the oracle projects the scene itself): the GPU's projection uses
the hardware reciprocal and square roots, so a few splats whose 3-sigma
ellipse grazes a tile border land in a tile on one side only.  Those tiles
are identified exactly (their lists differ); every pixel outside them is
within 2/255 and the pixels inside them within 6/255 (a grazing splat adds at
most opacity * exp(-4.5) < 0.0112 of colour at a pixel of such a tile and
scales the light behind it by as much: 2 x 2.84 levels, plus 1 for the 8-bit
truncation); PSNR >= 50 dB per view.
"""
import numpy as np
import pytest

from helpers import psnr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

IMG_TOL = 2
GRAZE_TOL = 6
PSNR_MIN = 50.0
RESOLUTIONS = [(1280, 720), (1600, 900), (1920, 1080)]


@pytest.fixture(scope="module")
def bench3(gs, O):
    sc = gs.scenes.config_scene("batch3m")
    sh = gs.scenes.grouped_sh(sc["sh"])
    eyes = gs.scenes.orbit_ring(64, 15.0, seed=1000)
    cams = [gs.look_at(eyes[i], (0, 0, 0), (0, 1, 0), 50.0, *RESOLUTIONS[i], 0.1, 100.0) for i in range(3)]
    ctx = gs.Context(0)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
    rc = gs.RenderConfig()  # T_min, 16x16 tiles, tile buckets: the benchmark's frame
    n = sc["pos4"].shape[0]
    V = len(cams)
    xy = torch.zeros((V * n, 2), dtype=torch.float32, device="cuda")
    z = torch.zeros(V * n, dtype=torch.float32, device="cuda")
    ell = torch.zeros((V * n, 4), dtype=torch.float32, device="cuda")
    con = torch.zeros((V * n, 4), dtype=torch.float32, device="cuda")
    col = torch.zeros((V * n, 4), dtype=torch.float32, device="cuda")
    outs = [torch.zeros((c.GetHeight(), c.GetWidth(), 4), dtype=torch.uint8, device="cuda") for c in cams]
    st = gs.probe_frame(ctx, scene, cams, rc, outs, xy, z, ell, con, col)
    torch.cuda.synchronize()
    lists = gs.probe_tile_lists(ctx)
    probe_imgs = [o.cpu().numpy() for o in outs]
    # the benchmark's entry point: one batch, images to host memory
    total = sum(c.GetWidth() * c.GetHeight() * 4 for c in cams)
    host = np.zeros(total, np.uint8)
    gs.render_batch_host(ctx, scene, cams, rc, host)
    imgs, off = [], 0
    for c in cams:
        size = c.GetWidth() * c.GetHeight() * 4
        imgs.append(host[off:off + size].reshape(c.GetHeight(), c.GetWidth(), 4).copy())
        off += size
    d = {"sc": sc, "sh": sh, "cams": cams, "rc": rc, "n": n, "stats": st, "lists": lists, "imgs": imgs,
         "probe_imgs": probe_imgs,
         "xy": xy.cpu().numpy(), "z": z.cpu().numpy(), "ell": ell.cpu().numpy(), "con": con.cpu().numpy(),
         "col": col.cpu().numpy()}
    scene.close()
    ctx.close()
    return d


def _gpu_entries(gs, O, d):
    """(global tile, depth bits, view * n + index) of every entry of the GPU's
    tile lists, in blend order: tiles sorted by their raster CTA are ordered
    by (depth, index) from the emitted keys, larger tiles are read in the
    order the big-tile sort wrote."""
    L = d["lists"]
    ranges = L["ranges"]
    T = ranges.shape[0]
    cnt = (ranges[:, 1] - ranges[:, 0]).astype(np.int64)
    assert np.all(ranges[1:, 0] == ranges[:-1, 1]) and ranges[0, 0] == 0
    K = int(ranges[-1, 1])
    assert K == d["stats"]["num_keys"] == L["keys"].size
    tile = np.repeat(np.arange(T, dtype=np.int64), cnt)
    keys = L["keys"]
    slot = (keys & np.uint64(0xFFFFFFFF)).astype(np.int64)
    gi = L["slot_index"][slot].astype(np.int64)
    depth = (keys >> np.uint64(32)).astype(np.int64)
    big = np.repeat(cnt > L["fused_cap"], cnt)
    # depth bits of every (view, Gaussian) from its projected depth, for the
    # entries read through the big-tile order
    all_depth = (O.key(np.zeros(d["z"].size, np.int32), d["z"]) & np.uint64(0xFFFFFFFF)).astype(np.int64)
    bgi = L["slot_index"][L["order"][big].astype(np.int64)].astype(np.int64)
    gi[big] = bgi
    depth[big] = all_depth[bgi]
    # small tiles: (depth, index) order inside the tile; big tiles keep their order
    key_small = np.where(big, np.arange(K), 0)
    order = np.lexsort((np.where(big, 0, gi), np.where(big, 0, depth), key_small, tile))
    return tile[order], depth[order], gi[order]


def _oracle_entries(gs, O, d, xy, ell, z):
    """The same triple from the oracle's build + stable sort of each view."""
    tiles, depths, gis = [], [], []
    toff = 0
    n = d["n"]
    for v, cam in enumerate(d["cams"]):
        s = slice(v * n, (v + 1) * n)
        k, val = O.build(xy[s], ell[s], z[s], cam, d["rc"])
        T = gs.num_tiles(cam.GetWidth(), cam.GetHeight(), d["rc"])
        sk, sv = O.sort(k, val, gs.key_bits(T))
        tiles.append((sk >> np.uint64(32)).astype(np.int64) + toff)
        depths.append((sk & np.uint64(0xFFFFFFFF)).astype(np.int64))
        gis.append(sv.astype(np.int64) + v * n)
        toff += T
    return np.concatenate(tiles), np.concatenate(depths), np.concatenate(gis), toff


def _tile_signature(tile, depth, gi, T):
    """Per tile: count and order-sensitive sums of its (depth, index) list
    (wrapping 64-bit arithmetic)."""
    cnt = np.bincount(tile, minlength=T)
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    pos = np.arange(tile.size) - start[tile]
    h = (gi.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)) ^ (depth.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F))
    h = h * (pos.astype(np.uint64) + np.uint64(1))
    sig = np.zeros(T, np.uint64)
    np.add.at(sig, tile, h)
    return cnt, sig


def test_bench_views_batch_host_equals_probe_frame(bench3):
    for a, b in zip(bench3["imgs"], bench3["probe_imgs"]):
        assert np.array_equal(a, b)


def test_bench_views_tile_lists_bit_exact_vs_oracle_build(gs, O, bench3):
    d = bench3
    gt, gdep, ggi = _gpu_entries(gs, O, d)
    ot, odep, ogi, T = _oracle_entries(gs, O, d, d["xy"], d["ell"], d["z"])
    assert d["lists"]["ranges"].shape[0] == T
    assert gt.size == ot.size, (gt.size, ot.size)
    assert np.array_equal(gt, ot)
    assert np.array_equal(gdep, odep)
    assert np.array_equal(ggi, ogi)


def test_bench_views_raster_vs_oracle_raster(gs, O, bench3):
    """The GPU's images against the oracle's raster of the same lists and the
    GPU's own projected centres, conics and colours."""
    d = bench3
    n = d["n"]
    for v, cam in enumerate(d["cams"]):
        s = slice(v * n, (v + 1) * n)
        k, val = O.build(d["xy"][s], d["ell"][s], d["z"][s], cam, d["rc"])
        T = gs.num_tiles(cam.GetWidth(), cam.GetHeight(), d["rc"])
        sk, sv = O.sort(k, val, gs.key_bits(T))
        rng = O.ranges(sk, T)
        oimg = O.raster(cam, d["rc"], rng, sv, d["xy"][s], d["con"][s], d["col"][s])
        img = d["imgs"][v]
        diff = np.abs(img.astype(int) - oimg.astype(int))
        p = psnr(img, oimg)
        print(f"view {v} {cam.GetWidth()}x{cam.GetHeight()}: max diff {diff.max()}, psnr {p:.2f} dB")
        assert diff.max() <= IMG_TOL
        assert p >= PSNR_MIN


def test_bench_views_tuned_knobs_vs_oracle_raster(gs, O, bench3):
    """The knobs the autotuner picks for the benchmark (64-entry raster
    chunks, 32 views per block) against the oracle's raster of the same
    lists: the chunk size moves only where a warp stops after its pixels
    fell below t_min, the view grouping nothing."""
    d = bench3
    n = d["n"]
    rc = gs.RenderConfig(raster_chunk=64, views_per_block=32)
    ctx = gs.Context(0)
    scene = gs.Scene(ctx, d["sc"]["pos4"], d["sc"]["sr4"], d["sh"], 3)
    total = sum(c.GetWidth() * c.GetHeight() * 4 for c in d["cams"])
    host = np.zeros(total, np.uint8)
    gs.render_batch_host(ctx, scene, d["cams"], rc, host)
    scene.close()
    ctx.close()
    off = 0
    for v, cam in enumerate(d["cams"]):
        W, H = cam.GetWidth(), cam.GetHeight()
        img = host[off:off + W * H * 4].reshape(H, W, 4)
        off += W * H * 4
        s = slice(v * n, (v + 1) * n)
        k, val = O.build(d["xy"][s], d["ell"][s], d["z"][s], cam, d["rc"])
        T = gs.num_tiles(W, H, d["rc"])
        sk, sv = O.sort(k, val, gs.key_bits(T))
        oimg = O.raster(cam, d["rc"], O.ranges(sk, T), sv, d["xy"][s], d["con"][s], d["col"][s])
        diff = np.abs(img.astype(int) - oimg.astype(int))
        p = psnr(img, oimg)
        print(f"view {v} (64-entry chunks): max diff {diff.max()}, psnr {p:.2f} dB")
        assert diff.max() <= IMG_TOL
        assert p >= PSNR_MIN


def test_bench_views_end_to_end_vs_oracle(gs, O, bench3):
    """The GPU's images against the oracle's whole frame (its own SH,
    projection, build, sort and raster)."""
    d = bench3
    n = d["n"]
    sc = d["sc"]
    oxy, oz, oell = [], [], []
    for cam in d["cams"]:
        a, b, c, _ = O.project(sc["pos4"], sc["sr4"], cam)
        oxy.append(a)
        oz.append(b)
        oell.append(c)
    ot, odep, ogi, T = _oracle_entries(gs, O, d, np.concatenate(oxy), np.concatenate(oell), np.concatenate(oz))
    gt, gdep, ggi = _gpu_entries(gs, O, d)
    gc, gsig = _tile_signature(gt, gdep, ggi, T)
    oc, osig = _tile_signature(ot, odep, ogi, T)
    moved = (gc != oc) | (gsig != osig)
    toff = 0
    for v, cam in enumerate(d["cams"]):
        W, H = cam.GetWidth(), cam.GetHeight()
        tx = (W + 15) // 16
        Tv = tx * ((H + 15) // 16)
        oimg, K, _, _ = O.render(sc, d["sh"], cam, d["rc"])
        assert K == int(oc[toff:toff + Tv].sum())
        mask = np.zeros((H, W), bool)
        for t in np.nonzero(moved[toff:toff + Tv])[0]:
            ty, txx = divmod(int(t), tx)
            mask[ty * 16:(ty + 1) * 16, txx * 16:(txx + 1) * 16] = True
        img = d["imgs"][v]
        diff = np.abs(img.astype(int) - oimg.astype(int)).max(axis=2)
        p = psnr(img, oimg)
        print(f"view {v}: {int(moved[toff:toff + Tv].sum())} of {Tv} tiles with a grazing splat on one side; "
              f"max diff outside {diff[~mask].max()}, inside {diff[mask].max() if mask.any() else 0}, "
              f"psnr {p:.2f} dB")
        assert diff[~mask].max() <= IMG_TOL
        if mask.any():
            assert diff[mask].max() <= GRAZE_TOL
        assert p >= PSNR_MIN
        # grazing splats are rare: a small fraction of the view's tiles
        assert moved[toff:toff + Tv].sum() <= max(8, Tv // 100)
        toff += Tv

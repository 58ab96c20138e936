"""GPU tests of the C++ renderer API and the continuous-batching server."""
import os
import subprocess
import threading
import time

import numpy as np
import pytest

from helpers import ROOT

pytestmark = pytest.mark.gpu


def test_cpp_renderer_api_matches_c_abi(gs, tmp_path):
    """A C++ program using gauss_render::{LoadPly, Camera, Renderer} renders the
    same image as the C ABI for the same PLY and pose."""
    exe = str(tmp_path / "renderer_api_main")
    pkg = os.path.join(ROOT, "3dgaussianrenderer_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "renderer_api_main.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L", pkg, "-lgs_b200",
                    "-L/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{pkg}", "-o", exe], check=True)
    sc = gs.scenes.uniform_scene(20_000, seed=8, sh_degree=3)
    sh = gs.scenes.grouped_sh(sc["sh"])
    ply = str(tmp_path / "scene.ply")
    gs.save_ply(ply, sc["pos4"], sc["sr4"], sc["color4"], sh, 3)
    m = gs.load_ply(ply)
    ctx = gs.Context(0)
    scene = gs.Scene(ctx, m["pos4"], m["sr4"], m["sh_grouped"], 3)
    for ref_mode in (0, 1):
        out = str(tmp_path / f"img{ref_mode}.raw")
        r = subprocess.run([exe, ply, out, "640", "480", str(ref_mode)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        img = np.fromfile(out, np.uint8).reshape(480, 640, 4)
        assert os.path.getsize(out + ".png") > 640 * 480 * 4  # gauss_render::SaveImage, uncompressed
        cam = gs.look_at((0.3, 0.2, 3.0), (0, 0, 0), (0, 1, 0), 60.0, 640, 480, 0.1, 100.0)
        rc = gs.RenderConfig.reference() if ref_mode else gs.RenderConfig()
        want, _ = gs.render_host(ctx, scene, cam, rc)
        assert np.array_equal(img, want)
    # Renderer::Autotune: the tuned options render the same colours to
    # within the image bar (tile lists of other shapes differ by faint tails)
    out = str(tmp_path / "tuned.raw")
    r = subprocess.run([exe, ply, out, "640", "480", "0", "1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "tuned tile" in r.stdout
    img = np.fromfile(out, np.uint8).reshape(480, 640, 4)
    cam = gs.look_at((0.3, 0.2, 3.0), (0, 0, 0), (0, 1, 0), 60.0, 640, 480, 0.1, 100.0)
    want, _ = gs.render_host(ctx, scene, cam, gs.RenderConfig())
    assert np.percentile(np.abs(img[..., :3].astype(int) - want[..., :3].astype(int)), 99.9) <= 2
    scene.close()
    ctx.close()


def _server_scenes(gs):
    out = []
    for k, n in enumerate((40_000, 90_000, 150_000)):
        sc = gs.scenes.cluster_scene(n, 16, 4.0, seed=100 + k, log_scale_mu=-4.5)
        out.append((sc, gs.scenes.grouped_sh(sc["sh"])))
    return out


def test_server_results_same_alone_and_in_mix(gs):
    """Requests submitted concurrently from several threads are batched with
    others (continuous batching); each image equals the same view rendered
    alone, bit for bit."""
    scenes = _server_scenes(gs)
    srv = gs.Server(0, budget_bytes=40 << 30, max_batch_views=8, num_workers=2)
    ids = [srv.add_scene(sc["pos4"], sc["sr4"], sh, 3) for sc, sh in scenes]
    rng = np.random.default_rng(9)
    res = [(1280, 720), (1920, 1080), (2560, 1440), (640, 480)]
    reqs = []
    for i in range(36):
        s = int(rng.integers(0, len(ids)))
        W, H = res[int(rng.integers(0, len(res)))]
        cam = gs.look_at(gs.scenes.sphere_pose(rng, 12.0), (0, 0, 0), (0, 1, 0), 50.0, W, H, 0.1, 100.0)
        reqs.append((s, cam, np.zeros((H, W, 4), np.uint8)))
    rids = [None] * len(reqs)

    def client(lo, hi):
        for j in range(lo, hi):
            s, cam, out = reqs[j]
            rids[j] = srv.submit(ids[s], cam, out)
            time.sleep(0.001 * (j % 3))

    th = [threading.Thread(target=client, args=(k * 12, (k + 1) * 12)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    lat = [srv.wait(r) for r in rids]
    st = srv.stats()
    assert st["views_done"] == len(reqs)
    assert st["max_batch"] > 1, "requests were never batched"
    assert st["p99_ms"] >= st["p50_ms"] > 0 and all(x > 0 for x in lat)
    ctx = gs.Context(0)
    for (s, cam, out) in reqs:
        sc, sh = scenes[s]
        scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], sh, 3)
        alone, _ = gs.render_host(ctx, scene, cam, gs.RenderConfig())
        assert np.array_equal(out, alone)
        scene.close()
    ctx.close()
    srv.close()


def test_server_budget_and_errors(gs):
    sc = gs.scenes.uniform_scene(50_000, seed=2)
    sh = gs.scenes.grouped_sh(sc["sh"])
    srv = gs.Server(0, budget_bytes=1 << 20, max_batch_views=4, num_workers=1)
    with pytest.raises(gs.GsError) as e:
        srv.add_scene(sc["pos4"], sc["sr4"], sh, 3)
    assert e.value.status == gs.GS_ERR_CAPACITY
    srv.close()
    srv = gs.Server(0, budget_bytes=8 << 30, max_batch_views=4, num_workers=1)
    sid = srv.add_scene(sc["pos4"], sc["sr4"], sh, 3)
    cam = gs.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 60.0, 320, 240, 0.1, 100.0)
    with pytest.raises(gs.GsError) as e:
        srv.submit(sid + 5, cam, np.zeros((240, 320, 4), np.uint8))
    assert e.value.status == gs.GS_ERR_INVALID
    out = np.zeros((240, 320, 4), np.uint8)
    srv.wait(srv.submit(sid, cam, out))
    assert out.any()
    srv.close()


def test_perf_overlay_draws_the_stats_text(gs):
    """gs_draw_stats writes exactly the glyph pixels of the formatted lines
    (white, upright from the displayed top-left corner, row 0 = bottom) and
    leaves every other pixel of the rendered frame as it was."""
    torch = pytest.importorskip("torch")
    ctx = gs.Context(0)
    sc = gs.scenes.uniform_scene(20_000, seed=12)
    scene = gs.Scene(ctx, sc["pos4"], sc["sr4"], gs.scenes.grouped_sh(sc["sh"]), 3)
    W, H = 320, 200
    cam = gs.look_at((0.2, 0.1, 3.0), (0, 0, 0), (0, 1, 0), 60.0, W, H, 0.1, 100.0)
    out = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    st = gs.render(ctx, scene, cam, gs.RenderConfig(), out)
    before = out.cpu().numpy().copy()
    gs.draw_stats(out, W, H, 20_000, st, 123.4)
    torch.cuda.synchronize()
    after = out.cpu().numpy()
    # expected text mask from the formatted lines and the library's font
    mask = np.zeros((H, W), bool)
    for ln, text in enumerate(gs.format_stats(20_000, st, 123.4).splitlines()):
        for col, ch in enumerate(text):
            rows = gs.font_glyph(ch)
            for gy in range(7):
                for gx in range(5):
                    if (rows[gy] >> (4 - gx)) & 1:
                        x, y_top = 5 + 6 * col + gx, 5 + 9 * ln + gy
                        if x < W and y_top < H:
                            mask[H - 1 - y_top, x] = True
    assert mask.sum() > 200
    assert (after[mask] == 255).all()
    assert np.array_equal(after[~mask], before[~mask])
    scene.close()
    ctx.close()

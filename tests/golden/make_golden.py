"""Generates the golden fixtures in tests/golden/ from the reference's own
CUDA kernels (oracle/_ref/libgsref.so, built by oracle/ref/build_ref.sh from
RobinSongx/3DGaussianRenderer core/gaussian_render.cu).  Needs a B200.

    python tests/golden/make_golden.py OUT_DIR [--cube PATH_TO_random_cube.ply]

Writes
  probes.npz        inputs and reference outputs of the device helpers
                    getAABBRect, ellipseRectOverlap and getKey
                    (gaussian_render.cu:234-310), on candidate (splat, tile)
                    pairs of real frames plus random and edge cases;
  frame_<name>.npz  inputs of one 1024x1024 frame and every reference
                    output: colours (SH scenes), clip xy/z, ellipse, conic,
                    K, sorted keys and values (values inside equal-key runs
                    sorted, since the reference emits them in atomic order),
                    tile ranges and the RGBA image.

Scenes are the package's seeded generators; their arrays are stored in
the fixtures, so the tests do not depend on the generators staying the
same.  The random_cube scene is the first 2048 vertices of the
reference's data/random_cube.ply, parsed with the reference's transforms
(ply_parser.cpp:354-390); pass its path when generating.
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
gs = importlib.import_module("3dgaussianrenderer_b200")
import oracle  # noqa: E402

SC = gs.scenes


def parse_inria_ply(path: str, limit: int):
    """Reads a float-only binary PLY and applies the reference's load
    transforms (ply_parser.cpp:241-393) to the first `limit` vertices."""
    with open(path, "rb") as f:
        props, count = [], None
        while True:
            line = f.readline().decode().strip()
            if line.startswith("element vertex"):
                count = int(line.split()[2])
            elif line.startswith("property float"):
                props.append(line.split()[2])
            elif line == "end_header":
                break
        data = np.frombuffer(f.read(4 * len(props) * count), np.float32).reshape(count, len(props))[:limit]
    col = {p: data[:, i] for i, p in enumerate(props)}
    means = np.stack([col["x"], col["y"], col["z"]], 1)
    q = np.stack([col["rot_0"], col["rot_1"], col["rot_2"], col["rot_3"]], 1)
    ls = np.stack([col["scale_0"], col["scale_1"], col["scale_2"]], 1)
    dc = np.stack([col["f_dc_0"], col["f_dc_1"], col["f_dc_2"]], 1)
    return SC.make_scene(means, ls, q, col["opacity"], dc.astype(np.float32), 0)


def canonical(keys, vals):
    order = np.lexsort((vals, keys))
    return keys[order], vals[order]


def run_ref_frame(ref: oracle.Ref, scene: dict, cam) -> dict:
    n = scene["n"]
    dev = "cuda"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    pos = t(scene["pos4"])
    sr = t(scene["sr4"])
    deg = scene["sh_degree"]
    if deg > 0:
        sh = t(SC.grouped_sh(scene["sh"]))
        color = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        sh_count = 3 * (deg + 1) ** 2
    else:
        sh = torch.zeros(1, dtype=torch.float32, device=dev)
        color = t(scene["color4"])
        sh_count = 3
    xy = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    z = torch.zeros(n, dtype=torch.float32, device=dev)
    conic = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    ell = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    img = torch.zeros((1024, 1024, 4), dtype=torch.uint8, device=dev)
    ranges = torch.zeros(2 * 4096, dtype=torch.int32, device=dev)
    cap = 8 * n
    import ctypes
    while True:
        k0 = torch.zeros(cap, dtype=torch.int64, device=dev)
        k1 = torch.zeros(cap, dtype=torch.int64, device=dev)
        v0 = torch.zeros(cap, dtype=torch.int32, device=dev)
        v1 = torch.zeros(cap, dtype=torch.int32, device=dev)
        ms = (ctypes.c_float * 6)()
        fms = ctypes.c_float(0)
        sel = ctypes.c_int(0)
        cam56 = oracle.Ref.camera56(cam)
        size = ref.lib.gsref_render_frame(cam56.ctypes.data, pos.data_ptr(), sr.data_ptr(), color.data_ptr(), deg,
                                          sh_count, sh.data_ptr(), xy.data_ptr(), z.data_ptr(), conic.data_ptr(),
                                          ell.data_ptr(), n, img.data_ptr(), ranges.data_ptr(), k0.data_ptr(),
                                          k1.data_ptr(), v0.data_ptr(), v1.data_ptr(), cap, 148 * 8, ms,
                                          ctypes.byref(fms), ctypes.byref(sel))
        torch.cuda.synchronize()
        if size < cap:
            break
        cap *= 2  # saturated: grow and render again (main.cpp:330-338)
    kk = (k1 if sel.value else k0)[:size].cpu().numpy().view(np.uint64)
    vv = (v1 if sel.value else v0)[:size].cpu().numpy()
    kk, vv = canonical(kk, vv)
    image_raw = img.cpu().numpy()
    # The reference's emission order decides how entries with equal keys are
    # blended, so its image is one sample of several.  Re-run its ranges and
    # raster kernels on the canonical order (equal keys by index) to get the
    # deterministic image of the same kernels.
    ck = torch.from_numpy(kk.view(np.int64).copy()).to(dev)
    cv = torch.from_numpy(vv.copy()).to(dev)
    img.zero_()
    ranges_c = torch.full((2 * 4096,), -1, dtype=torch.int32, device=dev)
    ref.lib.gsref_set_global_args(cam56.ctypes.data, pos.data_ptr(), sr.data_ptr(), color.data_ptr(), deg, sh_count,
                                  sh.data_ptr(), xy.data_ptr(), z.data_ptr(), conic.data_ptr(), ell.data_ptr(), n,
                                  img.data_ptr(), ranges_c.data_ptr())
    ref.lib.gsref_set_tile_list_args(ck.data_ptr(), cv.data_ptr(), size, cap)
    if size:
        ref.lib.gsref_ranges(size)
    ref.lib.gsref_raster()
    torch.cuda.synchronize()
    assert np.array_equal(ranges_c.cpu().numpy(), ranges.cpu().numpy())
    out = {
        "image_canonical": img.cpu().numpy(),
        "K": np.int64(size),
        "xy": xy.cpu().numpy(), "z": z.cpu().numpy(), "ell": ell.cpu().numpy(), "conic": conic.cpu().numpy(),
        "keys": kk, "vals": vv, "ranges": ranges.cpu().numpy(), "image": image_raw,
    }
    if deg > 0:
        out["color"] = color.cpu().numpy()
    return out


def camera_fields(cam) -> dict:
    c = cam.c
    return {"cam_view": np.array(c.view, np.float32), "cam_pos": np.array(c.position, np.float32),
            "cam_cot": np.array(c.fov_cotangent, np.float32), "cam_dsb": np.array(c.depth_scale_bias, np.float32),
            "cam_aspect": np.float32(c.aspect), "cam_wh": np.array([c.width, c.height], np.int32)}


def frame_cases(cube_path: str | None):
    cases = []
    s = SC.uniform_scene(2048, seed=21, sh_degree=3)
    cases.append(("uniform_sh3", s, gs.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 60.0, 1024, 1024, 0.1, 100.0)))
    s = SC.cluster_scene(4096, 8, 2.0, seed=22, sh_degree=1, log_scale_mu=-4.0, log_scale_sigma=0.6)
    cases.append(("clusters_sh1", s, gs.look_at((3.0, 2.5, 5.0), (0, 0, 0), (0, 1, 0), 50.0, 1024, 1024, 0.1, 100.0)))
    rng = np.random.default_rng(23)
    s = SC.uniform_scene(2048, seed=23, sh_degree=0, log_scale_mu=-3.5)
    s["color4"][:, :3] = rng.uniform(-0.5, 1.5, (2048, 3)).astype(np.float32)  # out-of-range colours
    cases.append(("hdr_deg0", s, gs.look_at((0.3, -0.2, 2.5), (0, 0, 0), (0, 1, 0), 60.0, 1024, 1024, 0.1, 100.0)))
    if cube_path and os.path.exists(cube_path):
        s = parse_inria_ply(cube_path, 2048)
        cases.append(("random_cube", s, gs.look_at((2.0, 3.0, 9.0), (0, 0, 0), (0, 1, 0), 50.0, 1024, 1024, 0.1,
                                                   100.0)))
    return cases


def probe_inputs(O, frames, rng):
    """Candidate (ellipse, tile rect) pairs of real frames + random + edge cases."""
    ells, rects = [], []
    for scene, cam, out in frames:
        xy, ell = out["xy"], out["ell"]
        rc = gs.RenderConfig.reference()
        rect, cand, _ = O.tile_counts(xy, ell, cam, rc)
        idx = np.nonzero((cand > 0) & (cand <= 64))[0]
        idx = rng.choice(idx, min(len(idx), 1500), replace=False)
        for i in idx:
            x0, y0, w, h = rect[i]
            for c in range(w * h):
                gx, gy = x0 + c % w, y0 + c // w
                tx = gx * 0.03125 - 1.0
                ty = gy * 0.03125 - 1.0
                ells.append([xy[i, 0], xy[i, 1], *ell[i]])
                rects.append([tx, ty, tx + 0.03125, ty + 0.03125])
    ells = np.array(ells, np.float32)
    rects = np.array(rects, np.float32)
    m = 4000
    r_ell = np.stack([rng.uniform(-1, 1, m), rng.uniform(-1, 1, m), *(lambda a: (np.cos(a), np.sin(a)))(
        rng.uniform(-np.pi, np.pi, m)), rng.uniform(0, 0.1, m), rng.uniform(0, 0.05, m)], 1).astype(np.float32)
    tx = np.floor(rng.uniform(0, 64, m)) * 0.03125 - 1
    ty = np.floor(rng.uniform(0, 64, m)) * 0.03125 - 1
    r_rect = np.stack([tx, ty, tx + 0.03125, ty + 0.03125], 1).astype(np.float32)
    edge_e = np.array([
        [0.0, 0.0, np.nan, np.nan, 0.1, 0.05],
        [0.01, 0.01, 1.0, 0.0, 0.0, 0.0],
        [-128.0, -128.0, 1.0, 0.0, 0.0, 0.0],
        [0.0, 0.0, 0.0, 1.0, np.inf, 0.01],
        [0.015625, 0.015625, 1.0, 0.0, 0.015625, 0.015625],
        [0.03125, 0.0, 0.7071068, 0.7071068, 0.03125, 0.0],
        [0.0, 0.0, 1.0, 0.0, 1e-20, 1e-20],
        [np.nan, 0.0, 1.0, 0.0, 0.1, 0.1],
    ], np.float32)
    edge_r = np.tile(np.array([[0.0, 0.0, 0.03125, 0.03125]], np.float32), (len(edge_e), 1))
    return (np.concatenate([ells, r_ell, edge_e]), np.concatenate([rects, r_rect, edge_r]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--cube", default=None)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    ref = oracle.Ref()
    O = oracle.get()
    rng = np.random.default_rng(2024)
    frames = []
    for name, scene, cam in frame_cases(args.cube):
        out = run_ref_frame(ref, scene, cam)
        frames.append((scene, cam, out))
        rec = {"pos4": scene["pos4"], "sr4": scene["sr4"], "sh_degree": np.int32(scene["sh_degree"]),
               "color4": scene["color4"], **camera_fields(cam), **{"ref_" + k: v for k, v in out.items()}}
        if scene["sh_degree"] > 0:
            rec["sh"] = scene["sh"]
        np.savez_compressed(os.path.join(args.out, f"frame_{name}.npz"), **rec)
        print(name, "K", int(out["K"]), "covered", float((out["image"][..., 3] > 0).mean()))

    ell6, rect4 = probe_inputs(O, frames, rng)
    n = ell6.shape[0]
    dev = "cuda"
    d_ell = torch.from_numpy(ell6).to(dev)
    d_rect = torch.from_numpy(rect4).to(dev)
    d_ov = torch.zeros(n, dtype=torch.int32, device=dev)
    d_aabb = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    assert ref.lib.gsref_probe_overlap(n, d_ell.data_ptr(), d_rect.data_ptr(), d_ov.data_ptr()) == 0
    assert ref.lib.gsref_probe_aabb(n, d_ell.data_ptr(), d_aabb.data_ptr()) == 0
    m = 20000
    tiles = rng.integers(0, 4096, m).astype(np.int32)
    depth = np.concatenate([rng.uniform(-1.2, 1.2, m - 8),
                            np.array([-1, 1, 0, np.nan, np.inf, -np.inf, 0.9999999, -0.9999999])]).astype(np.float32)
    d_t = torch.from_numpy(tiles).to(dev)
    d_z = torch.from_numpy(depth).to(dev)
    d_k = torch.zeros(m, dtype=torch.int64, device=dev)
    assert ref.lib.gsref_probe_key(m, d_t.data_ptr(), d_z.data_ptr(), d_k.data_ptr()) == 0
    np.savez_compressed(os.path.join(args.out, "probes.npz"), ell6=ell6, rect4=rect4,
                        overlap=d_ov.cpu().numpy(), aabb=d_aabb.cpu().numpy(), key_tile=tiles, key_depth=depth,
                        key=d_k.cpu().numpy().view(np.uint64))
    print("probes", n, "overlap hits", int(d_ov.sum()))


if __name__ == "__main__":
    main()

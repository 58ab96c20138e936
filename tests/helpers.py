"""Shared helpers of the test suite."""
import importlib
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def gs_mod():
    return importlib.import_module("3dgaussianrenderer_b200")


def camera_from_fixture(d):
    """Rebuilds the product camera stored in a golden frame fixture."""
    gs = gs_mod()
    cam = gs.Camera()
    c = gs.gs_camera()
    c.view[:] = d["cam_view"].tolist()
    c.position[:] = d["cam_pos"].tolist()
    c.fov_cotangent[:] = d["cam_cot"].tolist()
    c.depth_scale_bias[:] = d["cam_dsb"].tolist()
    c.aspect = float(d["cam_aspect"])
    c.width, c.height = (int(x) for x in d["cam_wh"])
    cam.c = c
    cam._w, cam._h = c.width, c.height
    return cam


def scene_from_fixture(d):
    deg = int(d["sh_degree"])
    return {"pos4": d["pos4"], "sr4": d["sr4"], "color4": d["color4"], "sh_degree": deg,
            "sh": d["sh"] if deg > 0 else None, "n": d["pos4"].shape[0]}


def load_frame(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def psnr(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    mse = np.mean((a - b) ** 2)
    return float("inf") if mse == 0 else 10 * np.log10(255.0 ** 2 / mse)


def canonical(keys, vals):
    order = np.lexsort((vals, keys))
    return keys[order], vals[order]


def tie_pixel_mask(keys, width=1024, height=1024, tile=16):
    """Pixels of tiles whose sorted list holds equal keys.  The reference
    emits keys through atomics, so entries with identical (tile, depth) keys
    reach its raster in an arbitrary order; its image there is one sample of
    several valid blends and is compared by PSNR only."""
    keys = np.asarray(keys, np.uint64)
    mask = np.zeros((height, width), bool)
    if len(keys) < 2:
        return mask
    tiles_x = (width + tile - 1) // tile
    for t in np.unique((keys[1:][keys[1:] == keys[:-1]] >> np.uint64(32)).astype(np.int64)):
        ty, tx = divmod(int(t), tiles_x)
        mask[ty * tile:(ty + 1) * tile, tx * tile:(tx + 1) * tile] = True
    return mask


def reference_image_check(img, d):
    """(max abs diff, PSNR) of an image against a golden frame's reference
    image: the canonical-order image of the reference's kernels when the
    fixture has it, otherwise its raw image with tied-key tiles masked out."""
    if "ref_image_canonical" in d:
        ref = d["ref_image_canonical"]
        diff = np.abs(img.astype(int) - ref.astype(int))
        return int(diff.max()), psnr(img, ref)
    ref = d["ref_image"]
    mask = tie_pixel_mask(d["ref_keys"], ref.shape[1], ref.shape[0])
    diff = np.abs(img.astype(int) - ref.astype(int))
    diff[mask] = 0
    return int(diff.max()), psnr(img[~mask], ref[~mask])


def bits_equal(a, b):
    """Bitwise equality of float arrays, treating +0 and -0 as equal."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    same = a.view(np.uint32) == b.view(np.uint32)
    return same | ((a == 0) & (b == 0))

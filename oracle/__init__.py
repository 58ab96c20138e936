"""Test-infrastructure bindings: the CPU oracle and the reference harness.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the product package.

* ``libgsoracle.so`` (oracle/_build, from gs_oracle.c): plain-C
  restatement of the reference pipeline (RobinSongx/3DGaussianRenderer,
  core/gaussian_render.cu), OpenMP-parallel.
* ``libgsref.so`` (oracle/_ref, from oracle/ref/build_ref.sh): the
  reference's own CUDA kernels behind a small C-ABI harness; GPU only.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libgsoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgsref.so")
# the same frame-loop harness over include/gs_stage_compat.hpp (gs_b200
# behind the reference's stage declarations): the stage-API drop-in
COMPAT_LIB = os.path.join(HERE, "_ref", "libgscompat.so")

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64


class gso_camera(ctypes.Structure):
    _fields_ = [
        ("view", ctypes.c_float * 16),
        ("position", ctypes.c_float * 3),
        ("fov_cotangent", ctypes.c_float * 2),
        ("depth_scale_bias", ctypes.c_float * 2),
        ("aspect", ctypes.c_float),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
    ]


class gso_cfg(ctypes.Structure):
    _fields_ = [
        ("sh_max_degree", ctypes.c_int32),
        ("termination", ctypes.c_int32),
        ("t_min", ctypes.c_float),
        ("tile_w", ctypes.c_int32),
        ("tile_h", ctypes.c_int32),
    ]


def camera(cam) -> gso_camera:
    """Oracle camera from a product Camera / gs_camera (identical layout)."""
    if isinstance(cam, gso_camera):
        return cam
    c = getattr(cam, "c", cam)
    return gso_camera.from_buffer_copy(bytes(c))


def cfg(rc) -> gso_cfg:
    if isinstance(rc, gso_cfg):
        return rc
    return gso_cfg(rc.sh_max_degree, rc.termination, rc.t_min, rc.tile_w, rc.tile_h)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _addr(a):
    return None if a is None else a.ctypes.data


class Oracle:
    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C {HERE}`")
        self.lib = L = ctypes.CDLL(path)
        pc, pg = ctypes.POINTER(gso_camera), ctypes.POINTER(gso_cfg)
        sig = {
            "gso_set_fma_mode": (None, [ctypes.c_int]),
            "gso_get_fma_mode": (ctypes.c_int, []),
            "gso_set_u8_mode": (None, [ctypes.c_int]),
            "gso_set_threads": (None, [ctypes.c_int]),
            "gso_max_threads": (ctypes.c_int, []),
            "gso_sh": (None, [_I64, _P, _P, _I32, _I32, _P, _P]),
            "gso_project": (None, [_I64, _P, _P, pc, _P, _P, _P, _P]),
            "gso_aabb": (None, [_I64, _P, _P]),
            "gso_overlap": (None, [_I64, _P, _P, _P]),
            "gso_key": (None, [_I64, _P, _P, _P]),
            "gso_tile_counts": (None, [_I64, _P, _P, pc, pg, _P, _P, _P]),
            "gso_build": (_I64, [_I64, _P, _P, _P, pc, pg, _P, _P, _I64]),
            "gso_sort": (None, [_I64, _P, _P, _I32]),
            "gso_ranges": (None, [_I64, _P, _I32, _P]),
            "gso_raster": (None, [pc, pg, _P, _P, _P, _P, _P, _P, _P]),
            "gso_render": (_I64, [_I64, _P, _P, _P, _P, _I32, _I32, pc, pg, _P, _I64, _P, _P]),
            "gso_set_count_block_evals": (None, [_I32]),
            "gso_look_at": (None, [pc, _P, _P, _P, ctypes.c_float, _I32, _I32, ctypes.c_float, ctypes.c_float]),
            "gso_block_evals": (_I64, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args

    def set_fma_mode(self, m: int):
        self.lib.gso_set_fma_mode(m)

    def set_u8_mode(self, m: int):
        self.lib.gso_set_u8_mode(m)

    def fma_mode(self) -> int:
        return self.lib.gso_get_fma_mode()

    def set_threads(self, n: int):
        self.lib.gso_set_threads(n)

    def look_at(self, eye, target, up=(0.0, 1.0, 0.0), fovy_deg=50.0, width=1024, height=1024, near=0.1,
                far=100.0) -> gso_camera:
        """A camera built by the oracle alone (no product library), with the
        same float arithmetic as gs_camera_look_at: fovy in degrees, converted
        to radians in double precision and rounded to float."""
        cam = gso_camera()
        e, t, u = (np.ascontiguousarray(x, np.float32) for x in (eye, target, up))
        self.lib.gso_look_at(ctypes.byref(cam), _addr(e), _addr(t), _addr(u), float(np.radians(fovy_deg)),
                             int(width), int(height), float(near), float(far))
        return cam

    def count_block_evals(self, on: bool):
        """Counts, in later T_min rasters, the (pixel, entry) evaluations the
        GPU's warp-culled raster executes (read with block_evals())."""
        self.lib.gso_set_count_block_evals(1 if on else 0)

    def block_evals(self) -> int:
        return int(self.lib.gso_block_evals())

    def max_threads(self) -> int:
        return self.lib.gso_max_threads()

    def sh(self, pos4, sh_grouped, sh_count, degree, cam_pos):
        pos4 = _f32(pos4)
        n = pos4.shape[0]
        out = np.zeros((n, 4), np.float32)
        cp = _f32(cam_pos)
        self.lib.gso_sh(n, _addr(pos4), _addr(_f32(sh_grouped)), sh_count, degree, _addr(cp), _addr(out))
        return out

    def project(self, pos4, sr4, cam):
        pos4, sr4 = _f32(pos4), _f32(sr4)
        n = pos4.shape[0]
        xy = np.zeros((n, 2), np.float32)
        z = np.zeros(n, np.float32)
        ell = np.zeros((n, 4), np.float32)
        con = np.zeros((n, 4), np.float32)
        c = camera(cam)
        self.lib.gso_project(n, _addr(pos4), _addr(sr4), ctypes.byref(c), _addr(xy), _addr(z), _addr(ell), _addr(con))
        return xy, z, ell, con

    def aabb(self, ell6):
        ell6 = _f32(ell6)
        out = np.zeros((ell6.shape[0], 4), np.float32)
        self.lib.gso_aabb(ell6.shape[0], _addr(ell6), _addr(out))
        return out

    def overlap(self, ell6, rect4):
        ell6, rect4 = _f32(ell6), _f32(rect4)
        out = np.zeros(ell6.shape[0], np.int32)
        self.lib.gso_overlap(ell6.shape[0], _addr(ell6), _addr(rect4), _addr(out))
        return out

    def key(self, tile, depth):
        tile = np.ascontiguousarray(tile, np.int32)
        depth = _f32(depth)
        out = np.zeros(tile.shape[0], np.uint64)
        self.lib.gso_key(tile.shape[0], _addr(tile), _addr(depth), _addr(out))
        return out

    def tile_counts(self, xy, ell, cam, rc):
        xy, ell = _f32(xy), _f32(ell)
        n = xy.shape[0]
        rect = np.zeros((n, 4), np.int32)
        cand = np.zeros(n, np.int32)
        hits = np.zeros(n, np.int32)
        c, g = camera(cam), cfg(rc)
        self.lib.gso_tile_counts(n, _addr(xy), _addr(ell), ctypes.byref(c), ctypes.byref(g), _addr(rect), _addr(cand),
                                 _addr(hits))
        return rect, cand, hits

    def build(self, xy, ell, z, cam, rc):
        xy, ell, z = _f32(xy), _f32(ell), _f32(z)
        n = xy.shape[0]
        c, g = camera(cam), cfg(rc)
        k = self.lib.gso_build(n, _addr(xy), _addr(ell), _addr(z), ctypes.byref(c), ctypes.byref(g), None, None, 0)
        keys = np.zeros(max(k, 1), np.uint64)
        vals = np.zeros(max(k, 1), np.int32)
        self.lib.gso_build(n, _addr(xy), _addr(ell), _addr(z), ctypes.byref(c), ctypes.byref(g), _addr(keys),
                           _addr(vals), k)
        return keys[:k], vals[:k]

    def sort(self, keys, vals, bits):
        keys = np.ascontiguousarray(keys, np.uint64).copy()
        vals = np.ascontiguousarray(vals, np.int32).copy()
        self.lib.gso_sort(keys.shape[0], _addr(keys), _addr(vals), bits)
        return keys, vals

    def ranges(self, keys, tiles):
        keys = np.ascontiguousarray(keys, np.uint64)
        r = np.full(2 * tiles, -1, np.int32)
        self.lib.gso_ranges(keys.shape[0], _addr(keys), tiles, _addr(r))
        return r

    def raster(self, cam, rc, ranges, vals, xy, conic, color, count_evals=False):
        c, g = camera(cam), cfg(rc)
        img = np.zeros((c.height, c.width, 4), np.uint8)
        ev = _I64(0)
        self.lib.gso_raster(ctypes.byref(c), ctypes.byref(g), _addr(np.ascontiguousarray(ranges, np.int32)),
                            _addr(np.ascontiguousarray(vals, np.int32)), _addr(_f32(xy)), _addr(_f32(conic)),
                            _addr(_f32(color)), _addr(img), ctypes.byref(ev))
        return (img, int(ev.value)) if count_evals else img

    def render(self, scene: dict, sh_grouped, cam, rc, key_capacity=1 << 40):
        """Whole frame; returns (image, K, evals, stage_ms[6])."""
        c, g = camera(cam), cfg(rc)
        img = np.zeros((c.height, c.width, 4), np.uint8)
        ev = _I64(0)
        ms = (ctypes.c_double * 6)()
        pos4, sr4 = _f32(scene["pos4"]), _f32(scene["sr4"])
        col = _f32(scene["color4"])
        sh = None if sh_grouped is None else _f32(sh_grouped)
        deg = scene["sh_degree"]
        k = self.lib.gso_render(pos4.shape[0], _addr(pos4), _addr(sr4), _addr(col), _addr(sh), deg,
                                3 * (deg + 1) ** 2, ctypes.byref(c), ctypes.byref(g), _addr(img), key_capacity,
                                ctypes.byref(ev), ms)
        return img, int(k), int(ev.value), list(ms)


_oracle = None


def get() -> Oracle:
    global _oracle
    if _oracle is None:
        _oracle = Oracle()
    return _oracle


# ---------------------------------------------------------------------------
# reference harness (GPU)
# ---------------------------------------------------------------------------

class Ref:
    """The reference's CUDA stages (oracle/_ref/libgsref.so); device pointers."""

    SCREEN = 1024
    TILES = 64 * 64

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/ref/build_ref.sh where the reference sources exist")
        self.lib = L = ctypes.CDLL(path)
        F = ctypes.c_float
        sig = {
            "gsref_set_global_args": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P,
                                                     ctypes.c_int, _P, _P]),
            "gsref_set_tile_list_args": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int]),
            "gsref_eval_sh": (F, [ctypes.c_int]),
            "gsref_eval_clip": (F, [ctypes.c_int]),
            "gsref_build": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(F)]),
            "gsref_sort": (F, [ctypes.c_int, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_int)]),
            "gsref_ranges": (F, [ctypes.c_int]),
            "gsref_raster": (F, []),
            "gsref_render_frame": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P,
                                                  ctypes.c_int, _P, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(F), ctypes.POINTER(F),
                                                  ctypes.POINTER(ctypes.c_int)]),
            "gsref_sync": (ctypes.c_int, []),
            "gsref_probe_overlap": (ctypes.c_int, [ctypes.c_int, _P, _P, _P]),
            "gsref_probe_aabb": (ctypes.c_int, [ctypes.c_int, _P, _P]),
            "gsref_probe_key": (ctypes.c_int, [ctypes.c_int, _P, _P, _P]),
            "gsref_cub_sort_timed": (F, [ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P, _P, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int)]),
        }
        for name, (res, args) in sig.items():
            if (name.startswith("gsref_probe_") or name == "gsref_cub_sort_timed") and not hasattr(L, name):
                continue  # the stage-compat build has neither the probes nor CUB
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args

    def time_frames(self, pos4, sr4, sh_grouped, sh_degree, cam, frames=30, warmup=3):
        """Renders the scene `warmup + frames` times with the reference's own
        frame loop (gsref_render_frame: every stage behind its blocking
        CudaTimer, the tile counter read back after the build, as
        app/main.cpp:360-432 runs it), growing the tile lists like the
        reference whenever they saturate.  Returns (image, K, per-frame ms of
        the timed frames (CUDA events around each whole frame), mean stage ms
        (sh, clip, build, sort, ranges, raster))."""
        import torch
        n = int(pos4.shape[0])
        dev = "cuda"
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        pos, sr = t(pos4), t(sr4)
        sh = t(sh_grouped)
        color = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        xy = torch.zeros((n, 2), dtype=torch.float32, device=dev)
        z = torch.zeros(n, dtype=torch.float32, device=dev)
        conic = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        ell = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        img = torch.zeros((self.SCREEN, self.SCREEN, 4), dtype=torch.uint8, device=dev)
        ranges = torch.zeros(2 * self.TILES, dtype=torch.int32, device=dev)
        cap = 8 * n  # app/main.cpp:305
        cam56 = self.camera56(cam)
        sh_count = 3 * (sh_degree + 1) ** 2
        while True:
            keys = [torch.zeros(cap, dtype=torch.int64, device=dev) for _ in range(2)]
            vals = [torch.zeros(cap, dtype=torch.int32, device=dev) for _ in range(2)]
            times, stage = [], []
            k = 0
            for f in range(frames + warmup):
                ms = (ctypes.c_float * 6)()
                fms = ctypes.c_float(0)
                sel = ctypes.c_int(0)
                k = self.lib.gsref_render_frame(cam56.ctypes.data, pos.data_ptr(), sr.data_ptr(), color.data_ptr(),
                                                sh_degree, sh_count, sh.data_ptr(), xy.data_ptr(), z.data_ptr(),
                                                conic.data_ptr(), ell.data_ptr(), n, img.data_ptr(),
                                                ranges.data_ptr(), keys[0].data_ptr(), keys[1].data_ptr(),
                                                vals[0].data_ptr(), vals[1].data_ptr(), cap, 148 * 8, ms,
                                                ctypes.byref(fms), ctypes.byref(sel))
                if k >= cap:
                    break
                if f >= warmup:
                    times.append(fms.value)
                    stage.append(list(ms))
            if k < cap:
                break
            cap *= 2  # saturated: the reference doubles its lists for the next frame (main.cpp:330-338)
        return img.cpu().numpy(), int(k), times, np.mean(np.array(stage), 0).tolist()

    @staticmethod
    def camera56(cam) -> np.ndarray:
        """CameraData (gaussian_render.cuh:16-25) from a gs_camera; the
        projection matrices are unused by the kernels and left zero."""
        c = getattr(cam, "c", cam)
        out = np.zeros(56, np.float32)
        out[32:48] = np.array(c.view, np.float32)
        out[48:50] = np.array(c.fov_cotangent, np.float32)
        out[50:52] = np.array(c.depth_scale_bias, np.float32)
        out[52:55] = np.array(c.position, np.float32)
        out[55] = c.aspect
        return out

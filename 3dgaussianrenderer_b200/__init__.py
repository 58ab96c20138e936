"""gs_b200: B200-native 3D Gaussian splatting frame pipeline.

Python binding of the C ABI in include/gs_b200.h (libgs_b200.so, built
in-tree for sm_100a by ``make -C 3dgaussianrenderer_b200/csrc``).  The
binding is thin: device memory comes from PyTorch tensors (or raw
pointers), every call goes straight to the CUDA library, and there is no
CPU fallback -- importing this module fails loudly when the library is
missing.

The package name starts with a digit, so import it with
``importlib.import_module("3dgaussianrenderer_b200")``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgs_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "gs_b200.h")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C {os.path.join(_HERE, 'csrc')}` "
        "(there is no CPU fallback)")

lib = ctypes.CDLL(LIB_PATH)

GS_OK = 0
GS_ERR_INVALID = 1
GS_ERR_OOM = 2
GS_ERR_CAPACITY = 3
GS_ERR_DEVICE_TIMEOUT = 4
GS_ERR_CUDA = 5
GS_ERR_NO_DEVICE = 6
GS_ERR_CANCELLED = 7
GS_TERM_REFERENCE = 0
GS_TERM_TMIN = 1
GS_ORDER_BUCKETS = 0
GS_ORDER_ONESWEEP = 1
GS_ORDER_AUTO = 2
GS_SCENE_KEEP_ORDER = 1


class GsError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = lib.gs_status_string(status).decode()
        detail = lib.gs_last_error_string().decode()
        super().__init__(f"{where}: {msg} ({detail})")


class gs_camera(ctypes.Structure):
    _fields_ = [
        ("view", ctypes.c_float * 16),
        ("position", ctypes.c_float * 3),
        ("fov_cotangent", ctypes.c_float * 2),
        ("depth_scale_bias", ctypes.c_float * 2),
        ("aspect", ctypes.c_float),
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
    ]


class gs_render_cfg(ctypes.Structure):
    _fields_ = [
        ("sh_max_degree", ctypes.c_int32),
        ("termination", ctypes.c_int32),
        ("t_min", ctypes.c_float),
        ("tile_w", ctypes.c_int32),
        ("tile_h", ctypes.c_int32),
        ("ordering", ctypes.c_int32),
        ("sort_variant", ctypes.c_int32),
        ("views_per_block", ctypes.c_int32),
        ("graph", ctypes.c_int32),
        ("raster_chunk", ctypes.c_int32),
        ("raster_persistent", ctypes.c_int32),
        ("sort_bits", ctypes.c_int32),
    ]


class gs_stats(ctypes.Structure):
    _fields_ = [
        ("sh_eval_ms", ctypes.c_double),
        ("project_ms", ctypes.c_double),
        ("build_tile_ms", ctypes.c_double),
        ("sort_ms", ctypes.c_double),
        ("raster_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("num_keys", ctypes.c_int64),
        ("num_tiles", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64),
        ("graph_replay", ctypes.c_int32),
        ("attempts", ctypes.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class gs_tune_result(ctypes.Structure):
    _fields_ = [("cfg", gs_render_cfg), ("ms", ctypes.c_double)]


class gs_frame_probe(ctypes.Structure):
    _fields_ = [("d_xy", ctypes.c_void_p), ("d_z", ctypes.c_void_p), ("d_ellipse", ctypes.c_void_p),
                ("d_conic", ctypes.c_void_p), ("d_color", ctypes.c_void_p)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_F = ctypes.c_float


def _sig(name, restype, *argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


_sig("gs_version", _I)
_sig("gs_status_string", ctypes.c_char_p, _I)
_sig("gs_last_error_string", ctypes.c_char_p)
_sig("gs_default_cfg", None, ctypes.POINTER(gs_render_cfg))
_sig("gs_camera_look_at", None, ctypes.POINTER(gs_camera), ctypes.POINTER(_F), ctypes.POINTER(_F),
     ctypes.POINTER(_F), _F, _I32, _I32, _F, _F)
_sig("gs_ctx_create", _I, _I, ctypes.POINTER(_P))
_sig("gs_ctx_destroy", _I, _P)
_sig("gs_ctx_device_bytes", _I64, _P)
_sig("gs_scene_create", _I, _P, _I64, _P, _P, _P, _P, _I32, ctypes.POINTER(_P))
_sig("gs_draw_stats", _I, _P, _I32, _I32, _I64, ctypes.POINTER(gs_stats), ctypes.c_double, _P)
_sig("gs_format_stats", _I, _I64, ctypes.POINTER(gs_stats), ctypes.c_double, ctypes.c_char_p, _I32)
_sig("gs_font_glyph", _I, _I32, ctypes.POINTER(ctypes.c_uint8))
_sig("gs_write_ppm", _I, ctypes.c_char_p, _P, _I32, _I32)
_sig("gs_write_png", _I, ctypes.c_char_p, _P, _I32, _I32)
_sig("gs_scene_create_ex", _I, _P, _I64, _P, _P, _P, _P, _I32, ctypes.c_uint32, ctypes.POINTER(_P))
_sig("gs_scene_destroy", _I, _P)
_sig("gs_scene_size", _I64, _P)
_sig("gs_scene_device_bytes", _I64, _P)
_sig("gs_render", _I, _P, _P, ctypes.POINTER(gs_camera), ctypes.POINTER(gs_render_cfg), _P,
     ctypes.POINTER(gs_stats), _P)
_sig("gs_render_host", _I, _P, _P, ctypes.POINTER(gs_camera), ctypes.POINTER(gs_render_cfg), _P,
     ctypes.POINTER(gs_stats), _P)
_sig("gs_render_batch", _I, _P, _P, ctypes.POINTER(gs_camera), _I32, ctypes.POINTER(gs_render_cfg),
     ctypes.POINTER(_P), ctypes.POINTER(gs_stats), _P)
_sig("gs_render_batch_host", _I, _P, _P, ctypes.POINTER(gs_camera), _I32, ctypes.POINTER(gs_render_cfg), _P,
     ctypes.POINTER(gs_stats), _P)
_sig("gs_autotune", _I, _P, _P, ctypes.POINTER(gs_camera), _I32, ctypes.POINTER(gs_render_cfg), _I32,
     ctypes.POINTER(gs_render_cfg), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(gs_tune_result), _I32,
     ctypes.POINTER(_I32), _P)
_sig("gs_autotune_lookup", _I, _P, _I64, _I32, _I32, _I32, ctypes.POINTER(gs_render_cfg), ctypes.POINTER(_I32))
_sig("gs_autotune_entries", _I32, _P)
_sig("gs_autotune_bucket", _I, _I64, _I32, _I32, _I32, ctypes.POINTER(_I32))
_sig("gs_stage_sh", _I, _I64, _P, _P, _I32, _I32, ctypes.POINTER(gs_camera), _P, _P)
_sig("gs_stage_project", _I, _I64, _P, _P, ctypes.POINTER(gs_camera), _P, _P, _P, _P, _P)
_sig("gs_stage_build", _I, _P, _I64, _P, _P, _P, ctypes.POINTER(gs_camera), ctypes.POINTER(gs_render_cfg), _P, _P,
     _I64, ctypes.POINTER(_I64), _P)
_sig("gs_stage_sort", _I, _P, _I64, _I32, _P, _P, _P, _P, ctypes.POINTER(_I32), _P)
_sig("gs_stage_ranges", _I, _I64, _P, _I64, _P, _P)
_sig("gs_probe_sort_timed", _I, _P, _I64, _I32, _P, _P, _P, _P, _P, _P, _I32, ctypes.POINTER(_I32),
     ctypes.POINTER(ctypes.c_double))
_sig("gs_stage_raster", _I, ctypes.POINTER(gs_camera), ctypes.POINTER(gs_render_cfg), _P, _P, _P, _P, _P, _P, _P)
_sig("gs_probe_frame", _I, _P, _P, ctypes.POINTER(gs_camera), _I32, ctypes.POINTER(gs_render_cfg), ctypes.POINTER(_P),
     ctypes.POINTER(gs_frame_probe), ctypes.POINTER(gs_stats), _P)
_sig("gs_probe_tile_lists", _I, _P, _P, _I64, _P, _P, _I64, _P, _I64, ctypes.POINTER(_I64), ctypes.POINTER(_I32))
_sig("gs_test_fail_allocations", None, _I32, _I32)
_sig("gs_test_pending_allocation_failures", _I32)
_sig("gs_test_bounded_wait", _I, _I32, _P)
_sig("gs_num_tiles", _I64, _I32, _I32, ctypes.POINTER(gs_render_cfg))
_sig("gs_key_bits", _I32, _I64)


def check(status: int, where: str) -> None:
    if status != GS_OK:
        raise GsError(status, where)


def _ptr(x) -> int | None:
    """Device/host address of a torch tensor, numpy array or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ---------------------------------------------------------------------------
# Camera (core/camera.h:11-59) and render options
# ---------------------------------------------------------------------------

class Camera:
    """Pinhole camera with the reference Camera's setters and getters
    (core/camera.h:11-59).  Depth uses the built frame loop's convention
    (app/main.cpp:352-358): clip z = -2/(f-n) * z_view - (f+n)/(f-n)."""

    def __init__(self):
        self._fovy = np.radians(50.0)
        self._w, self._h = 1024, 1024
        self._near, self._far = 0.01, 100.0
        self._eye = np.array([0.0, 0.0, 3.0], np.float32)
        self._target = np.zeros(3, np.float32)
        self._up = np.array([0.0, 1.0, 0.0], np.float32)
        self._update()

    def SetFovY(self, fov_y_rad: float):
        self._fovy = float(fov_y_rad)
        self._update()

    def SetResolution(self, width: int, height: int):
        self._w, self._h = int(width), int(height)
        self._update()

    def SetNearFar(self, near: float, far: float):
        self._near, self._far = float(near), float(far)
        self._update()

    def SetPose(self, position, look_at, up=(0.0, 1.0, 0.0)):
        self._eye = np.asarray(position, np.float32)
        self._target = np.asarray(look_at, np.float32)
        self._up = np.asarray(up, np.float32)
        self._update()

    def _update(self):
        c = gs_camera()
        eye = (_F * 3)(*self._eye.tolist())
        tgt = (_F * 3)(*self._target.tolist())
        up = (_F * 3)(*self._up.tolist())
        lib.gs_camera_look_at(ctypes.byref(c), eye, tgt, up, _F(self._fovy), self._w, self._h, _F(self._near),
                              _F(self._far))
        self.c = c

    def GetView(self):
        return np.array(self.c.view, np.float32).reshape(4, 4)  # [col][row]

    def GetPosition(self):
        return np.array(self.c.position, np.float32)

    def GetAspect(self):
        return float(self.c.aspect)

    def GetFovCotangent(self):
        return np.array(self.c.fov_cotangent, np.float32)

    def GetDepthScaleBias(self):
        return np.array(self.c.depth_scale_bias, np.float32)

    def GetWidth(self):
        return self._w

    def GetHeight(self):
        return self._h

    def GetFovY(self):
        return self._fovy

    def GetZNear(self):
        return self._near

    def GetZFar(self):
        return self._far


def look_at(eye, target, up=(0.0, 1.0, 0.0), fovy_deg=50.0, width=1024, height=1024, near=0.1, far=100.0) -> Camera:
    cam = Camera()
    cam._fovy = float(np.radians(fovy_deg))
    cam._w, cam._h = int(width), int(height)
    cam._near, cam._far = float(near), float(far)
    cam._eye = np.asarray(eye, np.float32)
    cam._target = np.asarray(target, np.float32)
    cam._up = np.asarray(up, np.float32)
    cam._update()
    return cam


@dataclass
class RenderConfig:
    """Pipeline options (gs_render_cfg).  reference() gives the reference
    renderer's behaviour (SH degree <= 2, tile-wide T <= 0.02 termination
    at 32-entry granularity); the default is full SH-3 with per-pixel
    T < 1e-4 termination."""
    sh_max_degree: int = 3
    termination: int = GS_TERM_TMIN
    t_min: float = 1e-4
    tile_w: int = 16
    tile_h: int = 16
    ordering: int = 0  # GS_ORDER_BUCKETS
    sort_variant: int = 0
    views_per_block: int = 0
    graph: int = 1
    raster_chunk: int = 0       # T_min raster: Gaussians per shared-memory batch (0 = 32, or 64)
    raster_persistent: int = 0  # T_min raster: persistent CTAs over the atomic tile queue
    sort_bits: int = 0          # per-tile sort: radix-sorted top depth bits (0 = 16, 8..32)

    @staticmethod
    def reference() -> "RenderConfig":
        return RenderConfig(sh_max_degree=2, termination=GS_TERM_REFERENCE, t_min=1e-4, tile_w=16, tile_h=16)

    def c(self) -> gs_render_cfg:
        return gs_render_cfg(self.sh_max_degree, self.termination, self.t_min, self.tile_w, self.tile_h,
                             self.ordering, self.sort_variant, self.views_per_block, self.graph, self.raster_chunk,
                             self.raster_persistent, self.sort_bits)


def num_tiles(width: int, height: int, cfg: RenderConfig) -> int:
    c = cfg.c()
    return int(lib.gs_num_tiles(width, height, ctypes.byref(c)))


def key_bits(tiles: int) -> int:
    return int(lib.gs_key_bits(tiles))


# ---------------------------------------------------------------------------
# Context / scene / frame
# ---------------------------------------------------------------------------

class Context:
    def __init__(self, device: int = 0):
        h = _P()
        check(lib.gs_ctx_create(device, ctypes.byref(h)), "gs_ctx_create")
        self.h = h

    def close(self):
        if self.h:
            lib.gs_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_bytes(self) -> int:
        return int(lib.gs_ctx_device_bytes(self.h))


class Scene:
    """Device-resident scene (Renderer::UploadModel)."""

    def __init__(self, ctx: Context, pos4: np.ndarray, sr4: np.ndarray, sh_grouped: np.ndarray | None,
                 sh_degree: int, color4: np.ndarray | None = None, keep_order: bool = False):
        """keep_order: store the Gaussians in the caller's order
        (GS_SCENE_KEEP_ORDER) instead of Morton order of their centres."""
        self.ctx = ctx
        pos4 = np.ascontiguousarray(pos4, np.float32)
        sr4 = np.ascontiguousarray(sr4, np.float32)
        n = pos4.shape[0]
        col = None if color4 is None else np.ascontiguousarray(color4, np.float32)
        sh = None if sh_grouped is None else np.ascontiguousarray(sh_grouped, np.float32)
        h = _P()
        check(lib.gs_scene_create_ex(ctx.h, n, _ptr(pos4), _ptr(sr4), _ptr(col), _ptr(sh), sh_degree,
                                     GS_SCENE_KEEP_ORDER if keep_order else 0, ctypes.byref(h)),
              "gs_scene_create_ex")
        self.h = h
        self.n = n
        self.sh_degree = sh_degree

    def close(self):
        if self.h:
            lib.gs_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render(ctx: Context, scene: Scene, cam: Camera, cfg: RenderConfig, out_rgba, stream=None) -> dict:
    """Renders into a device tensor (uint8, H*W*4)."""
    st = gs_stats()
    c = cfg.c()
    check(lib.gs_render(ctx.h, scene.h, ctypes.byref(cam.c), ctypes.byref(c), _ptr(out_rgba), ctypes.byref(st),
                        _stream_ptr(stream)), "gs_render")
    return st.as_dict()


def render_host(ctx: Context, scene: Scene, cam: Camera, cfg: RenderConfig, out: np.ndarray | None = None,
                stream=None):
    """Renders into host memory; returns (image HxWx4 uint8, stats)."""
    if out is None:
        out = np.zeros((cam.GetHeight(), cam.GetWidth(), 4), np.uint8)
    st = gs_stats()
    c = cfg.c()
    check(lib.gs_render_host(ctx.h, scene.h, ctypes.byref(cam.c), ctypes.byref(c), _ptr(out), ctypes.byref(st),
                             _stream_ptr(stream)), "gs_render_host")
    return out, st.as_dict()


def render_batch(ctx: Context, scene: Scene, cams: list, cfg: RenderConfig, outs: list, stream=None) -> dict:
    arr = (gs_camera * len(cams))(*[c.c for c in cams])
    ptrs = (_P * len(outs))(*[_ptr(o) for o in outs])
    st = gs_stats()
    c = cfg.c()
    check(lib.gs_render_batch(ctx.h, scene.h, arr, len(cams), ctypes.byref(c), ptrs, ctypes.byref(st),
                              _stream_ptr(stream)), "gs_render_batch")
    return st.as_dict()


def render_batch_host(ctx: Context, scene: Scene, cams: list, cfg: RenderConfig, out: np.ndarray,
                      stream=None) -> dict:
    arr = (gs_camera * len(cams))(*[c.c for c in cams])
    st = gs_stats()
    c = cfg.c()
    check(lib.gs_render_batch_host(ctx.h, scene.h, arr, len(cams), ctypes.byref(c), _ptr(out), ctypes.byref(st),
                                   _stream_ptr(stream)), "gs_render_batch_host")
    return st.as_dict()


def probe_frame(ctx: Context, scene: Scene, cams: list, cfg: RenderConfig, outs: list, xy, z, ell, conic,
                color=None, stream=None) -> dict:
    """A tile-bucket frame (as render_batch, never a graph replay) that also
    writes, per (view, Gaussian) at view * n + caller index, the projected
    centre, depth, ellipse and conic (and the colour of the Gaussians that
    reach a tile) into the given device tensors."""
    arr = (gs_camera * len(cams))(*[c.c for c in cams])
    ptrs = (_P * len(outs))(*[_ptr(o) for o in outs])
    pr = gs_frame_probe(_ptr(xy), _ptr(z), _ptr(ell), _ptr(conic), _ptr(color))
    st = gs_stats()
    c = cfg.c()
    check(lib.gs_probe_frame(ctx.h, scene.h, arr, len(cams), ctypes.byref(c), ptrs, ctypes.byref(pr),
                             ctypes.byref(st), _stream_ptr(stream)), "gs_probe_frame")
    return st.as_dict()


def probe_tile_lists(ctx: Context) -> dict:
    """Tile lists of the context's last tile-bucket frame: ranges (T, 2),
    keys as emitted (depth << 32 | slot), order (slots in blend order of the
    tiles larger than fused_cap), slot_index (view * n + caller index)."""
    sizes = (_I64 * 3)()
    cap = _I32()
    check(lib.gs_probe_tile_lists(ctx.h, None, 0, None, None, 0, None, 0, sizes, ctypes.byref(cap)),
          "gs_probe_tile_lists")
    T, K, S = (int(x) for x in sizes)
    ranges = np.zeros(2 * max(T, 1), np.int32)
    keys = np.zeros(max(K, 1), np.uint64)
    order = np.zeros(max(K, 1), np.int32)
    slots = np.zeros(max(S, 1), np.int32)
    check(lib.gs_probe_tile_lists(ctx.h, _ptr(ranges), ranges.size, _ptr(keys), _ptr(order), keys.size, _ptr(slots),
                                  slots.size, sizes, ctypes.byref(cap)), "gs_probe_tile_lists")
    return {"ranges": ranges[:2 * T].reshape(T, 2), "keys": keys[:K], "order": order[:K], "slot_index": slots[:S],
            "fused_cap": cap.value}


def _from_c(c: gs_render_cfg) -> "RenderConfig":
    return RenderConfig(c.sh_max_degree, c.termination, c.t_min, c.tile_w, c.tile_h, c.ordering, c.sort_variant,
                        c.views_per_block, c.graph, c.raster_chunk, c.raster_persistent, c.sort_bits)


def autotune(ctx: Context, scene: Scene, cams: list, cfg: RenderConfig, iterations: int = 5, stream=None):
    """Times the batching knobs (tile shape, views per block, onesweep tile
    shape) on this batch and stores the fastest in the context's table for
    the batch's (N, resolution, views) bucket.  Returns (best RenderConfig,
    its ms per batch, [(RenderConfig, ms) of every timed candidate])."""
    arr = (gs_camera * len(cams))(*[c.c for c in cams])
    c = cfg.c()
    best = gs_render_cfg()
    best_ms = ctypes.c_double()
    res = (gs_tune_result * 64)()
    count = _I32()
    check(lib.gs_autotune(ctx.h, scene.h, arr, len(cams), ctypes.byref(c), iterations, ctypes.byref(best),
                          ctypes.byref(best_ms), res, 64, ctypes.byref(count), _stream_ptr(stream)), "gs_autotune")
    return _from_c(best), best_ms.value, [(_from_c(r.cfg), r.ms) for r in res[:min(count.value, 64)]]


def autotune_bucket(n: int, width: int, height: int, num_views: int) -> tuple:
    """(floor log2 N, floor log2 pixels, view-count class) of a batch: the
    key of the tuning table."""
    b = (_I32 * 3)()
    check(lib.gs_autotune_bucket(n, width, height, num_views, b), "gs_autotune_bucket")
    return tuple(b)


def autotune_lookup(ctx: Context, n: int, width: int, height: int, num_views: int, cfg: RenderConfig):
    """The tuned knobs of the bucket applied to cfg, or None when the bucket
    was not tuned."""
    c = cfg.c()
    found = _I32()
    check(lib.gs_autotune_lookup(ctx.h, n, width, height, num_views, ctypes.byref(c), ctypes.byref(found)),
          "gs_autotune_lookup")
    return _from_c(c) if found.value else None


# ---------------------------------------------------------------------------
# Stage API (core/gaussian_render.cuh:113-126 equivalents)
# ---------------------------------------------------------------------------

def stage_sh(n, d_pos, d_sh, sh_count, eval_degree, cam: Camera, d_color, stream=None):
    check(lib.gs_stage_sh(n, _ptr(d_pos), _ptr(d_sh), sh_count, eval_degree, ctypes.byref(cam.c), _ptr(d_color),
                          _stream_ptr(stream)), "gs_stage_sh")


def stage_project(n, d_pos, d_sr, cam: Camera, d_xy, d_z, d_ell, d_conic, stream=None):
    check(lib.gs_stage_project(n, _ptr(d_pos), _ptr(d_sr), ctypes.byref(cam.c), _ptr(d_xy), _ptr(d_z), _ptr(d_ell),
                               _ptr(d_conic), _stream_ptr(stream)), "gs_stage_project")


def stage_build(ctx: Context, n, d_xy, d_z, d_ell, cam: Camera, cfg: RenderConfig, d_keys, d_values, capacity,
                stream=None) -> int:
    k = _I64(0)
    c = cfg.c()
    status = lib.gs_stage_build(ctx.h, n, _ptr(d_xy), _ptr(d_z), _ptr(d_ell), ctypes.byref(cam.c), ctypes.byref(c),
                                _ptr(d_keys), _ptr(d_values), capacity, ctypes.byref(k), _stream_ptr(stream))
    if status == GS_ERR_CAPACITY:
        raise GsError(status, f"gs_stage_build (K={k.value})")
    check(status, "gs_stage_build")
    return int(k.value)


def stage_sort(ctx: Context, num_keys, bits, d_keys, d_values, d_keys_alt, d_values_alt, stream=None) -> int:
    sel = _I32(0)
    check(lib.gs_stage_sort(ctx.h, num_keys, bits, _ptr(d_keys), _ptr(d_values), _ptr(d_keys_alt),
                            _ptr(d_values_alt), ctypes.byref(sel), _stream_ptr(stream)), "gs_stage_sort")
    return int(sel.value)


def probe_sort_timed(ctx: Context, num_keys, bits, src_keys, src_values, d_keys, d_values, d_keys_alt,
                     d_values_alt, iterations: int = 15):
    """gs_probe_sort_timed: the onesweep sort alone between CUDA events, the
    unsorted input restored before each of `iterations` runs.  Returns
    (selector, median ms)."""
    sel = _I32(0)
    ms = ctypes.c_double()
    check(lib.gs_probe_sort_timed(ctx.h, num_keys, bits, _ptr(src_keys), _ptr(src_values), _ptr(d_keys),
                                  _ptr(d_values), _ptr(d_keys_alt), _ptr(d_values_alt), iterations,
                                  ctypes.byref(sel), ctypes.byref(ms)), "gs_probe_sort_timed")
    return int(sel.value), ms.value


def stage_ranges(num_keys, d_keys, tiles, d_ranges, stream=None):
    check(lib.gs_stage_ranges(num_keys, _ptr(d_keys), tiles, _ptr(d_ranges), _stream_ptr(stream)), "gs_stage_ranges")


def _stats_struct(stats: dict) -> gs_stats:
    st = gs_stats()
    for name, _ in gs_stats._fields_:
        if name in stats:
            setattr(st, name, stats[name])
    return st


def draw_stats(d_rgba, width: int, height: int, num_gaussians: int, stats: dict, fps: float, stream=None):
    """Performance overlay (DrawPerformanceOverlay) into a device RGBA8 image."""
    st = _stats_struct(stats)
    check(lib.gs_draw_stats(_ptr(d_rgba), width, height, num_gaussians, ctypes.byref(st), float(fps),
                            _stream_ptr(stream)), "gs_draw_stats")


def format_stats(num_gaussians: int, stats: dict, fps: float) -> str:
    st = _stats_struct(stats)
    buf = ctypes.create_string_buffer(1024)
    check(lib.gs_format_stats(num_gaussians, ctypes.byref(st), float(fps), buf, len(buf)), "gs_format_stats")
    return buf.value.decode()


def write_image(path: str, rgba: np.ndarray) -> None:
    """Writes a host RGBA8 frame (H x W x 4, row 0 at the bottom as rendered)
    as .ppm or .png, top row first."""
    img = np.ascontiguousarray(rgba, np.uint8)
    if img.ndim != 3 or img.shape[2] != 4:
        raise ValueError("expected an H x W x 4 uint8 image")
    H, W = img.shape[:2]
    fn = lib.gs_write_png if path.lower().endswith(".png") else lib.gs_write_ppm
    check(fn(path.encode(), img.ctypes.data, W, H), "gs_write_png" if fn is lib.gs_write_png else "gs_write_ppm")


def font_glyph(c: str) -> list:
    rows = (ctypes.c_uint8 * 7)()
    check(lib.gs_font_glyph(ord(c), rows), "gs_font_glyph")
    return list(rows)


def stage_raster(cam: Camera, cfg: RenderConfig, d_ranges, d_values, d_xy, d_conic, d_color, d_rgba, stream=None):
    c = cfg.c()
    check(lib.gs_stage_raster(ctypes.byref(cam.c), ctypes.byref(c), _ptr(d_ranges), _ptr(d_values), _ptr(d_xy),
                              _ptr(d_conic), _ptr(d_color), _ptr(d_rgba), _stream_ptr(stream)), "gs_stage_raster")


# ---------------------------------------------------------------------------
# Serving (continuous batching over resident scenes)
# ---------------------------------------------------------------------------

class gs_server_cfg(ctypes.Structure):
    _fields_ = [
        ("budget_bytes", ctypes.c_int64),
        ("max_batch_views", ctypes.c_int32),
        ("num_workers", ctypes.c_int32),
        ("render", gs_render_cfg),
        ("batch_target_ms", ctypes.c_double),
    ]


class gs_server_stats(ctypes.Structure):
    _fields_ = [
        ("views_done", ctypes.c_int64),
        ("batches_done", ctypes.c_int64),
        ("max_batch", ctypes.c_int64),
        ("p50_ms", ctypes.c_double),
        ("p99_ms", ctypes.c_double),
        ("mean_ms", ctypes.c_double),
        ("views_per_s", ctypes.c_double),
        ("resident_bytes", ctypes.c_int64),
        ("frame_bytes", ctypes.c_int64),
        ("pending", ctypes.c_int64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_sig("gs_server_default_cfg", None, ctypes.POINTER(gs_server_cfg))
_sig("gs_server_create", _I, _I, ctypes.POINTER(gs_server_cfg), ctypes.POINTER(_P))
_sig("gs_server_destroy", _I, _P)
_sig("gs_server_add_scene", _I, _P, _I64, _P, _P, _P, _P, _I32, ctypes.POINTER(_I32))
_sig("gs_server_submit", _I, _P, _I32, ctypes.POINTER(gs_camera), _P, ctypes.POINTER(_I64))
_sig("gs_server_wait", _I, _P, _I64, ctypes.c_double, ctypes.POINTER(ctypes.c_double))
_sig("gs_server_get_stats", _I, _P, ctypes.POINTER(gs_server_stats))
_sig("gs_server_reset_stats", _I, _P)
_sig("gs_server_cancel", _I, _P, _I64)
_sig("gs_server_pause", _I, _P, _I32)
_sig("gs_ply_info", _I, ctypes.c_char_p, ctypes.POINTER(_I64), ctypes.POINTER(_I32))
_sig("gs_ply_last_error", ctypes.c_char_p)
_sig("gs_ply_read", _I, ctypes.c_char_p, _P, _P, _P, _P, _P)
_sig("gs_ply_write", _I, ctypes.c_char_p, _I64, _P, _P, _P, _P, _I32)


class Server:
    """Continuous-batching server (gs_server_*): resident scenes, requests
    from any thread, batched frames formed as workers free up."""

    def __init__(self, device: int = 0, budget_bytes: int = 150 << 30, max_batch_views: int = 16,
                 num_workers: int = 2, cfg: RenderConfig | None = None, batch_target_ms: float | None = None):
        c = gs_server_cfg()
        lib.gs_server_default_cfg(ctypes.byref(c))
        c.budget_bytes = budget_bytes
        c.max_batch_views = max_batch_views
        c.num_workers = num_workers
        if batch_target_ms is not None:
            c.batch_target_ms = batch_target_ms
        if cfg is not None:
            c.render = cfg.c()
        h = _P()
        check(lib.gs_server_create(device, ctypes.byref(c), ctypes.byref(h)), "gs_server_create")
        self.h = h

    def close(self):
        if self.h:
            lib.gs_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, pos4, sr4, sh_grouped, sh_degree, color4=None) -> int:
        pos4 = np.ascontiguousarray(pos4, np.float32)
        sr4 = np.ascontiguousarray(sr4, np.float32)
        sh = None if sh_grouped is None else np.ascontiguousarray(sh_grouped, np.float32)
        col = None if color4 is None else np.ascontiguousarray(color4, np.float32)
        sid = _I32(0)
        check(lib.gs_server_add_scene(self.h, pos4.shape[0], _ptr(pos4), _ptr(sr4), _ptr(col), _ptr(sh), sh_degree,
                                      ctypes.byref(sid)), "gs_server_add_scene")
        return int(sid.value)

    def submit(self, scene_id: int, cam: Camera, out: np.ndarray) -> int:
        rid = _I64(0)
        check(lib.gs_server_submit(self.h, scene_id, ctypes.byref(cam.c), _ptr(out), ctypes.byref(rid)),
              "gs_server_submit")
        return int(rid.value)

    def wait(self, rid: int, timeout_ms: float = 60_000.0) -> float:
        lat = ctypes.c_double(0)
        check(lib.gs_server_wait(self.h, rid, timeout_ms, ctypes.byref(lat)), "gs_server_wait")
        return float(lat.value)

    def wait_status(self, rid: int, timeout_ms: float = 60_000.0) -> int:
        """The request's completion status (GS_OK, GS_ERR_CANCELLED, ...)
        without raising."""
        lat = ctypes.c_double(0)
        return int(lib.gs_server_wait(self.h, rid, timeout_ms, ctypes.byref(lat)))

    def cancel(self, rid: int) -> int:
        """Cancels a queued request; GS_ERR_INVALID when it is already on the
        device, finished or unknown."""
        return int(lib.gs_server_cancel(self.h, rid))

    def pause(self, paused: bool = True):
        check(lib.gs_server_pause(self.h, 1 if paused else 0), "gs_server_pause")

    def stats(self) -> dict:
        s = gs_server_stats()
        check(lib.gs_server_get_stats(self.h, ctypes.byref(s)), "gs_server_get_stats")
        return s.as_dict()

    def reset_stats(self):
        check(lib.gs_server_reset_stats(self.h), "gs_server_reset_stats")


# ---------------------------------------------------------------------------
# PLY (parsePly / savePly)
# ---------------------------------------------------------------------------

def load_ply(path: str) -> dict:
    """Reads a 3DGS PLY with the reference's load transforms; returns a scene
    dict (pos4, sr4, color4, sh_grouped, sh_degree, n, bounds)."""
    n = _I64(0)
    deg = _I32(0)
    if lib.gs_ply_info(path.encode(), ctypes.byref(n), ctypes.byref(deg)) != GS_OK:
        raise ValueError(lib.gs_ply_last_error().decode())
    n, deg = int(n.value), int(deg.value)
    # every element is written by gs_ply_read (the last SH group's padding
    # included): no zero fill
    pos4 = np.empty((n, 4), np.float32)
    sr4 = np.empty((n, 4), np.float32)
    color4 = np.empty((n, 4), np.float32)
    groups = (n + 255) // 256
    sh = np.empty(groups * 256 * 3 * (deg + 1) ** 2, np.float32) if deg > 0 else None
    bounds = np.zeros(6, np.float32)
    if lib.gs_ply_read(path.encode(), _ptr(pos4), _ptr(sr4), _ptr(color4), _ptr(sh), _ptr(bounds)) != GS_OK:
        raise ValueError(lib.gs_ply_last_error().decode())
    return {"pos4": pos4, "sr4": sr4, "color4": color4, "sh_grouped": sh, "sh_degree": deg, "n": n,
            "bounds": bounds}


def save_ply(path: str, pos4, sr4, color4, sh_grouped, sh_degree: int):
    pos4 = np.ascontiguousarray(pos4, np.float32)
    sr4 = np.ascontiguousarray(sr4, np.float32)
    col = None if color4 is None else np.ascontiguousarray(color4, np.float32)
    sh = None if sh_grouped is None else np.ascontiguousarray(sh_grouped, np.float32)
    check(lib.gs_ply_write(path.encode(), pos4.shape[0], _ptr(pos4), _ptr(sr4), _ptr(col), _ptr(sh), sh_degree),
          "gs_ply_write")


from . import scenes  # noqa: E402,F401

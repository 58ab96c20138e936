"""PLY ingest (gs_ply_read / gs_ply_write) against the reference's own parsePly
(core/ply_parser.cpp, compiled into oracle/_ref/libplyref.so), on CPU."""
import ctypes
import os

import numpy as np
import pytest

from helpers import ROOT

PLYREF = os.path.join(ROOT, "oracle", "_ref", "libplyref.so")


def ref_parse(path):
    lib = ctypes.CDLL(PLYREF)
    lib.plyref_parse.restype = ctypes.c_int
    lib.plyref_parse.argtypes = [ctypes.c_char_p]
    lib.plyref_error.restype = ctypes.c_char_p
    n = lib.plyref_parse(path.encode())
    if n < 0:
        raise ValueError(lib.plyref_error().decode())
    deg, cnt = ctypes.c_int(0), ctypes.c_int(0)
    bounds = np.zeros(6, np.float32)
    lib.plyref_info(ctypes.byref(deg), ctypes.byref(cnt), bounds.ctypes.data_as(ctypes.c_void_p))
    pos = np.zeros((n, 4), np.float32)
    sr = np.zeros((n, 4), np.float32)
    col = np.zeros((n, 4), np.float32)
    sh = np.zeros((n, cnt.value), np.float32) if deg.value > 0 else None
    lib.plyref_copy(ctypes.c_void_p(pos.ctypes.data), ctypes.c_void_p(sr.ctypes.data),
                    ctypes.c_void_p(col.ctypes.data), ctypes.c_void_p(sh.ctypes.data) if sh is not None else None)
    return {"pos4": pos, "sr4": sr, "color4": col, "sh": sh, "sh_degree": deg.value, "bounds": bounds}


needs_ref = pytest.mark.skipif(not os.path.exists(PLYREF), reason="reference parsePly harness not built")


@needs_ref
@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_ply_read_matches_reference_parse(gs, tmp_path, deg):
    sc = gs.scenes.uniform_scene(3001, seed=40 + deg, sh_degree=deg, extent=3.0)
    rng = np.random.default_rng(deg)
    n = sc["n"]
    path = str(tmp_path / f"s{deg}.ply")
    # raw (pre-activation) values straight into the file, INRIA layout
    gs.scenes.write_ply(path, sc, log_scales=rng.normal(-4, 1, (n, 3)).astype(np.float32),
                        quats_wxyz=rng.normal(0, 1, (n, 4)).astype(np.float32),
                        opacity_logit=rng.normal(0, 2, n).astype(np.float32))
    ref = ref_parse(path)
    got = gs.load_ply(path)
    assert got["n"] == n and got["sh_degree"] == ref["sh_degree"] == deg
    for k in ("pos4", "color4"):
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
    # scales (exp) and the 8-bit quaternion bits
    assert np.array_equal(got["sr4"].view(np.uint32), ref["sr4"].view(np.uint32))
    assert np.array_equal(got["bounds"], ref["bounds"])
    if deg > 0:
        assert np.array_equal(got["sh_grouped"], gs.scenes.grouped_sh(ref["sh"]))


@needs_ref
def test_ply_write_read_round_trip(gs, tmp_path):
    sc = gs.scenes.cluster_scene(2000, 4, 2.0, seed=5, sh_degree=3)
    sh = gs.scenes.grouped_sh(sc["sh"])
    path = str(tmp_path / "rt.ply")
    gs.save_ply(path, sc["pos4"], sc["sr4"], sc["color4"], sh, 3)
    a = gs.load_ply(path)
    r = ref_parse(path)
    assert np.array_equal(a["pos4"].view(np.uint32), r["pos4"].view(np.uint32))
    np.testing.assert_allclose(a["pos4"][:, :3], sc["pos4"][:, :3])
    np.testing.assert_allclose(a["pos4"][:, 3], sc["pos4"][:, 3], rtol=1e-5)
    np.testing.assert_allclose(a["sr4"][:, :3], sc["sr4"][:, :3], rtol=1e-5)
    np.testing.assert_allclose(a["sh_grouped"], sh)
    # the quaternion goes through one decode/normalise/encode cycle: within one step
    qa = gs.scenes.decode_quat8(a["sr4"][:, 3].view(np.uint32))
    qs = gs.scenes.decode_quat8(sc["sr4"][:, 3].view(np.uint32))
    qs = qs / np.linalg.norm(qs, axis=1, keepdims=True)
    assert np.abs(qa - qs).max() <= 2.5 / 255 * 2


@pytest.mark.parametrize("header,msg", [
    (b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n", "Format"),
    (b"ply\nformat binary_little_endian 1.0\nelement face 1\nend_header\n", "element"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty double x\nend_header\n", "float"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\nproperty float x\nend_header\n",
     "Duplicated"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 0\nproperty float x\nend_header\n", "Missing"),
])
def test_ply_rejects_what_the_reference_rejects(gs, tmp_path, header, msg):
    path = str(tmp_path / "bad.ply")
    open(path, "wb").write(header)
    with pytest.raises(ValueError, match=msg):
        gs.load_ply(path)
    if os.path.exists(PLYREF):
        with pytest.raises(ValueError):
            ref_parse(path)


def test_ply_sh_degree_mismatch_rejected(gs, tmp_path):
    names = ["x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2", "f_dc_0",
             "f_dc_1", "f_dc_2", "f_rest_0", "f_rest_1", "opacity"]
    hdr = b"ply\nformat binary_little_endian 1.0\nelement vertex 1\n" + b"".join(
        f"property float {n}\n".encode() for n in names) + b"end_header\n"
    path = str(tmp_path / "bad_sh.ply")
    open(path, "wb").write(hdr + np.zeros(len(names), np.float32).tobytes())
    with pytest.raises(ValueError, match="extra spherical harmonics"):
        gs.load_ply(path)


def test_ply_truncated_vertex_data_rejected(gs, tmp_path):
    sc = gs.scenes.uniform_scene(300, seed=3, sh_degree=1)
    path = str(tmp_path / "t.ply")
    gs.save_ply(path, sc["pos4"], sc["sr4"], sc["color4"], gs.scenes.grouped_sh(sc["sh"]), 1)
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-4])
    with pytest.raises(ValueError, match="truncated"):
        gs.load_ply(path)


@needs_ref
def test_ply_read_faster_than_reference_parse(gs, tmp_path):
    """The ingest row's measurement: the 1M-Gaussian SH-3 configuration
    scene as a 236 MB PLY, parsed into the device layouts by gs_ply_read
    (memory map + one thread per core) and by the reference's parsePly
    (per-float stream reads), best of a few runs each, same output."""
    import time
    sc = gs.scenes.config_scene("plain1m")
    path = str(tmp_path / "plain1m.ply")
    gs.save_ply(path, sc["pos4"], sc["sr4"], sc["color4"], gs.scenes.grouped_sh(sc["sh"]), 3)
    del sc

    def best(f, k):
        t = []
        for _ in range(k):
            t0 = time.perf_counter()
            out = f()
            t.append(time.perf_counter() - t0)
        return min(t), out

    t_ours, got = best(lambda: gs.load_ply(path), 3)
    t_ref, ref = best(lambda: ref_parse(path), 2)
    print(f"\nPLY ingest, 1M SH3 ({os.path.getsize(path) / 1e6:.0f} MB, {os.cpu_count()} cores): "
          f"gs_ply_read {t_ours * 1e3:.0f} ms, parsePly {t_ref * 1e3:.0f} ms ({t_ref / t_ours:.1f}x)")
    assert np.array_equal(got["pos4"].view(np.uint32), ref["pos4"].view(np.uint32))
    assert t_ref / t_ours >= 2.0

"""Seeded synthetic scenes and cameras, in the reference's buffer layouts.

A scene is a dict of numpy arrays:
  pos4   (n, 4) float32  x, y, z, opacity (sigmoid applied, ply_parser.cpp:377)
  sr4    (n, 4) float32  exp(log-scale) xyz, quantised quaternion bit-cast in w
  sh     (n, 3(d+1)^2) float32, RGB interleaved per coefficient
         (the reorder of ply_parser.cpp:332-348), or None for degree 0
  color4 (n, 4) float32  DC colour f_dc*C0 + 0.5 and opacity (ply_parser.cpp:383,389)
  sh_degree int

``grouped_sh`` produces the device layout [ceil(n/256)][coef][256]
(app/main.cpp:147-177).  ``write_ply`` stores a scene with the INRIA 3DGS
property names (f_rest channel-major), so the reference's parsePly reads
back the same buffers.
"""
from __future__ import annotations

import numpy as np

SH_C0 = np.float32(0.28209479177387814)


def sigmoid(x):
    x = np.asarray(x, np.float32)
    return (np.float32(1.0) / (np.float32(1.0) + np.exp(-x))).astype(np.float32)


def encode_quat8(q_xyzw: np.ndarray) -> np.ndarray:
    """encodeVec4((q + 1) * 0.5) of ply_parser.cpp:231-239,385: byte = (uint32)(clamp(v,0,1)*255),
    x in bits 31..24, y 23..16, z 15..8, w 7..0.  Returns uint32."""
    v = ((q_xyzw.astype(np.float32) + np.float32(1.0)) * np.float32(0.5)).astype(np.float32)
    v = np.clip(v, np.float32(0.0), np.float32(1.0))
    b = (v * np.float32(255.0)).astype(np.uint32)
    return (b[:, 0] << 24) | (b[:, 1] << 16) | (b[:, 2] << 8) | b[:, 3]


def decode_quat8(bits: np.ndarray) -> np.ndarray:
    b = np.stack([(bits >> 24) & 0xFF, (bits >> 16) & 0xFF, (bits >> 8) & 0xFF, bits & 0xFF], 1).astype(np.float32)
    return b / np.float32(255.0) * np.float32(2.0) - np.float32(1.0)


def _normalize_quat(q_wxyz: np.ndarray) -> np.ndarray:
    q = q_wxyz.astype(np.float32)
    n = np.sqrt((q * q).sum(1, keepdims=True)).astype(np.float32)
    n[n == 0] = 1
    return (q / n).astype(np.float32)


def make_scene(means, log_scales, quats_wxyz, opacity_logit, sh_coeffs, sh_degree):
    """Applies the load-time transforms of ply_parser.cpp:354-390."""
    n = means.shape[0]
    q = _normalize_quat(quats_wxyz)
    bits = encode_quat8(np.stack([q[:, 1], q[:, 2], q[:, 3], q[:, 0]], 1))
    scale = np.exp(log_scales.astype(np.float32)).astype(np.float32)
    opac = sigmoid(opacity_logit)
    pos4 = np.empty((n, 4), np.float32)
    pos4[:, :3] = means
    pos4[:, 3] = opac
    sr4 = np.empty((n, 4), np.float32)
    sr4[:, :3] = scale
    sr4[:, 3] = bits.view(np.float32)
    dc = sh_coeffs[:, 0:3]
    color4 = np.empty((n, 4), np.float32)
    color4[:, :3] = dc * SH_C0 + np.float32(0.5)
    color4[:, 3] = opac
    return {"pos4": pos4, "sr4": sr4, "sh": sh_coeffs.astype(np.float32) if sh_degree > 0 else None,
            "color4": color4, "sh_degree": sh_degree, "n": n}


def _sh(rng, n, degree):
    k = (degree + 1) ** 2
    sh = np.empty((n, 3 * k), np.float32)
    sh[:, :3] = rng.normal(0.0, 0.5, (n, 3))
    if k > 1:
        sh[:, 3:] = rng.normal(0.0, 0.05, (n, 3 * (k - 1)))
    return sh


def _quats(rng, n):
    return rng.normal(0.0, 1.0, (n, 4)).astype(np.float32)


def uniform_scene(n: int, seed: int = 1, sh_degree: int = 3, extent: float = 1.0, log_scale_mu: float = -4.0,
                  log_scale_sigma: float = 0.5):
    """Means uniform in [-extent, extent]^3, log-scales N(mu, sigma), random unit
    quaternions, opacity sigmoid(N(0, 1.5)), SH DC N(0, 0.5), rest N(0, 0.05)."""
    rng = np.random.default_rng(seed)
    means = rng.uniform(-extent, extent, (n, 3)).astype(np.float32)
    ls = rng.normal(log_scale_mu, log_scale_sigma, (n, 3)).astype(np.float32)
    q = _quats(rng, n)
    op = rng.normal(0.0, 1.5, n).astype(np.float32)
    return make_scene(means, ls, q, op, _sh(rng, n, sh_degree), sh_degree)


def cluster_scene(n: int, clusters: int, extent: float, seed: int = 1, sh_degree: int = 3,
                  log_scale_mu: float = -5.0, log_scale_sigma: float = 0.7):
    """Mixture of `clusters` anisotropic Gaussians: centres uniform in
    [-extent, extent]^3, per-cluster diagonal covariance ~U(0.05, 1)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-extent, extent, (clusters, 3)).astype(np.float32)
    var = rng.uniform(0.05, 1.0, (clusters, 3)).astype(np.float32)
    which = rng.integers(0, clusters, n)
    means = (centres[which] + rng.normal(0.0, 1.0, (n, 3)).astype(np.float32) * np.sqrt(var[which])).astype(
        np.float32)
    ls = rng.normal(log_scale_mu, log_scale_sigma, (n, 3)).astype(np.float32)
    q = _quats(rng, n)
    op = rng.normal(0.0, 1.5, n).astype(np.float32)
    return make_scene(means, ls, q, op, _sh(rng, n, sh_degree), sh_degree)


def grouped_sh(sh: np.ndarray, group: int = 256) -> np.ndarray:
    """realignSphericalHarmonics (app/main.cpp:147-177): [group][coef][256], zero padded."""
    n, c = sh.shape
    g = (n + group - 1) // group
    pad = np.zeros((g * group, c), np.float32)
    pad[:n] = sh
    return np.ascontiguousarray(pad.reshape(g, group, c).transpose(0, 2, 1)).reshape(-1)


# ---------------------------------------------------------------------------
# configs
# ---------------------------------------------------------------------------

def config_scene(name: str, seed: int | None = None):
    """Scenes of the five benchmark configurations (seeded)."""
    if name == "plain100k":
        return uniform_scene(100_000, seed=seed or 11, sh_degree=3)
    if name == "plain1m":
        return cluster_scene(1_000_000, 64, 5.0, seed=seed or 12, log_scale_mu=-5.0, log_scale_sigma=0.7)
    if name == "batch3m":
        return cluster_scene(3_000_000, 256, 10.0, seed=seed or 13, log_scale_mu=-5.0, log_scale_sigma=0.7)
    if name == "stress10m":
        return cluster_scene(10_000_000, 256, 10.0, seed=seed or 15, log_scale_mu=-2.5, log_scale_sigma=0.8)
    raise KeyError(name)


def sphere_pose(rng, radius: float):
    """Uniform direction on a sphere, rejecting near-vertical poses (|y|/r > 0.99)."""
    while True:
        d = rng.normal(0.0, 1.0, 3)
        d /= np.linalg.norm(d)
        if abs(d[1]) <= 0.99:
            return (d * radius).astype(np.float32)


def orbit_ring(num: int, radius: float, seed: int):
    """`num` eyes evenly spaced on a horizontal ring with a seeded phase and height."""
    rng = np.random.default_rng(seed)
    phase = rng.uniform(0, 2 * np.pi)
    height = rng.uniform(-0.2, 0.2) * radius
    eyes = []
    for k in range(num):
        a = phase + 2 * np.pi * k / num
        eyes.append(np.array([radius * np.cos(a), height, radius * np.sin(a)], np.float32))
    return eyes


BATCH_RESOLUTIONS = [(1280, 720), (1600, 900), (1920, 1080)]


def write_ply(path: str, scene: dict, log_scales=None, quats_wxyz=None, opacity_logit=None):
    """Binary little-endian PLY with INRIA 3DGS property names.  When the raw
    (pre-activation) values are not given they are recovered from the scene
    buffers (log of scale, logit of opacity, decoded quaternion)."""
    n = scene["n"]
    pos = scene["pos4"][:, :3]
    if log_scales is None:
        log_scales = np.log(scene["sr4"][:, :3])
    if quats_wxyz is None:
        q = decode_quat8(scene["sr4"][:, 3].view(np.uint32))
        quats_wxyz = np.stack([q[:, 3], q[:, 0], q[:, 1], q[:, 2]], 1)
    if opacity_logit is None:
        o = np.clip(scene["pos4"][:, 3], 1e-6, 1 - 1e-6)
        opacity_logit = np.log(o / (1 - o))
    deg = scene["sh_degree"]
    if deg > 0:
        sh = scene["sh"]
        k = (deg + 1) ** 2
        dc = sh[:, :3]
        rest = sh[:, 3:].reshape(n, k - 1, 3).transpose(0, 2, 1).reshape(n, 3 * (k - 1))  # channel-major
    else:
        dc = (scene["color4"][:, :3] - np.float32(0.5)) / SH_C0
        rest = np.zeros((n, 0), np.float32)
    names = ["x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2",
             "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(rest.shape[1])] + ["opacity"]
    cols = np.concatenate([pos, quats_wxyz, log_scales, dc, rest, opacity_logit.reshape(n, 1)], 1).astype(
        np.float32)
    with open(path, "wb") as f:
        f.write(b"ply\nformat binary_little_endian 1.0\n")
        f.write(f"element vertex {n}\n".encode())
        for nm in names:
            f.write(f"property float {nm}\n".encode())
        f.write(b"end_header\n")
        f.write(np.ascontiguousarray(cols).tobytes())

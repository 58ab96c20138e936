"""The margin rule of the frame kernel's cheap ellipse/tile overlap test
(ellipse_rect_overlap_clear in 3dgaussianrenderer_b200/csrc/gs_common.cuh),
restated in single precision with numpy, against the oracle's IEEE test
(core/gaussian_render.cu:250-272 via oracle/gs_oracle.c).

The cheap evaluation computes the tile's corners in ellipse coordinates as
a parallelogram with hardware reciprocals and compares the rectangle centre
and, of each pair of parallel edges, the nearer one; it may only decide a
candidate when every compared value lies more than 256 u R + 2^-15 from 1 (u = 2^-24,
R = image-space corner offset / smallest extent).  Here every decided
candidate must agree with the oracle, with the reciprocals perturbed by one
ulp either way, and the measured difference of the compared values must stay
far inside the margin.  Splats with a zero extent (the trace bump leaves
lambda1 = 0 for sub-pixel splats) overlap a tile only when their centre lies
inside it.
"""
import numpy as np
import pytest

f = np.float32
U = 2.0 ** -24


def _cases(n, seed):
    rng = np.random.default_rng(seed)
    W = 1920.0
    px = 2.0 / W
    ey = rng.uniform(1.69, 40, n) * px
    ex = ey * np.exp(rng.uniform(0, np.log(1500), n))
    ang = rng.uniform(-np.pi, np.pi, n)
    cs, sn = np.cos(ang), np.sin(ang)
    cx, cy = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    tc = f(16 * 2.0 / W)
    # a candidate tile inside the splat's bounding box
    bx = np.abs(cs * ex) + np.abs(sn * ey)
    by = np.abs(sn * ex) + np.abs(cs * ey)
    gx = np.floor((cx + rng.uniform(-1, 1, n) * bx + 1) / tc).astype(f)
    gy = np.floor((cy + rng.uniform(-1, 1, n) * by + 1) / tc).astype(f)
    x0 = (gx * tc - f(1)).astype(f)
    y0 = (gy * tc - f(1)).astype(f)
    e = [a.astype(f) for a in (cx, cy, cs, sn, ex, ey)]
    return e, (x0, y0, (x0 + tc).astype(f), (y0 + tc).astype(f))


def _rcp(x, jitter):
    with np.errstate(divide="ignore"):
        return ((f(1) / x) * (f(1) + f(jitter * 2.0 ** -23))).astype(f)


def _cheap(e, r, jitter):
    """The five compared values and the margin, in the kernel's order."""
    cx, cy, cs, sn, ex, ey = e
    x0, y0, x1, y1 = r
    with np.errstate(all="ignore"):
        iex, iey = _rcp(ex, jitter), _rcp(ey, -jitter)
        dx0, dy0 = (x0 - cx).astype(f), (y0 - cy).astype(f)
        ax = ((dx0 * cs + dy0 * sn) * iex).astype(f)
        ay = ((dy0 * cs - dx0 * sn) * iey).astype(f)
        w, h = (x1 - x0).astype(f), (y1 - y0).astype(f)
        ux, uy = ((w * cs) * iex).astype(f), (-(w * sn) * iey).astype(f)
        vx, vy = ((h * sn) * iex).astype(f), ((h * cs) * iey).astype(f)
        R = ((np.abs(dx0) + np.abs(dy0) + w + h) * np.maximum(np.abs(iex), np.abs(iey))).astype(f)
        margin = (R * f(256.0 / 16777216.0) + f(1.0 / 32768.0)).astype(f)
        vals = [((ax + f(0.5) * (ux + vx)) ** 2 + (ay + f(0.5) * (uy + vy)) ** 2).astype(f)]
        iu = _rcp((ux * ux + uy * uy).astype(f), jitter)
        iv = _rcp((vx * vx + vy * vy).astype(f), -jitter)

        def edge(px_, py_, dx_, dy_, inv):
            t = np.clip(-(px_ * dx_ + py_ * dy_) * inv, 0, 1).astype(f)
            qx, qy = (px_ + t * dx_).astype(f), (py_ + t * dy_).astype(f)
            return (qx * qx + qy * qy).astype(f)

        bx, by = (ax + ux).astype(f), (ay + uy).astype(f)
        qcx, qcy = (bx + vx).astype(f), (by + vy).astype(f)
        qx, qy = (ax + vx).astype(f), (ay + vy).astype(f)
        vals += [edge(ax, ay, ux, uy, iu), edge(bx, by, vx, vy, iv), edge(qcx, qcy, -ux, -uy, iu),
                 edge(qx, qy, -vx, -vy, iv)]
    return np.stack(vals), margin, R


def _cheap_nearer(e, r, jitter):
    """The values the kernel compares: the rectangle centre and, of each
    pair of parallel edges, the one on the line nearer the origin (chosen by
    cross products, as in the kernel)."""
    cx, cy, cs, sn, ex, ey = e
    x0, y0, x1, y1 = r
    vals5, margin, _ = _cheap(e, r, jitter)
    with np.errstate(all="ignore"):
        iex, iey = _rcp(ex, jitter), _rcp(ey, -jitter)
        dx0, dy0 = (x0 - cx).astype(f), (y0 - cy).astype(f)
        ax = ((dx0 * cs + dy0 * sn) * iex).astype(f)
        ay = ((dy0 * cs - dx0 * sn) * iey).astype(f)
        w, h = (x1 - x0).astype(f), (y1 - y0).astype(f)
        ux, uy = ((w * cs) * iex).astype(f), (-(w * sn) * iey).astype(f)
        vx, vy = ((h * sn) * iex).astype(f), ((h * cs) * iey).astype(f)
        su = (ax * uy - ay * ux).astype(f)
        kuv = (vx * uy - vy * ux).astype(f)
        sv = (ax * vy - ay * vx).astype(f)
        u_at_a = np.abs(su) <= np.abs((su + kuv).astype(f))
        v_at_a = np.abs(sv) <= np.abs((sv - kuv).astype(f))
    # vals5: centre, edge (a, u), edge (a + u, v), edge (a + u + v, -u), edge (a + v, -v)
    eu = np.where(u_at_a, vals5[1], vals5[3])
    ev = np.where(v_at_a, vals5[4], vals5[2])
    return np.stack([vals5[0], eu, ev]), margin


def _decide(e, r, jitter):
    """1 / 0 / -1 as ellipse_rect_overlap_clear, after the caller's centre test."""
    vals, margin = _cheap_nearer(e, r, jitter)
    zero = (e[4] == 0) | (e[5] == 0)
    with np.errstate(invalid="ignore"):
        hit = np.any(vals < 1 - margin, axis=0)
        miss = np.all(vals > 1 + margin, axis=0)
    d = np.where(hit, 1, np.where(miss, 0, -1))
    d = np.where(~(margin <= 0.125), -1, d)
    return np.where(zero, 0, d)


def _centre(e, r):
    return (e[0] > r[0]) & (e[0] < r[2]) & (e[1] > r[1]) & (e[1] < r[3])


@pytest.mark.parametrize("seed", [7, 8])
def test_decided_candidates_agree_with_ieee(O, seed):
    e, r = _cases(200_000, seed)
    ref = O.overlap(np.stack(e, 1), np.stack(r, 1)).astype(bool)
    centre = _centre(e, r)
    for jitter in (0, 1, -1):
        d = _decide(e, r, jitter)
        decided = ~centre & (d >= 0)
        assert np.array_equal((d[decided] == 1), ref[decided])
        # undecided candidates are rare
        assert np.count_nonzero(~centre & (d < 0)) <= 0.002 * centre.size


def test_value_difference_far_inside_margin(O):
    """The compared values against the reference's own rounding of them
    (glm order, contracted or not): the measured gap is a small fraction
    of the margin at every R."""
    e, r = _cases(200_000, 9)
    cx, cy, cs, sn, ex, ey = e
    x0, y0, x1, y1 = r

    def to_e(px_, py_, fma):
        dx, dy = (px_ - cx).astype(f), (py_ - cy).astype(f)
        if fma:
            nx = (dx.astype(np.float64) * cs + (dy * sn).astype(f)).astype(f)
            ny = (dy.astype(np.float64) * cs - (dx * sn).astype(f)).astype(f)
        else:
            nx, ny = (dx * cs + dy * sn).astype(f), (dy * cs - dx * sn).astype(f)
        return (nx / ex).astype(f), (ny / ey).astype(f)

    def seg(a, b):
        dx, dy = (b[0] - a[0]).astype(f), (b[1] - a[1]).astype(f)
        t = np.clip((-a[0] * dx + -a[1] * dy) / (dx * dx + dy * dy).astype(f), 0, 1).astype(f)
        prx, pry = (a[0] + t * dx).astype(f), (a[1] + t * dy).astype(f)
        return (prx * prx + pry * pry).astype(f)

    worst = 0.0
    for fma in (False, True):
        rc = to_e((x0 + (x1 - x0) * f(0.5)).astype(f), (y0 + (y1 - y0) * f(0.5)).astype(f), fma)
        P = [to_e(x0, y0, fma), to_e(x1, y0, fma), to_e(x1, y1, fma), to_e(x0, y1, fma)]
        ref = np.stack([(rc[0] ** 2 + rc[1] ** 2).astype(f), seg(P[0], P[1]), seg(P[1], P[2]), seg(P[2], P[3]),
                        seg(P[3], P[0])])
        for jitter in (0, 1, -1):
            vals, margin, _ = _cheap(e, r, jitter)
            near = np.abs(ref - 1) < 0.05
            gap = np.where(near, np.abs(vals.astype(np.float64) - ref) / margin, 0)
            worst = max(worst, float(gap.max()))
    assert worst < 0.25, worst


def test_zero_extent_overlaps_only_at_centre(O):
    """With a zero extent the reference's divisions yield only inf or NaN:
    the oracle's test reduces to the centre-in-rectangle test."""
    e, r = _cases(100_000, 10)
    e = list(e)
    e[5] = np.zeros_like(e[5])
    ref = O.overlap(np.stack(e, 1), np.stack(r, 1)).astype(bool)
    assert np.array_equal(ref, _centre(e, r))
    e[4] = np.zeros_like(e[4])
    ref = O.overlap(np.stack(e, 1), np.stack(r, 1)).astype(bool)
    assert np.array_equal(ref, _centre(e, r))

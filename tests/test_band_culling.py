"""CPU check of the rasterisers' culling bound (raster_common.cuh: band_rows).

band_rows gives, for a tile's band of pixel columns, the pixel rows where a
Gaussian's alpha can still reach 1/255; the rasterisers skip every warp strip
outside those rows.  This restates the function step by step in float32 and
checks, over random conics (isotropic to elongated, small to large, every
orientation) and tiles near and across each ellipse, that no pixel outside the
returned rows would blend (alpha = o exp(power) >= 1/255 with power <= 0,
rasterizer_cpu.cpp:146-150), in both orientations the library uses it: rows of
a column band (the rasterisers) and, transposed, columns of a row band.
"""
import numpy as np

F = np.float32


def band_rows(mx, my, a, b, c, thr, x0, x1):
    """Float32 restatement of band_rows: mean (mx, my), conic (a, b, c)."""
    t2 = F(-2.0) * F(thr)
    if not t2 > 0:
        return 1e30, -1e30
    det = F(a * c - b * b)
    if not (a > 0 and c > 0 and det >= F(1e-3) * a * c):
        return -1e30, 1e30
    idet = F(1.0) / det
    xext, yext = np.sqrt(F(t2 * c * idet)), np.sqrt(F(t2 * a * idet))
    dlo, dhi = F(mx - x1), F(mx - x0)
    mxw = F(1.0) + F(1e-3) * xext
    if dlo > xext + mxw or dhi < -xext - mxw:
        return 1e30, -1e30
    ic = F(1.0) / c
    slo = np.sqrt(max(F(0.0), F(t2 * c - det * dlo * dlo)))
    shi = np.sqrt(max(F(0.0), F(t2 * c - det * dhi * dhi)))
    up = max((slo - b * dlo) * ic, (shi - b * dhi) * ic)
    dn = min((-slo - b * dlo) * ic, (-shi - b * dhi) * ic)
    xtop = F(-b * yext / a)
    if dlo <= xtop <= dhi:
        up = yext
    if dlo <= -xtop <= dhi:
        dn = -yext
    myw = F(1.0) + F(1e-3) * yext
    return my - up - myw, my - dn + myw


def _random_gaussian(rng):
    s1, s2 = np.exp(rng.uniform(np.log(0.3), np.log(150.0), 2))
    th = rng.uniform(0.0, np.pi)
    rot = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    cov = rot @ np.diag([s1 * s1, s2 * s2]) @ rot.T + 0.3 * np.eye(2)   # the +0.3 dilation
    con = np.linalg.inv(cov)
    o = F(rng.uniform(0.005, 1.0))
    return F(con[0, 0]), F(con[0, 1]), F(con[1, 1]), o, cov, max(s1, s2)


def test_band_rows_never_culls_a_blending_pixel():
    rng = np.random.default_rng(7)
    culled = 0
    for _ in range(600):
        a, b, c, o, cov, smax = _random_gaussian(rng)
        mx, my = F(rng.uniform(-20, 220)), F(rng.uniform(-20, 220))
        thr = F(np.log(F(1.0 / 255.0) / o) - F(1e-3))   # skip_threshold
        ext = 3.0 * smax
        tx = int((mx + rng.uniform(-ext, ext)) // 16)
        ty = int((my + rng.uniform(-ext, ext)) // 16)
        xs = np.arange(16 * tx, 16 * tx + 16, dtype=np.float32)
        ys = np.arange(16 * ty, 16 * ty + 16, dtype=np.float32)
        X, Y = np.meshgrid(mx - xs, my - ys)             # d = mean - pixel
        power = F(-0.5) * (a * X * X + c * Y * Y) - b * X * Y
        blends = (o * np.exp(power.astype(np.float64)) >= 1.0 / 255.0) & (power <= 0)
        # rows of the tile's column band
        y0, y1 = band_rows(mx, my, a, b, c, thr, F(16 * tx), F(16 * tx + 15))
        outside = (ys[:, None] < y0) | (ys[:, None] > y1)
        culled += int(outside.sum())
        assert not (blends & outside).any()
        # columns of the tile's row band (transposed frame: x <-> y, a <-> c)
        x0, x1 = band_rows(my, mx, c, b, a, thr, F(16 * ty), F(16 * ty + 15))
        outside_c = (xs[None, :] < x0) | (xs[None, :] > x1)
        assert not (blends & outside_c).any()
    assert culled > 0   # the bound does cull

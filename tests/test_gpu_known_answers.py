"""GPU: the reference's stage unit tests (tests/test_preprocessor.cpp,
tests/test_rasterizer.cpp) restated through the C ABI, and the rasteriser on a
caller's own PreprocessOutput / BinningOutput arrays (gs3dc_rasterize_arrays,
the form those unit tests use): bit-exact images / transmittance / counts
against the C oracle on seeded arrays, the raster backward after it, and the
refusals that keep every index inside the caller's arrays.
"""
import numpy as np
import pytest

from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def _test_camera(w: int, h: int, fov_deg: float = 60.0) -> S.Camera:
    """makeTestCamera of the reference test: identity view, simple perspective."""
    f = np.float32
    cam = S.Camera()
    cam.width, cam.height = w, h
    tx = f(np.tan(f(fov_deg) * f(0.5) * f(3.14159265) / f(180.0)))
    ty = f(tx * f(h) / f(w))
    cam.tan_fovx, cam.tan_fovy = float(tx), float(ty)
    for k in range(16):
        cam.view_matrix[k] = 1.0 if k % 5 == 0 else 0.0
    n, fa = f(0.01), f(100.0)
    r, t = tx * n, ty * n
    vp = [0.0] * 16
    vp[0], vp[5] = float(n / r), float(n / t)
    vp[10], vp[11], vp[14] = float(fa / (fa - n)), 1.0, float(-(fa * n) / (fa - n))
    for k in range(16):
        cam.viewproj_matrix[k] = vp[k]
    return cam


def _model(pos, opa):
    n = len(opa)
    sc = S.Scene(np.array(pos, np.float32).reshape(n, 3), np.zeros((n, 3), np.float32),
                 np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1)), np.full((n, 1, 3), 0.5, np.float32),
                 np.array(opa, np.float32), 0)
    act = dict(positions=sc.positions.reshape(-1), scales=np.ones(3 * n, np.float32),
               rotations=sc.rotations.reshape(-1), sh_coeffs=sc.sh.reshape(-1), opacities=sc.opacities)
    return sc, act


def test_preprocessor_known_answers(ctx):
    cam = _test_camera(320, 240)
    cfg = S.render_config(False, sh_degree=0)
    sc, act = _model([0, 0, 5, 1, 0, 5, 0, 0, -5], [0.9, 0.8, 0.7])
    ctx.set_gaussians(sc, act)
    pre = ctx.preprocess(cam, cfg)
    assert pre["radii"][0] > 0 and pre["radii"][1] > 0 and pre["radii"][2] == 0    # G2 behind the camera
    assert abs(pre["depths"][0] - 5.0) < 1e-5 and pre["tiles_touched"][0] > 0 and pre["tiles_touched"][2] == 0
    assert pre["opacities_2d"][0] > 0.0 and pre["rgb"][0] > 0.0
    ref = O.forward(sc, cam, cfg, "c", act=act)
    assert np.array_equal(pre["radii"], ref.radii) and np.array_equal(pre["tiles_touched"], ref.tiles)


def _grid_ranges(nt, pairs):
    rg = np.zeros(2 * nt, np.uint32)
    for t, (a, b) in pairs.items():
        rg[2 * t], rg[2 * t + 1] = a, b
    return rg


def test_rasterizer_background_only_and_hwc(ctx):
    cam = S.Camera()
    cam.width = cam.height = 32
    cfg = S.render_config(False)
    cfg.bg_color[0], cfg.bg_color[1], cfg.bg_color[2] = 1.0, 0.0, 0.0
    z = np.zeros(0, np.float32)
    img, T, nc = ctx.rasterize_arrays(cam, cfg, z, z, z, z, np.zeros(0, np.uint32), np.zeros(8, np.uint32))
    assert np.all(img.reshape(-1, 3) == [1.0, 0.0, 0.0]) and np.all(T == 1.0) and np.all(nc == 0)
    cam.width = cam.height = 4
    cfg.bg_color[0], cfg.bg_color[1], cfg.bg_color[2] = 0.1, 0.2, 0.3
    img, _, _ = ctx.rasterize_arrays(cam, cfg, z, z, z, z, np.zeros(0, np.uint32), np.zeros(2, np.uint32))
    assert list(img[:6]) == [np.float32(0.1), np.float32(0.2), np.float32(0.3)] * 2    # HWC interleaved


def test_rasterizer_single_gaussian_center(ctx):
    cam = S.Camera()
    cam.width = cam.height = 32
    cfg = S.render_config(False)
    img, T, nc = ctx.rasterize_arrays(cam, cfg, [16.0, 16.0], [0.111, 0.0, 0.111], [0.95], [0.8, 0.5, 0.2],
                                      np.array([0], np.uint32), _grid_ranges(4, {3: (0, 1)}))
    c = img.reshape(32, 32, 3)[16, 16]
    assert np.all(c > 0.0) and abs(c[0] - 0.8 * 0.95) < 0.1
    assert nc.reshape(32, 32)[16, 16] == 1 and nc.reshape(32, 32)[0, 0] == 0   # tile 0 has no pairs


@pytest.mark.parametrize("n,w,h", [(3000, 160, 120), (40_000, 640, 480)])
def test_rasterize_arrays_match_oracle(ctx, n, w, h):
    sc = S.random_scene(n, seed=100 + n % 97)
    cam = S.look_at_camera((0.2, -0.1, -3.0), w, h)
    cfg = S.render_config(False, bg=(0.1, 0.3, 0.2))
    ref = O.forward(sc, cam, cfg, "c")
    img, T, nc = ctx.rasterize_arrays(cam, cfg, ref.means2D, ref.conics, ref.opac2d, ref.rgb, ref.vals_sorted,
                                      ref.ranges)
    assert np.abs(img - ref.image).max() <= 1e-5 and np.abs(T - ref.T_final).max() <= 1e-5
    assert np.array_equal(nc, ref.n_contrib)
    # the raster backward of the imported forward equals the one of the device's own forward
    d_img = np.random.default_rng(1).normal(0, 1e-3, 3 * w * h).astype(np.float32)
    g_imp = ctx.raster_backward(cam, cfg, d_img)
    with pytest.raises(gs3d.Gs3dError):       # no device model behind imported records
        ctx.preprocess_backward(cam, cfg)
    ctx.set_gaussians(sc, O.activate(sc))
    ctx.preprocess(cam, cfg)
    ctx.bin(cam, cfg)
    ctx.sort(ref.total_pairs, ((w + 15) // 16) * ((h + 15) // 16))
    ctx.rasterize(cam, cfg)
    g_dev = ctx.raster_backward(cam, cfg, d_img)
    for k in g_dev:
        a, b = g_imp[k].astype(np.float64), g_dev[k].astype(np.float64)
        assert np.abs(a - b).max() <= 1e-4 * (np.abs(b).max() + 1e-30), k


def test_rasterize_arrays_refuses_out_of_range_indices(ctx):
    cam = S.Camera()
    cam.width = cam.height = 32
    cfg = S.render_config(False)
    one = ([16.0, 16.0], [0.1, 0.0, 0.1], [0.5], [1.0, 1.0, 1.0])
    with pytest.raises(gs3d.Gs3dError):       # value 1 names a second Gaussian that is not there
        ctx.rasterize_arrays(cam, cfg, *one, np.array([1], np.uint32), _grid_ranges(4, {0: (0, 1)}))
    with pytest.raises(gs3d.Gs3dError):       # a range past the pairs
        ctx.rasterize_arrays(cam, cfg, *one, np.array([0], np.uint32), _grid_ranges(4, {0: (0, 2)}))
    with pytest.raises(gs3d.Gs3dError):       # ranges for another grid
        ctx.rasterize_arrays(cam, cfg, *one, np.array([0], np.uint32), np.zeros(6, np.uint32))

"""GPU: the 3D-evaluation render mode (RenderConfig::eval_3D, AAA-Gaussians).

Against the reference's own outputs (tests/golden/seeded/eval3d_*.npz, made by
the reference's CPU stages) and the C oracle on larger seeded scenes:
- per-Gaussian outputs (radii, tile counts, means, depths, dilated opacities,
  colours, gauss2screen, inverse covariances, mean offsets), the unsorted
  pairs with their per-tile depth keys, the sorted pairs and the tile ranges:
  bit-exact;
- image and final transmittance: <= 1e-5 max abs; contributor counts: exact
  (the kernel's exp is correctly rounded, glibc's expf is 1 ulp off on ~0.004 %
  of inputs, so a count may flip only when such an input sits on a threshold);
plus the host-array binning path, gs3dc_render, the raw-model path and the
refusal of the training calls (the mode has no backward).
"""
import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PER_GAUSSIAN = (("depths", 1), ("means2D", 2), ("opacities_2d", 1), ("rgb", 3),
                ("gauss2screen", 16), ("cov3D_inv", 6), ("mean_offset", 3))
FIXTURE_KEY = {"opacities_2d": "opac2d"}


def _grid(cam):
    return ((cam.width + 15) // 16) * ((cam.height + 15) // 16)


def _check_forward(ctx, cam, cfg, ref, ref_ex=None):
    """Stage outputs of the device against a reference result (StepResult or fixture dict)."""
    get = (lambda k: ref[k]) if isinstance(ref, dict) or hasattr(ref, "files") else (lambda k: getattr(ref, k))
    pre = ctx.preprocess(cam, cfg)
    radii = get("radii")
    vis = radii > 0
    assert np.array_equal(pre["radii"], radii)
    assert np.array_equal(pre["tiles_touched"], get("tiles"))
    for k, w in PER_GAUSSIAN:
        if ref_ex is not None and k in ref_ex:
            want = ref_ex[k].reshape(-1, w)
        else:
            want = np.asarray(get(FIXTURE_KEY.get(k, k))).reshape(-1, w)
        got = pre[k].reshape(-1, w)
        assert U.bits_equal(got[vis], want[vis]), k
    P, keys, vals = ctx.bin(cam, cfg)
    assert P == int(get("total_pairs"))
    assert U.bits_equal(keys, get("keys_unsorted")) and U.bits_equal(vals, get("vals_unsorted"))
    ks, vs, rg = ctx.sort(P, _grid(cam))
    kr, vr = U.canon(np.asarray(get("keys_sorted")), np.asarray(get("vals_sorted")))
    assert U.bits_equal(ks, kr) and U.bits_equal(vs, vr)
    assert U.bits_equal(rg, get("ranges"))
    img, T, nc = ctx.rasterize(cam, cfg)
    d_img = float(np.abs(img - get("image")).max()) if img.size else 0.0
    d_T = float(np.abs(T - get("T_final")).max()) if T.size else 0.0
    flips = int((nc != get("n_contrib")).sum())
    print(f"P={P} image max |d| {d_img:.2e}, T_final {d_T:.2e}, contributor-count mismatches {flips}")
    assert d_img <= 1e-5 and d_T <= 1e-5
    assert flips == 0
    return pre, img


@pytest.mark.parametrize("name", U.eval3d_cases())
def test_eval3d_stages_match_reference_fixture(ctx, name):
    sc, f3, cam, cfg, z = U.load_eval3d(name)
    ctx.set_gaussians(sc, O.activate(sc), filter_3d=f3)
    pre, img = _check_forward(ctx, cam, cfg, z)
    # the one-call render gives the same image
    assert np.array_equal(ctx.render(cam, cfg), img)
    # binning host arrays reproduces the device's pairs
    arrays = dict(means2D=pre["means2D"], depths=pre["depths"], radii=pre["radii"],
                  tiles_touched=pre["tiles_touched"], cov3D_inv=pre["cov3D_inv"], mean_offset=pre["mean_offset"])
    P, keys, vals = ctx.bin(cam, cfg, arrays=arrays)
    assert P == int(z["total_pairs"])
    assert U.bits_equal(keys, z["keys_unsorted"]) and U.bits_equal(vals, z["vals_unsorted"])


@pytest.mark.parametrize("n,w,h,eye,seed", [
    (50_000, 640, 480, (0.3, 0.2, -3.0), 61),
    (30_000, 320, 240, (0.1, 0.0, -0.7), 62),     # close: near plane, camera inside, view-space boxes
])
def test_eval3d_against_c_oracle(ctx, n, w, h, eye, seed):
    sc = S.eval3d_scene(n, seed=seed)
    f3 = S.filter_3d_values(n, seed=seed)
    cam = S.look_at_camera(eye, w, h, 65.0)
    cfg = S.render_config(False)
    cfg.eval_3D = True
    act = O.activate(sc)
    ref, ex = O.forward_eval3d(sc, cam, cfg, "c", act=act, filter_3d=f3)
    ctx.set_gaussians(sc, act, filter_3d=f3)
    _check_forward(ctx, cam, cfg, ref, ex)


def test_eval3d_raw_model_path(ctx):
    """A raw (trainable) model is activated on the device first (correctly rounded
    exp): the same results as the oracle on that activation."""
    sc = S.eval3d_scene(20_000, seed=63)
    cam = S.look_at_camera((0.2, -0.3, -2.8), 200, 150)
    cfg = S.render_config(True)
    cfg.eval_3D = True
    ref, ex = O.forward_eval3d(sc, cam, cfg, "c", act=U.activate_cr(sc))
    ctx.set_raw_params(sc)
    _check_forward(ctx, cam, cfg, ref, ex)


def test_eval3d_has_no_training_calls(ctx):
    sc = S.random_scene(2000, seed=64)
    cam = S.look_at_camera((0.0, 0.0, -3.0), 64, 64)
    cfg = S.render_config(True)
    cfg.eval_3D = True
    ctx.set_raw_params(sc)
    gt = np.zeros(64 * 64 * 3, np.float32)
    with pytest.raises(gs3d.Gs3dError):
        ctx.train_step(cam, gt, cfg, S.train_config(), 0)
    ctx.preprocess(cam, cfg)
    ctx.sort(*ctx.bin(cam, cfg)[:1], _grid(cam))
    ctx.rasterize(cam, cfg)
    with pytest.raises(gs3d.Gs3dError):
        ctx.raster_backward(cam, cfg, gt)
    # a 2D rasterisation of 3D-mode pairs is refused, and the 2D path still trains afterwards
    cfg2 = S.render_config(True)
    with pytest.raises(gs3d.Gs3dError):
        ctx.rasterize(cam, cfg2)
    loss = ctx.train_step(cam, gt, cfg2, S.train_config(), 0)
    assert np.isfinite(loss)

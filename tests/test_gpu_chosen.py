"""GPU: the reduced-storage ("chosen") form of the train step, BF16 and FP16.

Accuracy is stated against the FP64 oracle evaluating the model the device
holds (its 16-bit parameters, dequantised), so what is measured is the form's
arithmetic: fast exp, FMA, FP32 accumulation, the cut tile rectangles.
- forward image: PSNR >= 50 dB (2k Gaussians at 128x128, 100k at 640x480);
- raw-parameter gradients: cosine >= 0.999 against the FP64 adjoint;
plus the storage round trip, the pair-count reduction against the plain form
and a 1M / 1080p training run that lowers the loss.
"""
import numpy as np
import pytest

from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

FORMS = {"bf16": gs3d.FORM_BF16, "fp16": gs3d.FORM_FP16}
# learning rates that leave every parameter unchanged (lr_schedule takes log(lr_pos): not 0)
ZERO_LR = dict(lr_pos=1e-30, lr_rest=0.0)


@pytest.fixture(params=sorted(FORMS))
def form(ctx, request):
    ctx.set_option(gs3d.OPT_FORM, FORMS[request.param])
    yield request.param
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(1.0 / mse)


def _render_step(ctx, sc, cam, cfg, gt=None):
    """One train step with zero learning rates (parameters unchanged): its forward image."""
    gt = np.zeros(cam.width * cam.height * 3, np.float32) if gt is None else gt
    loss = ctx.train_step(cam, gt, cfg, S.train_config(**ZERO_LR), 0)
    return loss, ctx.get_image(cam).reshape(cam.height, cam.width, 3)


def test_storage_round_trip(ctx, form):
    sc = S.random_scene(5000, seed=31)
    ctx.set_raw_params(sc)
    out = ctx.get_raw_params(sc.copy())
    assert np.array_equal(out.positions, sc.positions)   # positions stay FP32
    rel = 2.0 ** -8 if form == "bf16" else 2.0 ** -11     # half an ulp of the 16-bit format
    for k in ("scales", "rotations", "sh", "opacities"):
        a, b = getattr(out, k), getattr(sc, k)
        assert np.all(np.abs(a - b) <= rel * np.abs(b) + 1e-7), k


@pytest.mark.parametrize("n,w,h", [(2000, 128, 128), (100_000, 640, 480)])
def test_forward_psnr_against_fp64_oracle(ctx, form, n, w, h):
    sc = S.random_scene(n, seed=32)
    cam = S.look_at_camera((0.3, 0.2, -3.0), w, h)
    cfg = S.render_config(True)
    ctx.set_raw_params(sc)
    model = ctx.get_raw_params(sc.copy())
    _, img = _render_step(ctx, sc, cam, cfg)
    _, ref, _ = O.step_f64(model, cam, cfg, None, want_grads=False)
    p = psnr(img, ref)
    print(f"{form} N={n} {w}x{h}: PSNR {p:.1f} dB vs FP64 oracle")
    assert p >= 50.0


def test_gradients_against_fp64_oracle(ctx, form):
    sc = S.random_scene(2000, seed=33)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 128, 128)
    cfg = S.render_config(True)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 1)
    try:
        ctx.set_raw_params(sc)
        model = ctx.get_raw_params(sc.copy())
        ctx.train_step(cam, gt, cfg, S.train_config(**ZERO_LR), 0)
        g = ctx.get_gradients()
    finally:
        ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 0)
    _, _, g64 = O.step_f64(model, cam, cfg, gt)
    keys = ("pos", "sc", "rot", "sh", "op")
    a = np.concatenate([g[k] for k in keys]).astype(np.float64)
    b = np.concatenate([g64[k] for k in keys])
    cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    per = {k: float(g[k].astype(np.float64) @ g64[k] / (np.linalg.norm(g[k]) * np.linalg.norm(g64[k]) + 1e-300))
           for k in keys}
    print(f"{form}: gradient cosine {cos:.6f} vs FP64 oracle; per group {per}")
    assert cos >= 0.999
    assert min(per.values()) >= 0.99


def test_pixels_per_thread_keep_the_image(ctx, form):
    """The rasterisers' pixels per thread (1, 2, 4: 256, 128, 64 threads per
    tile) and staging batch (64, 128, 256 records) change neither the
    reduced-form image (bit for bit) nor, beyond FP32-summation order, the
    gradients."""
    sc = S.random_scene(20000, seed=35)
    cam = S.look_at_camera((0.2, -0.3, -3.0), 333, 251)
    cfg = S.render_config(True)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 1)
    out = {}
    settings = [(1, 128), (2, 128), (4, 128), (2, 64), (4, 256)]
    try:
        for ppt, batch in settings:
            ctx.set_option(gs3d.OPT_RASTER_PPT, ppt)
            ctx.set_option(gs3d.OPT_RASTER_BATCH, batch)
            ctx.set_raw_params(sc)
            loss = ctx.train_step(cam, gt, cfg, S.train_config(**ZERO_LR), 0)
            out[(ppt, batch)] = (loss, ctx.get_image(cam), ctx.get_gradients())
    finally:
        ctx.set_option(gs3d.OPT_RASTER_PPT, 0)
        ctx.set_option(gs3d.OPT_RASTER_BATCH, 0)
        ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 0)
    out[1] = out[(1, 128)]
    for ppt in settings[1:]:
        assert np.array_equal(out[ppt][1], out[1][1]), ppt
        assert abs(out[ppt][0] - out[1][0]) <= 1e-7 * out[1][0]   # the loss sums tiles in another order
        for k in ("pos", "sc", "rot", "sh", "op"):
            a, b = out[ppt][2][k].astype(np.float64), out[1][2][k].astype(np.float64)
            assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b), (ppt, k)


def test_fewer_pairs_than_plain(ctx):
    sc = S.random_scene(100_000, seed=34)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 640, 480)
    cfg = S.render_config(True)
    pairs = {}
    for name, f in (("plain", gs3d.FORM_PLAIN_FP32), ("bf16", gs3d.FORM_BF16)):
        ctx.set_option(gs3d.OPT_FORM, f)
        ctx.set_raw_params(sc)
        _render_step(ctx, sc, cam, cfg)
        pairs[name] = ctx.stat(gs3d.STAT_TOTAL_PAIRS)
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    print(f"tile pairs: plain {pairs['plain']}, bf16 {pairs['bf16']} ({pairs['bf16'] / pairs['plain']:.3f})")
    assert 0 < pairs["bf16"] < pairs["plain"]


def test_training_lowers_the_loss_1m_1080p(ctx, form):
    w = S.config_train_1m_1080p()
    cam = w.cameras[0]
    cfg, tc = S.render_config(True), S.train_config()
    # target: the perturbed scene rendered by the plain form
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    ctx.set_raw_params(w.target_scene)
    _, gt = _render_step(ctx, w.target_scene, cam, S.render_config(False))
    ctx.set_option(gs3d.OPT_FORM, FORMS[form])
    ctx.set_raw_params(w.scene)
    losses = [ctx.train_step(cam, gt.reshape(-1), cfg, tc, it) for it in range(30)]
    print(f"{form}: loss {losses[0]:.6f} -> {losses[-1]:.6f}")
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.9 * losses[0]


def test_stochastic_rounding_moves_parameters_in_expectation(ctx):
    """One Adam step whose update is a fraction of a BF16 ulp for most SH
    coefficients: round-to-nearest would leave them in place, stochastic
    rounding moves them by the update in expectation.  Adam's first step
    (optimizer.cpp:32-43, bias-corrected) is lr * g / (|g| + eps)."""
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_BF16)
    sc = S.random_scene(200_000, seed=35)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 640, 480)
    cfg = S.render_config(True)
    gt = np.zeros(640 * 480 * 3, np.float32)
    lr = 2e-5   # 0.08 ulp at the median SH coefficient, 0.001 ulp at the median raw scale
    ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 1)
    try:
        ctx.set_raw_params(sc)
        before = ctx.get_raw_params(sc.copy())
        ctx.train_step(cam, gt, cfg, S.train_config(lr_pos=1e-30, lr_rest=lr), 0)
        g = ctx.get_gradients()
        after = ctx.get_raw_params(sc.copy())
    finally:
        ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 0)
        ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    eps = S.train_config().adam_eps
    for key in ("sh", "scales"):
        gk = g["sh" if key == "sh" else "sc"].astype(np.float64).ravel()
        d = (getattr(after, key).astype(np.float64) - getattr(before, key).astype(np.float64)).ravel()
        sel = gk != 0.0
        want = -lr * gk[sel] / (np.abs(gk[sel]) + eps)   # the FP32 update before rounding
        got = d[sel]
        resid = got - want
        se = float(np.std(resid) / np.sqrt(resid.size))
        frac_zero = float(np.mean(got == 0.0))
        print(f"{key}: {got.size} coefficients, mean step {got.mean():.4e} (expected {want.mean():.4e}, "
              f"standard error {se:.1e}), unchanged {frac_zero:.3f}")
        assert frac_zero > 0.5, "most updates should be below half an ulp (the test would not test rounding)"
        assert abs(float(resid.mean())) < 6.0 * se + 0.005 * lr


def test_non_finite_parameters_stay_non_finite(ctx):
    """The BF16 optimiser updates two elements per 32-bit word and redoes a
    chunk element-wise when a result is not finite (adding the rounding bits
    would otherwise carry a NaN's mantissa into its sign: NaN -> -0).  Two
    Gaussians behind the camera (no pairs, zero gradients) hold a NaN and an
    infinite SH coefficient: after a step both stay as they were, and the other
    coefficients of their 8-element chunks, with a zero update, keep their
    values."""
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_BF16)
    sc = S.random_scene(20_000, seed=36)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 320, 240)
    cfg = S.render_config(True)
    gt = np.zeros(320 * 240 * 3, np.float32)
    bad = {101: np.nan, 202: np.inf}     # Gaussian -> value of its SH coefficient 9 (chunk 1)
    for i, val in bad.items():
        sc.positions[i] = (0.6, 0.4, -6.0)   # behind the camera at (0.3, 0.2, -3) looking at the origin
        sc.sh.reshape(sc.positions.shape[0], -1)[i, 9] = val
    try:
        ctx.set_raw_params(sc)
        before = ctx.get_raw_params(sc.copy())
        loss = ctx.train_step(cam, gt, cfg, S.train_config(lr_pos=1e-30, lr_rest=1e-3), 0)
        after = ctx.get_raw_params(sc.copy())
    finally:
        ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    assert np.isfinite(loss)
    n = sc.positions.shape[0]
    sh_b, sh_a = before.sh.reshape(n, -1), after.sh.reshape(n, -1)
    assert np.isnan(sh_a[101, 9]) and sh_a[202, 9] == np.inf
    for i in bad:
        chunk = [k for k in range(8, 16) if k != 9]
        assert np.array_equal(sh_a[i, chunk], sh_b[i, chunk]), i
    mask = np.ones_like(sh_a, bool)
    mask[101, 9] = mask[202, 9] = False
    assert np.all(np.isfinite(sh_a[mask]))

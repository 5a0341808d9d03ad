"""GPU: the multi-view train step (gs3dc_train_step_batch, reduced-storage form).

One launch sequence renders and differentiates several views of mixed
resolution.  With vanishing learning rates (lr_pos 1e-30: the reference's lr_schedule takes
log(lr), so an exact zero would give NaN) the parameters do not move.  The
reference's path for each view is Trainer::step (src/trainer.cpp:7-70); the
batched loss is the mean of the views' L1 means and its gradient the mean of
the views' gradients.  Checked:
- against the FP64 oracle evaluating the dequantised 16-bit model on six views
  from 11x173 (one ragged tile column) to 3840x2160: every view's image at
  PSNR >= 50 dB, every view's L1 mean and the batched loss within 1e-3
  relative, the view-mean raw-parameter gradients at cosine >= 0.999 (every
  parameter group >= 0.99), the bars of the single-view reduced form;
- a step of more than 2^31 tile pairs (128 views at 3840x2160, 1M Gaussians):
  the views' images bit-identical to the same views in a small batch, the
  gradients equal to the mean of four 32-view batches (FP32 sums in another
  order: cosine >= 0.99999, relative difference <= 1e-4);
- the batched step against the library's single-view steps (same tolerances),
  and repeated batched steps (graph replays) returning the same loss.
"""
import numpy as np
import pytest

from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

KEYS = ("pos", "sc", "rot", "sh", "op")


@pytest.fixture
def bf16(ctx):
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_BF16)
    ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 1)
    yield
    ctx.set_option(gs3d.OPT_KEEP_GRADIENTS, 0)
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)


ZERO_LR = dict(lr_pos=1e-30, lr_rest=0.0)
ORACLE_RES = [(3840, 2160), (11, 173), (320, 240), (640, 480), (1280, 720), (1920, 1080)]


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(1.0 / mse)


def _cams_at(res, seed, fov=None):
    """One camera per (W, H) at random points of the radius-3 sphere, looking at the origin."""
    rng = np.random.default_rng(seed)
    cams = []
    for w, h in res:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if abs(d[1]) > 0.99:
            d[1] = 0.99 * np.sign(d[1])
            d /= np.linalg.norm(d)
        f = float(rng.uniform(45.0, 75.0)) if fov is None else fov
        cams.append(S.look_at_camera(d * 3.0, w, h, f))
    return cams


def _views(n, seed):
    return S.sphere_cameras(n, seed=seed, resolutions=[(160, 120), (320, 240), (256, 144), (200, 200)],
                            fov_range=(45.0, 75.0))


def test_batched_step_equals_mean_of_single_views(ctx, bf16):
    sc = S.random_scene(20000, seed=41)
    cams = _views(5, seed=42)
    cfg = S.render_config(True)
    tc0 = S.train_config(lr_pos=1e-30, lr_rest=0.0)
    target = S.perturbed(sc)
    gts = [O.forward(target, cam, S.render_config(False), "c").image for cam in cams]

    losses, grads = [], []
    for cam, gt in zip(cams, gts):
        ctx.set_raw_params(sc)
        losses.append(ctx.train_step(cam, gt, cfg, tc0, 0))
        grads.append(ctx.get_gradients())
    ctx.set_raw_params(sc)
    loss_b = ctx.train_step_batch(cams, np.concatenate(gts), cfg, tc0, 0)
    g_b = ctx.get_gradients()

    ref_loss = float(np.mean(losses))
    print(f"batched loss {loss_b:.8f}, mean of singles {ref_loss:.8f}")
    assert abs(loss_b - ref_loss) <= 1e-5 * ref_loss
    for k in KEYS:
        ref = np.mean([g[k].astype(np.float64) for g in grads], axis=0)
        got = g_b[k].astype(np.float64)
        cos = float(got @ ref / (np.linalg.norm(got) * np.linalg.norm(ref)))
        rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        print(f"{k}: cosine {cos:.8f}, relative difference {rel:.2e}")
        assert cos >= 0.99999 and rel <= 1e-4, k


def test_batched_step_against_the_fp64_oracle(ctx, bf16):
    sc = S.random_scene(50000, seed=47)
    cams = _cams_at(ORACLE_RES, seed=48)
    cfg = S.render_config(True)
    target = S.perturbed(sc)
    gts = [O.forward(target, cam, S.render_config(False), "c").image for cam in cams]
    ctx.set_raw_params(sc)
    model = ctx.get_raw_params(sc.copy())   # the 16-bit model the device holds, dequantised
    loss_b = ctx.train_step_batch(cams, np.concatenate(gts), cfg, S.train_config(**ZERO_LR), 0)
    g_b = ctx.get_gradients()
    losses64, grads64 = [], []
    for v, (cam, gt) in enumerate(zip(cams, gts)):
        l64, img64, g64 = O.step_f64(model, cam, cfg, gt)
        img = ctx.get_batch_image(v, cam)
        p = psnr(img.reshape(img64.shape), img64)
        l1 = float(np.mean(np.abs(img.astype(np.float64) - gt.astype(np.float64))))
        print(f"view {v} {cam.width}x{cam.height}: PSNR {p:.1f} dB, L1 {l1:.7f} (FP64 oracle {l64:.7f})")
        assert p >= 50.0, v
        assert abs(l1 - l64) <= 1e-3 * l64, v
        losses64.append(l64)
        grads64.append(g64)
    ref_loss = float(np.mean(losses64))
    print(f"batched loss {loss_b:.7f}, FP64 oracle mean over views {ref_loss:.7f}")
    assert abs(loss_b - ref_loss) <= 1e-3 * ref_loss
    ref = {k: np.mean([g[k] for g in grads64], axis=0) for k in KEYS}
    a = np.concatenate([g_b[k] for k in KEYS]).astype(np.float64)
    b = np.concatenate([ref[k] for k in KEYS])
    cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    per = {k: float(g_b[k].astype(np.float64) @ ref[k] / (np.linalg.norm(g_b[k]) * np.linalg.norm(ref[k]) + 1e-300))
           for k in KEYS}
    print(f"view-mean gradient cosine {cos:.6f} vs FP64 oracle; per group {per}")
    assert cos >= 0.999
    assert min(per.values()) >= 0.99


def test_batched_step_beyond_2_to_the_31_pairs():
    """128 views at 3840x2160 of 1M Gaussians: > 2^31 tile pairs in one step
    (about 105 GB of device memory, in a context of its own that is closed after)."""
    import torch
    sc = S.random_scene(1_000_000, seed=49)
    cams = _cams_at([(3840, 2160)] * 128, seed=50, fov=60.0)
    cfg = S.render_config(True)
    tc0 = S.train_config(**ZERO_LR)
    pix = sum(c.width * c.height for c in cams)
    gt = torch.zeros(3 * pix, dtype=torch.float32, device="cuda")   # target: black
    c = gs3d.Context(0)
    try:
        c.set_option(gs3d.OPT_FORM, gs3d.FORM_BF16)
        c.set_option(gs3d.OPT_KEEP_GRADIENTS, 1)
        c.set_raw_params(sc)
        loss_big = c.train_step_batch(cams, None, cfg, tc0, 0, gt_device_ptr=gt.data_ptr())
        P = c.stat(gs3d.STAT_TOTAL_PAIRS)
        print(f"{len(cams)} views at 3840x2160: {P} tile pairs (2^31 = {1 << 31}), loss {loss_big:.6f}")
        assert P > (1 << 31)
        g_big = c.get_gradients()
        picks = (0, 63, 127)
        imgs_big = [c.get_batch_image(v, cams[v]) for v in picks]
        # the same views in a small batch: the forward is deterministic per (view, tile), so bit-identical
        c.train_step_batch([cams[v] for v in picks], None, cfg, tc0, 0, gt_device_ptr=gt.data_ptr())
        for k, v in enumerate(picks):
            assert np.array_equal(c.get_batch_image(k, cams[v]), imgs_big[k]), v
        # the gradient of the mean over 128 views = the mean of four 32-view means
        parts = []
        for q in range(4):
            c.train_step_batch(cams[32 * q:32 * q + 32], None, cfg, tc0, 0, gt_device_ptr=gt.data_ptr())
            parts.append(c.get_gradients())
    finally:
        c.close()
        del gt
        torch.cuda.empty_cache()
    for k in KEYS:
        ref = np.mean([p[k].astype(np.float64) for p in parts], axis=0)
        got = g_big[k].astype(np.float64)
        cos = float(got @ ref / (np.linalg.norm(got) * np.linalg.norm(ref)))
        rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        print(f"{k}: cosine {cos:.8f}, relative difference {rel:.2e}")
        assert cos >= 0.99999 and rel <= 1e-4, k


def test_batched_graph_replays_are_stable_and_training_moves(ctx, bf16):
    sc = S.random_scene(20000, seed=43)
    cams = _views(8, seed=44)
    cfg = S.render_config(True)
    gt = np.concatenate([O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image for cam in cams])
    ctx.set_raw_params(sc)
    tc0 = S.train_config(lr_pos=1e-30, lr_rest=0.0)
    l0 = [ctx.train_step_batch(cams, gt, cfg, tc0, it) for it in range(4)]   # eager, then graph replays
    assert max(l0) - min(l0) <= 1e-6 * l0[0]
    assert ctx.stat(gs3d.STAT_GRAPH_REPLAYS) > 0
    tc = S.train_config()
    losses = [ctx.train_step_batch(cams, gt, cfg, tc, it) for it in range(20)]
    print(f"batched training: {losses[0]:.6f} -> {losses[-1]:.6f}")
    assert losses[-1] < 0.95 * losses[0]


def test_batched_step_needs_the_reduced_form(ctx):
    sc = S.random_scene(1000, seed=45)
    cams = _views(2, seed=46)
    ctx.set_raw_params(sc)
    gt = np.zeros(sum(c.width * c.height * 3 for c in cams), np.float32)
    with pytest.raises(gs3d.Gs3dError):
        ctx.train_step_batch(cams, gt, S.render_config(True), S.train_config(), 0)

"""GPU: the multi-view train step (gs3dc_train_step_batch, reduced-storage form).

One launch sequence renders and differentiates several views of mixed
resolution.  With vanishing learning rates (lr_pos 1e-30: the reference's lr_schedule takes
log(lr), so an exact zero would give NaN) the parameters do not move, so the
batched step must reproduce the single-view steps over the same cameras:
- loss = the mean of the single-view losses;
- raw-parameter gradients = the mean of the single-view gradients (FP32 sums in
  another order: cosine >= 0.99999, relative norm difference <= 1e-4);
and repeated batched steps (graph replays) return the same loss.
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

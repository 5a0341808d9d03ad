"""GPU: checkpoint / resume of the whole training state (gs3dc_save_state,
gs3dc_load_state), plain FP32 and BF16 forms.

- save -> load restores the model bit for bit, the Adam step counter and the
  form, and saving the restored state writes the same bytes again;
- a run resumed from a checkpoint (in a fresh context holding another model)
  follows the uninterrupted run: the losses and parameters after five more
  steps agree to FP32-summation-order noise (the raster adjoint adds per-tile
  contributions with atomics, so the order of additions is not fixed);
- files that are not checkpoints, or are cut short, are refused.
"""
import numpy as np
import pytest

from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

FORMS = {"plain": gs3d.FORM_PLAIN_FP32, "bf16": gs3d.FORM_BF16}
FIELDS = ("positions", "scales", "rotations", "sh", "opacities")


@pytest.fixture(params=sorted(FORMS))
def form(ctx, request):
    ctx.set_option(gs3d.OPT_FORM, FORMS[request.param])
    yield request.param
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)


def _setup(seed):
    sc = S.random_scene(20000, seed=seed)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 320, 240)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    return sc, cam, gt


def test_round_trip_is_exact(ctx, form, tmp_path):
    sc, cam, gt = _setup(51)
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_raw_params(sc)
    for it in range(3):
        ctx.train_step(cam, gt, cfg, tc, it)
    a = tmp_path / "a.ckpt"
    ctx.save_state(a)
    before = ctx.get_raw_params(sc.copy())
    step = ctx.stat(gs3d.STAT_ADAM_STEP)
    assert step == 3
    ctx.set_raw_params(S.random_scene(777, seed=52))     # something else in between
    ctx.load_state(a)
    assert ctx.stat(gs3d.STAT_ADAM_STEP) == step
    after = ctx.get_raw_params(sc.copy())
    for k in FIELDS:
        assert np.array_equal(getattr(after, k), getattr(before, k)), k
    b = tmp_path / "b.ckpt"
    ctx.save_state(b)
    assert a.read_bytes() == b.read_bytes()


def test_resumed_run_follows_the_uninterrupted_one(ctx, form, tmp_path):
    sc, cam, gt = _setup(53)
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_raw_params(sc)
    for it in range(5):
        ctx.train_step(cam, gt, cfg, tc, it)
    path = tmp_path / "mid.ckpt"
    ctx.save_state(path)
    cont = [ctx.train_step(cam, gt, cfg, tc, it) for it in range(5, 10)]
    p_cont = ctx.get_raw_params(sc.copy())

    other = gs3d.Context(0)
    try:
        other.set_option(gs3d.OPT_FORM, FORMS[form])   # the file's form wins in any case
        other.set_raw_params(S.random_scene(1000, seed=54))
        other.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
        other.load_state(path)
        res = [other.train_step(cam, gt, cfg, tc, it) for it in range(5, 10)]
        p_res = other.get_raw_params(sc.copy())
    finally:
        other.close()
    print(f"{form}: continued {cont[-1]:.7f}, resumed {res[-1]:.7f}")
    np.testing.assert_allclose(res, cont, rtol=1e-4)
    for k in FIELDS:
        a, b = getattr(p_res, k), getattr(p_cont, k)
        # BF16 storage: a summation-order difference may flip one stochastic rounding step
        tol = 1e-4 if form == "plain" else 2.0 ** -6
        assert np.max(np.abs(a - b)) <= tol * (1.0 + np.max(np.abs(b))), k


def test_bad_files_are_refused(ctx, tmp_path):
    sc, cam, gt = _setup(55)
    ctx.set_raw_params(sc)
    junk = tmp_path / "junk.ckpt"
    junk.write_bytes(b"not a checkpoint" * 8)
    with pytest.raises(gs3d.Gs3dError):
        ctx.load_state(junk)
    good = tmp_path / "good.ckpt"
    ctx.save_state(good)
    cut = tmp_path / "cut.ckpt"
    cut.write_bytes(good.read_bytes()[:-100])
    with pytest.raises(gs3d.Gs3dError):
        ctx.load_state(cut)
    with pytest.raises(gs3d.Gs3dError):
        ctx.load_state(tmp_path / "missing.ckpt")
    ctx.load_state(good)   # still usable
    assert np.array_equal(ctx.get_raw_params(sc.copy()).positions, sc.positions)

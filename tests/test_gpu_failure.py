"""GPU: failure paths without faulting the device.

* a device-side wait on a flag that nothing sets gives up after its bound
  and reports GS3DC_ERR_DEVICE_TIMEOUT; the context keeps working;
* tile-pair capacity overflow is detected on the device, nothing is updated,
  the capacity grows and the step is redone;
* an overflow inside an asynchronous graph replay skips the step and is
  reported by the next synchronising call;
* invalid arguments are rejected before any launch.
"""
import numpy as np
import pytest

from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def _scene():
    sc = S.random_scene(3000, seed=8)
    cam = S.look_at_camera((0.0, 0.3, -3.0), 160, 120)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    return sc, cam, gt


def test_bounded_wait_times_out_and_context_survives(ctx):
    assert ctx.selftest_bounded_wait(2000) == gs3d.ERR_DEVICE_TIMEOUT
    sc, cam, gt = _scene()
    ctx.set_raw_params(sc)
    loss = ctx.train_step(cam, gt, S.render_config(True), S.train_config(), 0)
    assert np.isfinite(loss) and loss > 0


def test_capacity_overflow_grows_and_redoes_the_step():
    sc, cam, gt = _scene()
    cfg, tc = S.render_config(True), S.train_config()
    results = []
    for cap in (0, 4096):
        with gs3d.Context(0) as c:
            if cap:
                c.set_option(gs3d.OPT_PAIR_CAPACITY, cap)
            c.set_raw_params(sc)
            losses = [c.train_step(cam, gt, cfg, tc, it) for it in range(2)]
            assert c.stat(gs3d.STAT_ADAM_STEP) == 2
            results.append((losses, c.get_raw_params(sc.copy()), c.stat(gs3d.STAT_PAIR_CAPACITY)))
    assert results[1][2] > 4096
    assert np.allclose(results[0][0], results[1][0], rtol=1e-6)
    for k in ("positions", "scales", "rotations", "sh", "opacities"):
        assert np.abs(getattr(results[0][1], k) - getattr(results[1][1], k)).max() <= 1e-6


def test_overflow_in_async_replay_is_reported_and_skipped():
    sc, cam, gt = _scene()
    cfg, tc = S.render_config(True), S.train_config()
    big = sc.copy()
    big.scales += 2.5            # same N, ~8x more tile pairs than the capacity sized for sc
    with gs3d.Context(0) as c:
        c.set_raw_params(sc)
        c.train_step(cam, gt, cfg, tc, 0)
        c.train_step(cam, gt, cfg, tc, 1)             # captured graph, capacity sized for sc
        cap = c.stat(gs3d.STAT_PAIR_CAPACITY)
        c.set_raw_params(big)
        c.train_step(cam, gt, cfg, tc, 2, want_loss=False)   # asynchronous replay that overflows
        with pytest.raises(gs3d.Gs3dError) as e:
            c.synchronize()
        assert e.value.status == gs3d.ERR_PAIR_OVERFLOW
        after = c.get_raw_params(big.copy())
        for k in ("positions", "scales", "rotations", "sh", "opacities"):
            assert np.array_equal(getattr(big, k), getattr(after, k)), k   # nothing was updated
        assert c.stat(gs3d.STAT_ADAM_STEP) == 0
        # a synchronous step grows the capacity, redoes the step and trains
        loss = c.train_step(cam, gt, cfg, tc, 3)
        assert np.isfinite(loss) and c.stat(gs3d.STAT_PAIR_CAPACITY) > cap
        assert c.stat(gs3d.STAT_ADAM_STEP) == 1


def test_invalid_arguments_are_rejected(ctx):
    sc, cam, gt = _scene()
    ctx.set_raw_params(sc)
    bad = S.render_config(True)
    bad.tile_w = 8
    with pytest.raises(gs3d.Gs3dError) as e:
        ctx.train_step(cam, gt, bad, S.train_config(), 0)
    assert e.value.status == gs3d.ERR_INVALID_ARG
    ev = S.render_config(True)
    ev.eval_3D = True   # the 3D-evaluation mode renders only
    with pytest.raises(gs3d.Gs3dError) as e:
        ctx.train_step(cam, gt, ev, S.train_config(), 0)
    assert e.value.status == gs3d.ERR_INVALID_ARG
    with pytest.raises(gs3d.Gs3dError) as e:
        ctx.sort_pairs(np.array([5 << 32], np.uint64), np.array([0], np.uint32), 2)
    assert e.value.status == gs3d.ERR_INVALID_ARG
    with gs3d.Context(0) as c:
        with pytest.raises(gs3d.Gs3dError) as e:
            c.render(cam, S.render_config(False))
        assert e.value.status == gs3d.ERR_NO_MODEL
        with pytest.raises(gs3d.Gs3dError) as e:
            c.rasterize(cam, S.render_config(False))
        assert e.value.status in (gs3d.ERR_STATE, gs3d.ERR_NO_MODEL)

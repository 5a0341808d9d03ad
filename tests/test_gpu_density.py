"""GPU: adaptive density control on the device (the trainer's DensityController).

- densify_and_prune on the reference's own fixtures (tests/golden/seeded/density_*.npz)
  and, with many splits, against the C oracle: counts exact; kept originals,
  clones and every array but the split children's positions bit-exact; the
  children's positions within 1e-6 (their Box-Muller samples use correctly
  rounded log / cos where the reference's glibc logf / cosf may be 1 ulp off);
- the split sampler's state carries over between calls;
- reset_opacity bit-exact; the optimiser resets when the count changes;
- gs3dc_train_step_densify: with densification off it trains like
  gs3dc_train_step; with it on it follows the same steps run through the stage
  calls (train step, forward, raster backward, gs3dc_density_accumulate,
  gs3dc_densify_and_prune): the raster backward adds per-Gaussian gradients
  with float atomics in no fixed order, so an average gradient that sits on
  the threshold may fall either way -- the counts agree to 0.5 %.
"""
import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("positions", "scales", "rotations", "sh", "opacities")


def _compare(got, want, n_children_max: int):
    assert got.count == want.count
    for k in ("scales", "rotations", "sh", "opacities"):
        assert U.bits_equal(getattr(got, k), getattr(want, k)), k
    a, b = got.positions, want.positions
    diff = np.any(a.view(np.uint32) != b.view(np.uint32), axis=1)
    assert int(diff.sum()) <= n_children_max
    assert np.all(np.abs(a - b) <= 1e-6 * (1.0 + np.abs(b)))


@pytest.mark.parametrize("name", U.density_cases())
def test_densify_matches_reference_fixture(ctx, name):
    sc, acc, cfg, extent, z = U.load_density(name)
    ctx.set_option(gs3d.OPT_DENSITY_SEED, 12345)   # a fresh controller's sampler state
    ctx.set_raw_params(sc)
    for d, r in acc:
        ctx.density_accumulate(d, r)
    n = ctx.densify_and_prune(cfg, extent)
    assert n == int(z["out_count"])
    got = ctx.get_model(sc.sh_degree)
    want = S.Scene(z["out_positions"], z["out_scales"], z["out_rotations"], z["out_sh"], z["out_opacities"],
                   sc.sh_degree)
    _compare(got, want, n_children_max=6)
    ctx.reset_opacity()
    assert U.bits_equal(ctx.get_model(sc.sh_degree).opacities, z["out_reset_opacities"])


def test_densify_many_splits_two_rounds_against_oracle(ctx):
    rng = np.random.default_rng(71)
    n = 20_000
    sc = S.random_scene(n, seed=71)
    sc.scales[:] = rng.normal(-4.4, 0.6, sc.scales.shape).astype(np.float32)   # about half above 1 % of extent
    sc.opacities[rng.random(n) < 0.05] = -7.0
    cfg = S.densify_config(enabled=True)
    ora = O.DensityOracle()
    ctx.set_option(gs3d.OPT_DENSITY_SEED, 12345)
    ctx.set_raw_params(sc)
    cur = sc
    for rnd in range(2):
        m = cur.count
        for _ in range(3):
            d = rng.normal(0, 3e-4, (m, 2)).astype(np.float32)
            r = rng.integers(0, 24, m).astype(np.int32)
            ora.accumulate(d, r, m)
            ctx.density_accumulate(d, r)
        want = ora.densify(cur, cfg, 1.1)
        got_n = ctx.densify_and_prune(cfg, 1.1)
        got = ctx.get_model(sc.sh_degree)
        print(f"round {rnd}: {m} -> {got_n}")
        _compare(got, want, n_children_max=2 * m)
        cur = want
        ctx.set_raw_params(cur)   # continue from identical parameters; the sampler state stays in the context
    assert ctx.stat(gs3d.STAT_NUM_GAUSSIANS) == cur.count


def test_optimizer_resets_when_the_count_changes(ctx):
    w = S.config_fd_2k()
    cam, gt = w.cameras[0], np.zeros(128 * 128 * 3, np.float32)
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_raw_params(w.scene)
    for it in range(3):
        ctx.train_step(cam, gt, cfg, tc, it)
    assert ctx.stat(gs3d.STAT_ADAM_STEP) == 3
    n0 = w.scene.count
    d = np.zeros((n0, 2), np.float32)
    ctx.density_accumulate(d, None)
    assert ctx.densify_and_prune(S.densify_config(min_opacity=0.0, enabled=True), 100.0) == n0
    assert ctx.stat(gs3d.STAT_ADAM_STEP) == 3     # same count: the moments stay
    d[:50] = 1.0
    ctx.density_accumulate(d, None)
    n1 = ctx.densify_and_prune(S.densify_config(min_opacity=0.0, enabled=True), 100.0)
    assert n1 == n0 + 50                          # 50 clones (every Gaussian is small at extent 100)
    assert ctx.stat(gs3d.STAT_ADAM_STEP) == 0


def _target(sc, cam):
    return O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image


def test_train_step_densify_off_trains_like_train_step(ctx):
    sc = S.random_scene(5000, seed=72)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 160, 120)
    gt = _target(sc, cam)
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_raw_params(sc)
    plain = [ctx.train_step(cam, gt, cfg, tc, it) for it in range(5)]
    ctx.set_raw_params(sc)
    off = S.densify_config(enabled=False)
    dens = [ctx.train_step_densify(cam, gt, cfg, tc, off, 1.0, it) for it in range(5)]
    assert all(n == sc.count for _, n in dens)
    np.testing.assert_allclose([l for l, _ in dens], plain, rtol=1e-5)


def test_train_step_densify_matches_stage_calls(ctx):
    sc = S.random_scene(5000, seed=73)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 160, 120)
    gt = _target(sc, cam)
    cfg, tc = S.render_config(True), S.train_config()
    dcfg = S.densify_config(enabled=True, densify_from_iter=2, densify_interval=2, grad_threshold=2e-6,
                            opacity_reset_interval=5, max_screen_size=40)
    extent = 0.8
    ctx.set_option(gs3d.OPT_DENSITY_SEED, 12345)
    ctx.set_raw_params(sc)
    fused = [ctx.train_step_densify(cam, gt, cfg, tc, dcfg, extent, it) for it in range(6)]
    m_fused = ctx.get_model(sc.sh_degree)
    counts = [n for _, n in fused]
    print("counts", counts)
    assert len(set(counts)) > 1                      # the model grew or shrank
    # the same sequence through the stage calls
    ctx.set_option(gs3d.OPT_DENSITY_SEED, 12345)
    ctx.set_raw_params(sc)
    inv_n = np.float32(1.0) / np.float32(cam.width * cam.height * 3)
    for it in range(6):
        ctx.train_step(cam, gt, cfg, tc, it)
        ctx.preprocess(cam, cfg)
        ctx.bin(cam, cfg)
        ctx.sort(ctx.stat(gs3d.STAT_TOTAL_PAIRS), ((cam.width + 15) // 16) * ((cam.height + 15) // 16))
        img, _, _ = ctx.rasterize(cam, cfg)
        d_img = (np.sign(img - gt) * inv_n).astype(np.float32)
        ctx.raster_backward(cam, cfg, d_img)
        ctx.density_accumulate(None, None)
        if it >= 2 and it % 2 == 0:
            n = ctx.densify_and_prune(dcfg, extent)
            print(f"iteration {it}: stage calls {n}, fused {counts[it]}")
            assert abs(n - counts[it]) <= 0.005 * counts[it]
        if it > 0 and it % 5 == 0:
            ctx.reset_opacity()
    m_stage = ctx.get_model(sc.sh_degree)
    assert abs(m_stage.count - m_fused.count) <= 0.005 * m_fused.count
    # the opacity reset of iteration 5 reached every Gaussian on both paths
    assert np.all(m_fused.opacities <= np.log(0.01 / 0.99) + 0.05)


# ---- the reference's DensityController unit tests (tests/test_density_controller.cpp), restated ----

def _params(n: int) -> S.Scene:
    """make_test_params of the reference test: positions (0.5 i, 0, 5), scales 0.1, identity
    rotations, opacity 0.5, SH degree 0 with every coefficient 1."""
    pos = np.stack([np.arange(n) * 0.5, np.zeros(n), np.full(n, 5.0)], 1).astype(np.float32)
    sc = np.full((n, 3), np.log(np.float32(0.1)), np.float32)
    rot = np.tile(np.array([1, 0, 0, 0], np.float32), (n, 1))
    return S.Scene(pos, sc, rot, np.ones((n, 1, 3), np.float32), np.zeros(n, np.float32), 0)


def _inv_sigmoid(x):
    return np.float32(np.log(np.float32(x) / (np.float32(1.0) - np.float32(x))))


KA_CFG = dict(grad_threshold=0.0002, min_opacity=0.001, enabled=True)


def _densify(ctx, sc, d_means2D, cfg=None):
    ctx.set_raw_params(sc)
    ctx.density_accumulate(np.asarray(d_means2D, np.float32), None)
    return ctx.densify_and_prune(cfg or S.densify_config(**KA_CFG), 100.0)


def test_known_answer_clone_small(ctx):
    d = np.zeros((5, 2), np.float32)
    d[0] = d[2] = 0.1
    assert _densify(ctx, _params(5), d) == 7
    m = ctx.get_model(0)
    assert m.positions[5, 0] == m.positions[0, 0] and m.positions[6, 0] == m.positions[2, 0]


def test_known_answer_split_large(ctx):
    sc = _params(3)
    sc.scales[1] = np.log(np.float32(5.0))
    d = np.zeros((3, 2), np.float32)
    d[1] = 0.5
    assert _densify(ctx, sc, d) == 4
    m = ctx.get_model(0)
    assert np.all(np.exp(m.scales).max(1) < 5.0)      # the large original is gone
    assert np.sum(np.isclose(m.scales[:, 0], np.log(np.float32(5.0)) - np.log(np.float32(1.6)))) == 2


def test_known_answer_prune_low_opacity(ctx):
    sc = _params(5)
    sc.opacities[1] = _inv_sigmoid(0.001)
    sc.opacities[3] = _inv_sigmoid(0.002)
    assert _densify(ctx, sc, np.zeros((5, 2)), S.densify_config(grad_threshold=0.0002, min_opacity=0.005,
                                                                  enabled=True)) == 3
    assert np.all(1.0 / (1.0 + np.exp(-ctx.get_model(0).opacities)) > 0.005)


def test_known_answer_single_clone_and_clone_plus_split(ctx):
    assert _densify(ctx, _params(1), [[0.5, 0.5]]) == 2
    m = ctx.get_model(0)
    assert m.positions[0, 0] == m.positions[1, 0]
    sc = _params(3)
    sc.scales[1] = np.log(np.float32(5.0))
    assert _densify(ctx, sc, [[0.5, 0.5], [0.5, 0.5], [0.0, 0.0]]) == 5


def test_known_answer_cycles_empty_and_reset(ctx):
    assert _densify(ctx, _params(2), np.full((2, 2), 0.5)) == 4
    ctx.density_accumulate(np.full((4, 2), 0.5, np.float32), None)
    assert ctx.densify_and_prune(S.densify_config(**KA_CFG), 100.0) == 8
    m = ctx.get_model(0)
    assert np.all(np.isfinite(m.positions)) and np.all(np.isfinite(m.opacities))
    sc = _params(3)
    sc.opacities[:] = _inv_sigmoid(0.001)
    assert _densify(ctx, sc, np.zeros((3, 2)), S.densify_config(min_opacity=0.005, enabled=True)) == 0
    sc = _params(3)
    sc.opacities[:] = [_inv_sigmoid(0.9), _inv_sigmoid(0.5), _inv_sigmoid(0.1)]
    ctx.set_raw_params(sc)
    ctx.reset_opacity()
    assert np.allclose(1.0 / (1.0 + np.exp(-ctx.get_model(0).opacities)), 0.01, atol=1e-4)

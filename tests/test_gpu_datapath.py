"""GPU: the multi-view data path from files, as the reference's train driver
runs it (src/train_main.cpp:470-700): PLY model -> initRawFromGaussianData ->
device; cameras.json views (the reference repository's own 76 cameras,
720x960) with PPM targets -> the batched train step; the trained model back
to a PLY file.
"""
import os

import numpy as np
import pytest

from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S

pytestmark = pytest.mark.gpu

FX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_fixtures", "formats")


def test_files_to_batched_training_and_back(ctx, tmp_path):
    rng = np.random.default_rng(90)
    scene = S.random_scene(30_000, seed=90)
    scene.positions[:] = rng.normal(0.0, 1.0, scene.positions.shape).astype(np.float32)
    scene.scales[:] = rng.normal(-3.5, 0.4, scene.scales.shape).astype(np.float32)
    cams = [c for c, _ in gs3d.load_cameras(os.path.join(FX, "cameras.json"))]
    names = [n for _, n in gs3d.load_cameras(os.path.join(FX, "cameras.json"))]
    pick = [0, 19, 38, 57]
    # targets: the perturbed scene rendered by the plain form, written as the driver's PPMs
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    ctx.set_raw_params(S.perturbed(scene))
    for i in pick:
        img = ctx.render(cams[i], S.render_config(False))
        gs3d.write_ppm(tmp_path / f"{names[i]}.ppm", img, cams[i].width, cams[i].height)
    # the model goes through a PLY file and the driver's initialisation
    gs3d.save_ply(tmp_path / "init.ply", scene)
    loaded, _ = gs3d.load_ply(tmp_path / "init.ply")          # activated, like loadPly
    raw = gs3d.raw_from_gaussians(loaded)                     # initRawFromGaussianData
    views = gs3d.load_views(os.path.join(FX, "cameras.json"), str(tmp_path))
    assert len(views) == len(pick)
    v_cams = [c for c, _ in views]
    gt = np.concatenate([t for _, t in views])
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_BF16)
    try:
        ctx.set_raw_params(raw)
        losses = [ctx.train_step_batch(v_cams, gt, cfg, tc, it) for it in range(15)]
        trained = ctx.get_model(scene.sh_degree)
    finally:
        ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    print(f"4 views of cameras.json: loss {losses[0]:.5f} -> {losses[-1]:.5f}")
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.9 * losses[0]
    gs3d.save_ply(tmp_path / "trained.ply", trained)
    back, _ = gs3d.load_ply(tmp_path / "trained.ply", activate=False)
    assert back.count == scene.count
    assert np.array_equal(back.positions, trained.positions)

"""GPU parity of the backward, the optimiser and the fused train step.

Tolerances (plain FP32 form): image <= 1e-5 abs; gradients elementwise
|cuda - ref| <= 1e-4 |ref| + 1e-5 max|ref| (FP32 atomics sum in a different
order than the reference's serial loops); cosine >= 0.999 against the FP64
oracle's adjoint.
"""
import os

import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

GRAD_RTOL, GRAD_ATOL_FRAC = 1e-4, 1e-5
GRADS = (("g_pos", "grad_raw_positions", "pos"), ("g_sc", "grad_raw_scales", "sc"),
         ("g_rot", "grad_raw_rotations", "rot"), ("g_sh", "grad_raw_sh_coeffs", "sh"),
         ("g_op", "grad_raw_opacities", "op"))


def _grid(cam):
    return ((cam.width + 15) // 16) * ((cam.height + 15) // 16)


def _l1_grad(img, gt):
    """d_image of the L1 loss (loss.cpp:4-16), float32."""
    n = img.size
    inv_n = np.float32(1.0) / np.float32(n)
    d = np.where(img > gt, inv_n, np.where(img < gt, -inv_n, np.float32(0))).astype(np.float32)
    return d


def _stage_grads(ctx, sc, cam, cfg, gt):
    """Stage-level forward + backward through the C ABI: (image, raster grads, raw grads)."""
    ctx.set_raw_params(sc)
    ctx.preprocess(cam, cfg)
    P, _, _ = ctx.bin(cam, cfg)
    ctx.sort(P, _grid(cam))
    img, T, nc = ctx.rasterize(cam, cfg)
    rg = ctx.raster_backward(cam, cfg, _l1_grad(img, gt))
    g = ctx.preprocess_backward(cam, cfg)
    return img, rg, g


@pytest.mark.parametrize("scene", U.grads_ext_scenes())
def test_grads_ext_fixture_gradients(ctx, scene):
    """Reference golden gradients (train/verify_grads_ext/<scene>) through the CUDA backward."""
    sc, cam, cfg, gt, exp = U.load_grads_fixture(os.path.join(U.REF_FIXTURES, "verify_grads_ext", scene))
    img, _, g = _stage_grads(ctx, sc, cam, cfg, gt)
    assert np.abs(img - exp["rendered"]).max() <= 1e-5
    rtol = 2e-4 if scene in U.STALE_GRAD_SCENES else GRAD_RTOL
    afrac = 1e-4 if scene in U.STALE_GRAD_SCENES else GRAD_ATOL_FRAC
    for k, ek, _ in GRADS:
        ok, worst = U.rel_close(g[k], exp[ek], rtol, afrac)
        assert ok, (scene, k, worst)


def test_stage_backward_matches_oracle(ctx):
    """RasterizerBackward + PreprocessorBackward vs the oracle on 2k Gaussians, 128x128."""
    z = np.load(os.path.join(U.SEEDED, "train_2k_128x128_adam.npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), 3)
    cam = S.Camera.from_buffer_copy(z["cam_bytes"].tobytes())
    cfg = S.RenderConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    img, rg, g = _stage_grads(ctx, sc, cam, cfg, z["gt"])
    assert np.abs(img - z["s0_image"]).max() <= 1e-5
    for k in ("d_means2D", "d_conics", "d_rgb"):
        ok, worst = U.rel_close(rg[k], z[f"s0_{k}"], GRAD_RTOL, GRAD_ATOL_FRAC)
        assert ok, (k, worst)
    ok, worst = U.rel_close(rg["d_opac"], z["s0_d_opac"], GRAD_RTOL, GRAD_ATOL_FRAC)
    assert ok, ("d_opac", worst)
    for k, _, _ in GRADS:
        ok, worst = U.rel_close(g[k], z[f"s0_{k}"], GRAD_RTOL, GRAD_ATOL_FRAC)
        assert ok, (k, worst)


def test_train_step_matches_reference_trajectory(ctx):
    """Two fused Trainer::step calls (Adam) against the reference's own two steps."""
    z = np.load(os.path.join(U.SEEDED, "train_2k_128x128_adam.npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), 3)
    cam = S.Camera.from_buffer_copy(z["cam_bytes"].tobytes())
    cfg = S.RenderConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    tc = S.TrainConfig.from_buffer_copy(z["tc_bytes"].tobytes())
    ctx.set_raw_params(sc)
    for it in range(2):
        loss = ctx.train_step(cam, z["gt"], cfg, tc, it)
        assert abs(loss - float(z[f"s{it}_loss_acc64"])) <= 1e-6 * float(z[f"s{it}_loss_acc64"])
        out = ctx.get_raw_params(sc.copy())
        for k in ("positions", "scales", "rotations", "sh", "opacities"):
            d = np.abs(getattr(out, k) - z[f"s{it}_{k}"]).max()
            assert d <= 1e-5, (it, k, d)
    assert ctx.stat(gs3d.STAT_ADAM_STEP) == 2


def test_train_step_graph_matches_eager(ctx):
    """CUDA-graph replays give the same trajectory as un-captured steps."""
    sc = S.random_scene(3000, seed=5)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 160, 120)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    cfg, tc = S.render_config(True), S.train_config()
    res = []
    for graph in (0, 1):
        ctx.set_option(gs3d.OPT_USE_GRAPH, graph)
        ctx.set_raw_params(sc)
        losses = [ctx.train_step(cam, gt, cfg, tc, it) for it in range(4)]
        res.append((losses, ctx.get_raw_params(sc.copy())))
    ctx.set_option(gs3d.OPT_USE_GRAPH, 1)
    assert np.allclose(res[0][0], res[1][0], rtol=1e-6)
    for k in ("positions", "scales", "rotations", "sh", "opacities"):
        assert np.abs(getattr(res[0][1], k) - getattr(res[1][1], k)).max() <= 1e-6


@pytest.mark.parametrize("form", ["plain", "bf16"])
def test_host_target_steps_match_device_target_steps(ctx, form):
    """A host target runs the forward before its copy lands and the L1 as its
    own kernel; a device target keeps the L1 fused into the forward.  Both give
    the same sign bytes, so the same gradients up to the order of the screen
    gradients' atomics (parameters to 1e-6 in the plain form; in BF16 a
    stochastic rounding may flip by one ulp, so only the losses compare)."""
    import torch
    sc = S.random_scene(4000, seed=6)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 176, 144)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image.astype(np.float32).ravel()
    gt_dev = torch.from_numpy(gt).cuda()
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_BF16 if form == "bf16" else gs3d.FORM_PLAIN_FP32)
    res = []
    try:
        for on_device in (False, True):
            ctx.set_raw_params(sc)
            losses = []
            for it in range(4):   # later steps replay the shape's graphs
                if on_device:
                    losses.append(ctx.train_step(cam, None, cfg, tc, it, gt_device_ptr=gt_dev.data_ptr()))
                else:
                    losses.append(ctx.train_step(cam, gt, cfg, tc, it))
            res.append((losses, ctx.get_raw_params(sc.copy())))
    finally:
        ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    assert np.allclose(res[0][0], res[1][0], rtol=1e-5, atol=0.0)
    if form == "plain":
        for k in ("positions", "scales", "rotations", "sh", "opacities"):
            assert np.abs(getattr(res[0][1], k) - getattr(res[1][1], k)).max() <= 1e-6, k


def test_train_step_keeps_a_graph_per_camera_size(ctx):
    """Cycling through cameras of three sizes: each size is captured once and
    replayed afterwards (no re-capture when the size changes back), with the
    same trajectory as un-captured steps."""
    sc = S.random_scene(3001, seed=6)   # a model size and camera sizes no other test uses
    cams = [S.look_at_camera((0.3, 0.2, -3.0), 168, 120), S.look_at_camera((-0.2, 0.4, -3.0), 96, 72),
            S.look_at_camera((0.1, -0.3, -3.0), 200, 136)]
    gts = [O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image for cam in cams]
    cfg, tc = S.render_config(True), S.train_config()
    res = []
    for graph in (1, 0):
        ctx.set_option(gs3d.OPT_USE_GRAPH, graph)
        ctx.set_raw_params(sc)
        r0, c0 = ctx.stat(gs3d.STAT_GRAPH_REPLAYS), ctx.stat(gs3d.STAT_GRAPH_CAPTURES)
        losses = []
        for it in range(12):
            v = it % 3
            losses.append(ctx.train_step(cams[v], gts[v], cfg, tc, it))
        replays = ctx.stat(gs3d.STAT_GRAPH_REPLAYS) - r0
        captures = ctx.stat(gs3d.STAT_GRAPH_CAPTURES) - c0
        res.append((losses, ctx.get_raw_params(sc.copy()), replays, captures))
    ctx.set_option(gs3d.OPT_USE_GRAPH, 1)
    # the first step of each size runs un-captured; the other 9 replay 3 graphs captured once
    assert res[0][2] == 9 and res[0][3] == 3, res[0][2:]
    assert res[1][2] == 0 and res[1][3] == 0
    assert np.allclose(res[0][0], res[1][0], rtol=1e-6)
    for k in ("positions", "scales", "rotations", "sh", "opacities"):
        assert np.abs(getattr(res[0][1], k) - getattr(res[1][1], k)).max() <= 1e-6


@pytest.mark.parametrize("tied", [False, True])
def test_train_step_sort_modes_agree(ctx, tied):
    """Depth-first ordering (Gaussians sorted by depth, pairs sorted by tile
    only) renders bit-identically to the full-key sort, also when every
    Gaussian has the same depth bits (a plane facing the camera), where only
    the Gaussian-index tie-break decides the blend order."""
    sc = S.random_scene(20000, seed=21)
    if tied:
        sc.positions[:, 2] = 0.0
    cam = S.look_at_camera((0.0, 0.0, -3.0), 320, 240)
    cfg, tc = S.render_config(True), S.train_config()
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    ref = O.forward(sc, cam, cfg, "c")
    if tied:
        assert len(np.unique(ref.keys_sorted & np.uint64(0xFFFFFFFF))) == 1
    out = {}
    for mode in (gs3d.SORT_FULL_KEY, gs3d.SORT_DEPTH_FIRST):
        ctx.set_option(gs3d.OPT_SORT, mode)
        ctx.set_raw_params(sc)
        loss0 = ctx.train_step(cam, gt, cfg, tc, 0)
        img0 = ctx.get_image(cam)
        for it in range(1, 3):
            ctx.train_step(cam, gt, cfg, tc, it)
        out[mode] = (loss0, img0, ctx.get_raw_params(sc.copy()))
    ctx.set_option(gs3d.OPT_SORT, gs3d.SORT_DEPTH_FIRST)
    (la, ia, pa), (lb, ib, pb) = out[gs3d.SORT_FULL_KEY], out[gs3d.SORT_DEPTH_FIRST]
    assert U.bits_equal(ia, ib)
    assert np.abs(ib - ref.image).max() <= 1e-5
    assert abs(la - lb) <= 1e-6 * abs(la)
    for k in ("positions", "scales", "rotations", "sh", "opacities"):
        assert np.abs(getattr(pa, k) - getattr(pb, k)).max() <= 1e-6, k


def test_optimizer_stage_matches_reference(ctx):
    """Stage-level AdamOptimizer::step on the device equals the fused step."""
    z = np.load(os.path.join(U.SEEDED, "train_2k_128x128_adam.npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), 3)
    cam = S.Camera.from_buffer_copy(z["cam_bytes"].tobytes())
    cfg = S.RenderConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    tc = S.TrainConfig.from_buffer_copy(z["tc_bytes"].tobytes())
    _stage_grads(ctx, sc, cam, cfg, z["gt"])
    ctx.optimizer_step(tc, 0)
    out = ctx.get_raw_params(sc.copy())
    for k in ("positions", "scales", "rotations", "sh", "opacities"):
        assert np.abs(getattr(out, k) - z[f"s0_{k}"]).max() <= 1e-5, k


def test_adjoint_against_fp64_oracle_and_finite_differences(ctx):
    """The differentiation check: N=2k, 128x128.  CUDA adjoint vs the FP64
    oracle's adjoint (cosine >= 0.999 per parameter group and on 200 random
    parameters) and vs FP64 central finite differences."""
    w = S.config_fd_2k()
    sc, cam = w.scene, w.cameras[0]
    cfg = S.render_config(True)
    gt = O.forward(w.target_scene, cam, S.render_config(False), "c").image
    _, _, g = _stage_grads(ctx, sc, cam, cfg, gt)
    loss64, _, g64 = O.step_f64(sc, cam, cfg, gt)
    for k, _, k64 in GRADS:
        assert U.cosine(g[k], g64[k64]) >= 0.999, k
    p64 = [np.ascontiguousarray(x, np.float64).reshape(-1).copy() for x in
           (sc.positions, sc.scales, sc.rotations, sc.sh, sc.opacities)]
    picks = U.fd_picks([len(x) for x in p64], seed=S.SEED_FD)
    cuda = np.array([g[GRADS[grp][0]][i] for grp, i in picks])
    ana = np.array([g64[GRADS[grp][2]][i] for grp, i in picks])
    assert U.cosine(cuda, ana) >= 0.999
    # h=1e-6: cosine >= 0.999 and every element within the reference FD
    # tolerance; h=1e-4 (the configured step): >= 95% within it (quotients that
    # straddle an L1 kink or an alpha / transmittance threshold are outliers)
    for h, min_cos, min_within in ((1e-6, 0.999, 0.99), (1e-4, None, 0.95)):
        fd = []
        for grp, i in picks:
            o = p64[grp][i]
            p64[grp][i] = o + h
            lp, _, _ = O.step_f64(sc, cam, cfg, gt, want_grads=False, params64=p64)
            p64[grp][i] = o - h
            lm, _, _ = O.step_f64(sc, cam, cfg, gt, want_grads=False, params64=p64)
            p64[grp][i] = o
            fd.append((lp - lm) / (2 * h))
        fd = np.array(fd)
        if min_cos is not None:
            assert U.cosine(cuda, fd) >= min_cos, h
        assert U.fd_within(fd, cuda).mean() >= min_within, h


def test_recompute_backward_memory_vs_stored_lists():
    """N=100k at 640x480: the raster backward that recovers transmittance by
    division (gs3dc_raster_backward) against the reference's stored per-pixel
    contributor lists (gs3dc_raster_backward_lists,
    rasterizer_backward_cpu.cpp:40-67).  Device memory is measured with
    cudaMemGetInfo around each backward in a context of its own: the
    recompute backward allocates only its d_image upload (12 bytes per pixel),
    the list variant 4 bytes per pixel plus 8 per contributor.  Both give the
    same gradients (FP32 atomics in another order)."""
    import torch
    w = S.config_render_100k()
    cam, cfg = w.cameras[0], S.render_config(True)
    gt = O.forward(S.perturbed(w.scene), cam, S.render_config(False), "c").image
    c = gs3d.Context(0)
    try:
        c.set_raw_params(w.scene)

        def forward(cm):
            c.preprocess(cm, cfg)
            P, _, _ = c.bin(cm, cfg)
            c.sort(P, _grid(cm))
            return c.rasterize(cm, cfg)
        # both backwards once on a small camera first: kernel loading and the driver's
        # per-kernel reservations happen there, so the deltas below are the buffers' own
        small = S.look_at_camera((0.0, 0.0, -3.0), 64, 48)
        im_s, _, _ = forward(small)
        c.raster_backward(small, cfg, np.zeros_like(im_s))
        c.raster_backward_lists(small, cfg, np.zeros_like(im_s))
        img, _, nc = forward(cam)
        d_img = _l1_grad(img, gt)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rg = c.raster_backward(cam, cfg, d_img)
        free1 = torch.cuda.mem_get_info()[0]
        rl, list_bytes = c.raster_backward_lists(cam, cfg, d_img)
        free2 = torch.cuda.mem_get_info()[0]
    finally:
        c.close()
    npx = cam.width * cam.height
    contributors = int(nc.astype(np.int64).sum())
    used_recompute, used_lists = free0 - free1, free1 - free2
    print(f"recompute backward: {used_recompute / 2**20:.1f} MiB allocated (d_image upload {12 * npx / 2**20:.1f} "
          f"MiB); stored lists: {used_lists / 2**20:.1f} MiB allocated for {contributors} contributors "
          f"({list_bytes / 2**20:.1f} MiB of lists and offsets)")
    assert list_bytes == 4 * npx + 8 * contributors
    # measured by the driver: 2 MiB pages, and small buffers may land in pages the runtime already holds
    assert used_lists >= 0.95 * list_bytes
    assert used_recompute <= 12 * npx + (4 << 20)        # nothing beyond the d_image upload
    assert used_lists > 10 * used_recompute
    for k in ("d_means2D", "d_conics", "d_rgb", "d_opac"):
        ok, worst = U.rel_close(rl[k], rg[k], GRAD_RTOL, GRAD_ATOL_FRAC)
        assert ok, (k, worst)


@pytest.mark.parametrize("form", [gs3d.FORM_PLAIN_FP32, gs3d.FORM_BF16])
def test_autotuner_picks_a_setting_and_keeps_results(ctx, form):
    """GS3DC_OPT_AUTOTUNE: the first 6 steps try 1 / 2 / 4 pixels per thread,
    the next 4 the staging batches 64 / 256, then the picks stay; the forward
    image does not depend on the setting and the trajectory matches an untuned
    run to FP32-summation level."""
    sc = S.random_scene(20000, seed=51)
    cam = S.look_at_camera((0.3, 0.2, -3.0), 320, 240)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    cfg, tc = S.render_config(True), S.train_config()
    ctx.set_option(gs3d.OPT_FORM, form)
    res = []
    try:
        for tune in (0, 1):
            ctx.set_option(gs3d.OPT_AUTOTUNE, tune)
            ctx.set_raw_params(sc)
            losses = [ctx.train_step(cam, gt, cfg, tc, it) for it in range(12)]
            res.append((losses, ctx.get_raw_params(sc.copy()),
                        (ctx.stat(gs3d.STAT_FWD_PPT), ctx.stat(gs3d.STAT_BWD_PPT),
                         ctx.stat(gs3d.STAT_FWD_BATCH), ctx.stat(gs3d.STAT_BWD_BATCH))))
    finally:
        ctx.set_option(gs3d.OPT_AUTOTUNE, 0)
        ctx.set_option(gs3d.OPT_FORM, gs3d.FORM_PLAIN_FP32)
    (l0, p0, k0), (l1, p1, k1) = res
    print(f"form {form}: autotuner picked forward {k1[0]}, backward {k1[1]} pixels per thread, "
          f"staging batches {k1[2]} / {k1[3]}")
    assert k0 == (2, 2, 128, 128) and k1[0] in (1, 2, 4) and k1[1] in (1, 2, 4)
    assert k1[2] in (64, 128, 256) and k1[3] in (64, 128, 256)
    assert abs(l0[0] - l1[0]) <= 1e-6 * l0[0]     # same first forward whatever the setting
    assert np.allclose(l0, l1, rtol=2e-3)
    if form == gs3d.FORM_PLAIN_FP32:
        # the backward's FP32 sums change order with the setting; Adam moves by at most lr per step.
        # (In BF16 a stochastic-rounding decision can flip by one 16-bit ulp: only the losses compare.)
        for k in ("positions", "scales", "rotations", "sh", "opacities"):
            assert np.abs(getattr(p0, k) - getattr(p1, k)).max() <= 5e-3, k

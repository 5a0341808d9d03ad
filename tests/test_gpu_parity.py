"""GPU parity of the forward stages through the C ABI, against the oracle.

Integer outputs (radii, tiles_touched, keys, values, sorted order, tile
ranges, contributor counts) must be bit-exact; float outputs of the plain
FP32 form must match within 1e-5 (image) -- they are in fact bit-exact for
everything before the blend and within a few ulp after it.
"""
import os

import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O
from test_oracle_pin import SORTER_CASES, _sort as oracle_sort

pytestmark = pytest.mark.gpu

IMAGE_ATOL = 1e-5


def _grid(cam):
    return ((cam.width + 15) // 16) * ((cam.height + 15) // 16)


def _check_forward(ctx, sc, cam, cfg, exp, act_on_device: bool):
    if act_on_device:
        ctx.set_raw_params(sc)
    else:
        ctx.set_gaussians(sc, O.activate(sc))
    pre = ctx.preprocess(cam, cfg, want_cache=True)
    radii = exp["radii"]
    vis = radii > 0
    assert U.bits_equal(pre["radii"], radii)
    assert U.bits_equal(pre["tiles_touched"], exp["tiles"])
    assert U.bits_equal(pre["depths"][vis], exp["depths"][vis])
    if not act_on_device:
        assert U.bits_equal(pre["means2D"].reshape(-1, 2)[vis], exp["means2D"].reshape(-1, 2)[vis])
        assert U.bits_equal(pre["conics"].reshape(-1, 3)[vis], exp["conics"].reshape(-1, 3)[vis])
        assert U.bits_equal(pre["rgb"].reshape(-1, 3)[vis], exp["rgb"].reshape(-1, 3)[vis])
        for k, kk in (("cov3D", "cov3D"), ("p_view", "p_view"), ("p_hom_w", "p_hom_w"), ("cov2D", "cov2D"),
                      ("cov2D_det", "det")):
            assert U.bits_equal(pre[k], exp[kk]), k
    P, ku, vu = ctx.bin(cam, cfg)
    assert P == int(exp["total_pairs"])
    assert U.bits_equal(ku, exp["keys_unsorted"]) and U.bits_equal(vu, exp["vals_unsorted"])
    ks, vs, rg = ctx.sort(P, _grid(cam))
    # the CUDA sort is stable, i.e. already in (key, value) order
    assert U.bits_equal(ks, exp["keys_sorted"]) and U.bits_equal(vs, exp["vals_sorted"])
    assert U.bits_equal(rg, exp["ranges"])
    img, T, nc = ctx.rasterize(cam, cfg)
    assert np.abs(img - exp["image"]).max() <= IMAGE_ATOL
    assert np.abs(T - exp["T_final"]).max() <= IMAGE_ATOL
    assert U.bits_equal(nc, exp["n_contrib"])
    return img


@pytest.mark.parametrize("name", U.seeded_cases())
def test_seeded_forward_host_activation(ctx, name):
    """Reference-activated model (GaussianData) -> CUDA stages == reference CPU stages."""
    sc, cam, cfg, z = U.load_seeded(name)
    _check_forward(ctx, sc, cam, cfg, z, act_on_device=False)


@pytest.mark.parametrize("name", ["render_2k_128x128", "render_deg2_train_80x80", "render_aa_scale_64x48"])
def test_seeded_forward_device_activation(ctx, name):
    """Raw model activated on the device: integer outputs and depths stay exact."""
    sc, cam, cfg, z = U.load_seeded(name)
    _check_forward(ctx, sc, cam, cfg, z, act_on_device=True)


def test_render_entry_point_100k(ctx):
    """Renderer::render at the render config (100k Gaussians, 640x480)."""
    w = S.config_render_100k()
    cam, cfg = w.cameras[0], S.render_config(False)
    act = O.activate(w.scene)
    ref = O.forward(w.scene, cam, cfg, "c", act=act)
    ctx.set_gaussians(w.scene, act)
    img = ctx.render(cam, cfg)
    assert np.abs(img - ref.image).max() <= IMAGE_ATOL
    # the same forward, stage by stage, with every integer output exact
    exp = dict(radii=ref.radii, tiles=ref.tiles, depths=ref.depths, means2D=ref.means2D, conics=ref.conics,
               rgb=ref.rgb, cov3D=ref.cov3D, p_view=ref.p_view, p_hom_w=ref.p_hom_w, cov2D=ref.cov2D, det=ref.det,
               total_pairs=ref.total_pairs, keys_unsorted=ref.keys_unsorted, vals_unsorted=ref.vals_unsorted,
               keys_sorted=ref.keys_sorted, vals_sorted=ref.vals_sorted, ranges=ref.ranges, image=ref.image,
               T_final=ref.T_final, n_contrib=ref.n_contrib)
    img2 = _check_forward(ctx, w.scene, cam, cfg, exp, act_on_device=False)
    assert U.bits_equal(img, img2)   # idempotent


# ---- the reference's sorter / binner known answers through the C ABI ----

@pytest.mark.parametrize("case", sorted(SORTER_CASES))
def test_sort_pairs_known_answers(ctx, case):
    keys, vals, nt, exp_vals, exp_ranges = SORTER_CASES[case]
    ko, vo, rg = ctx.sort_pairs(np.array(keys, np.uint64), np.array(vals, np.uint32), nt)
    assert list(vo) == exp_vals and list(rg) == exp_ranges and list(ko) == sorted(keys)


# (1, 1): a single pair; 4095 / 4097: around the 4096-key onesweep CTA tile;
# (60_000, 5) / (150_000, 3): few tiles of ~12K / ~50K pairs each
@pytest.mark.parametrize("P,num_tiles,dups", [(1, 1, False), (4095, 7, True), (4097, 3000, False),
                                              (60_000, 5, True), (150_000, 3, True),
                                              (300_001, 8160, True), (2_000_000, 32400, True)])
def test_sort_pairs_random_stable(ctx, P, num_tiles, dups):
    """Random keys, ragged sizes around the 4096-key CTA tile, duplicate keys,
    very full tiles: the CUDA result equals the stable (key, index) order."""
    rng = np.random.default_rng(P)
    tiles = rng.integers(0, num_tiles, P).astype(np.uint64)
    depth = rng.integers(0x3E4CCCCD, 0x40C00000, P).astype(np.uint64)
    if dups:
        depth[rng.integers(0, P, P // 3)] = 0x3F800000
    keys = (tiles << np.uint64(32)) | depth
    vals = np.arange(P, dtype=np.uint32)
    ko, vo, rg = ctx.sort_pairs(keys, vals, num_tiles)
    order = np.argsort(keys, kind="stable")
    assert U.bits_equal(ko, keys[order]) and U.bits_equal(vo, vals[order])
    _, _, rr = oracle_sort(keys, vals, num_tiles)
    assert U.bits_equal(rg, rr)


def test_bin_host_arrays_known_answers(ctx):
    """TileBinner with hand-made PreprocessOutput arrays (tests/test_tile_binner.cpp)."""
    cam = S.Camera()
    cam.width, cam.height = 320, 240
    cam.tan_fovx = cam.tan_fovy = 1.0
    cfg = S.render_config(False)
    P, k, v = ctx.bin(cam, cfg, arrays=dict(means2D=[8.0, 8.0], depths=[5.0], radii=[5], tiles_touched=[1]))
    assert P == 1 and (int(k[0]) >> 32) == 0 and v[0] == 0
    assert (int(k[0]) & 0xFFFFFFFF) == int(np.float32(5.0).view(np.uint32))
    P, _, _ = ctx.bin(cam, cfg, arrays=dict(means2D=[8.0, 8.0], depths=[5.0], radii=[0], tiles_touched=[0]))
    assert P == 0
    P, _, _ = ctx.bin(cam, cfg, arrays=dict(means2D=[8, 8, 24, 8, 8, 24], depths=[5.0, 3.0, 7.0], radii=[5, 20, 5],
                                            tiles_touched=[2, 3, 1]))
    assert P == 6
    P, _, _ = ctx.bin(cam, cfg, arrays=dict(means2D=np.zeros(0), depths=np.zeros(0), radii=np.zeros(0, np.int32),
                                            tiles_touched=np.zeros(0, np.int32)))
    assert P == 0


def test_bin_host_arrays_match_oracle(ctx):
    """Binning of a preprocessed scene's host arrays equals the fused preprocess emission."""
    sc, cam, cfg, z = U.load_seeded("render_ragged_100x37_bg")
    P, k, v = ctx.bin(cam, cfg, arrays=dict(means2D=z["means2D"], depths=z["depths"], radii=z["radii"],
                                            tiles_touched=z["tiles"]))
    assert P == int(z["total_pairs"])
    assert U.bits_equal(k, z["keys_unsorted"]) and U.bits_equal(v, z["vals_unsorted"])


def test_grads_ext_forward_fixtures(ctx):
    """Reference golden renders (train/verify_grads_ext) through the CUDA forward."""
    for scene in U.grads_ext_scenes():
        sc, cam, cfg, gt, exp = U.load_grads_fixture(os.path.join(U.REF_FIXTURES, "verify_grads_ext", scene))
        ctx.set_raw_params(sc)
        ctx.preprocess(cam, cfg)
        P, _, _ = ctx.bin(cam, cfg)
        ctx.sort(P, _grid(cam))
        img, _, _ = ctx.rasterize(cam, cfg)
        assert np.abs(img - exp["rendered"]).max() <= IMAGE_ATOL, scene

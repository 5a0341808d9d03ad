"""CPU: pins the oracle (oracle/gs3d_oracle.c) to the reference.

* the reference's own golden vectors (train/verify_grads_ext, train/verify_forward,
  tests/test_data/l1_verify), copied under tests/golden/ref_fixtures/;
* outputs of the reference's CPU stages on seeded scenes (tests/golden/seeded/,
  made by tests/golden/make_golden.py from oracle/_ref);
* the reference's known-answer unit tests (tests/test_sorter.cpp,
  tests/test_tile_binner.cpp), restated.
"""
import ctypes
import json
import os

import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O


def _zero_lr():
    return S.train_config(lr_pos=0.0, lr_rest=0.0, use_adam=False)


@pytest.mark.parametrize("scene", U.grads_ext_scenes())
def test_grads_ext_fixture(scene):
    """verify_grads_main.cpp:47-200 on each fixture: image, loss, raw gradients."""
    sc, cam, cfg, gt, exp = U.load_grads_fixture(os.path.join(U.REF_FIXTURES, "verify_grads_ext", scene))
    r = O.train_step(sc.copy(), cam, gt, cfg, _zero_lr(), 0, O.AdamOracle(sc.count, sc.max_coeffs * 3), "c")
    grads = {"grad_raw_positions": r.g_pos, "grad_raw_scales": r.g_sc, "grad_raw_rotations": r.g_rot,
             "grad_raw_sh_coeffs": r.g_sh, "grad_raw_opacities": r.g_op}
    if scene in U.STALE_GRAD_SCENES:
        assert np.abs(r.image - exp["rendered"]).max() <= 5e-6
        assert abs(r.loss_acc64 - exp["loss"]) <= 1e-6
        for k, v in grads.items():
            ok, worst = U.rel_close(v, exp[k], rtol=2e-4, atol_frac=1e-4)
            assert ok, (k, worst)
    else:
        assert U.bits_equal(r.image, exp["rendered"])
        assert r.loss_acc64 == exp["loss"]
        for k, v in grads.items():
            assert U.bits_equal(v, exp[k]), k


def test_verify_forward_fixture():
    d = os.path.join(U.REF_FIXTURES, "verify_forward")
    sc, cam, cfg, gt, exp = U.load_grads_fixture(d)
    r = O.train_step(sc.copy(), cam, gt, cfg, _zero_lr(), 0, O.AdamOracle(sc.count, sc.max_coeffs * 3), "c")
    assert U.bits_equal(r.image, exp["rendered"])
    py = np.fromfile(os.path.join(d, "py_rendered.bin"), np.float32)
    assert np.abs(r.image - py).max() < 1e-6


def _l1_cases():
    return json.load(open(os.path.join(U.REF_FIXTURES, "l1_verify", "manifest.json")))


@pytest.mark.parametrize("case", _l1_cases(), ids=lambda c: c["name"])
def test_l1_golden(case):
    """tests/test_loss.cpp:142-212: loss within 1e-7 of the serial value, d_image exact."""
    d = os.path.join(U.REF_FIXTURES, "l1_verify")
    H, W, name = case["H"], case["W"], case["name"]
    img = np.fromfile(os.path.join(d, f"{name}_rendered.bin"), np.float32)
    gt = np.fromfile(os.path.join(d, f"{name}_gt.bin"), np.float32)
    dexp = np.fromfile(os.path.join(d, f"{name}_d_image.bin"), np.float32)
    dimg = np.zeros_like(img)
    f = ctypes.POINTER(ctypes.c_float)
    loss = O.lib_c().orc_l1_loss_f32(img.ctypes.data_as(f), gt.ctypes.data_as(f), ctypes.c_int(H), ctypes.c_int(W),
                                     dimg.ctypes.data_as(f))
    assert abs(loss - case["loss_serial"]) < 1e-7
    assert (np.abs(dimg - dexp) > 1e-8).sum() == 0


@pytest.mark.parametrize("name", U.seeded_cases())
def test_seeded_render_matches_reference(name):
    sc, cam, cfg, z = U.load_seeded(name)
    r = O.forward(sc, cam, cfg, "c")
    vis = z["radii"] > 0
    assert U.bits_equal(r.radii, z["radii"]) and U.bits_equal(r.tiles, z["tiles"])
    for k, w in (("depths", 1), ("means2D", 2), ("conics", 3), ("opac2d", 1), ("rgb", 3)):
        assert U.bits_equal(getattr(r, k).reshape(-1, w)[vis], z[k].reshape(-1, w)[vis]), k
    for k in ("cov3D", "p_view", "p_hom_w", "cov2D", "det"):
        assert U.bits_equal(getattr(r, k), z[k]), k
    assert r.total_pairs == int(z["total_pairs"])
    assert U.bits_equal(r.keys_unsorted, z["keys_unsorted"]) and U.bits_equal(r.vals_unsorted, z["vals_unsorted"])
    assert U.bits_equal(r.keys_sorted, z["keys_sorted"]) and U.bits_equal(r.vals_sorted, z["vals_sorted"])
    assert U.bits_equal(r.ranges, z["ranges"])
    assert U.bits_equal(r.image, z["image"]) and U.bits_equal(r.T_final, z["T_final"])
    assert U.bits_equal(r.n_contrib, z["n_contrib"])


def test_seeded_train_matches_reference():
    z = np.load(os.path.join(U.SEEDED, "train_2k_128x128_adam.npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), int(z["in_sh_degree"]))
    cam = S.Camera.from_buffer_copy(z["cam_bytes"].tobytes())
    cfg = S.RenderConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    tc = S.TrainConfig.from_buffer_copy(z["tc_bytes"].tobytes())
    st = O.AdamOracle(sc.count, sc.max_coeffs * 3)
    for it in range(2):
        r = O.train_step(sc, cam, z["gt"], cfg, tc, it, st, "c")
        assert r.loss == z[f"s{it}_loss"] and r.loss_acc64 == z[f"s{it}_loss_acc64"]
        for k in ("image", "d_means2D", "d_conics", "d_rgb", "d_opac", "g_pos", "g_sc", "g_rot", "g_sh", "g_op"):
            assert U.bits_equal(getattr(r, k), z[f"s{it}_{k}"]), (it, k)
        for k in ("positions", "scales", "rotations", "sh", "opacities"):
            assert U.bits_equal(getattr(sc, k), z[f"s{it}_{k}"]), (it, k)


@pytest.mark.parametrize("name", U.eval3d_cases())
def test_eval3d_oracle_matches_reference_fixture(name):
    """The C restatement of the eval_3D forward against the reference's own outputs."""
    sc, f3, cam, cfg, z = U.load_eval3d(name)
    r, ex = O.forward_eval3d(sc, cam, cfg, "c", filter_3d=f3)
    vis = z["radii"] > 0
    assert U.bits_equal(r.radii, z["radii"]) and U.bits_equal(r.tiles, z["tiles"])
    for k, w in (("depths", 1), ("means2D", 2), ("opac2d", 1), ("rgb", 3)):
        assert U.bits_equal(getattr(r, k).reshape(-1, w)[vis], z[k].reshape(-1, w)[vis]), k
    for k in ("gauss2screen", "cov3D_inv", "mean_offset"):
        assert U.bits_equal(ex[k][vis], z[k].reshape(len(vis), -1)[vis]), k
    assert r.total_pairs == int(z["total_pairs"])
    assert U.bits_equal(r.keys_unsorted, z["keys_unsorted"]) and U.bits_equal(r.vals_unsorted, z["vals_unsorted"])
    assert U.bits_equal(r.keys_sorted, z["keys_sorted"]) and U.bits_equal(r.vals_sorted, z["vals_sorted"])
    assert U.bits_equal(r.ranges, z["ranges"])
    assert U.bits_equal(r.image, z["image"]) and U.bits_equal(r.T_final, z["T_final"])
    assert U.bits_equal(r.n_contrib, z["n_contrib"])


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the reference tree)")
def test_eval3d_oracle_matches_reference_live():
    """A fresh seed of the eval_3D forward, both oracles side by side (20k Gaussians, 160x120)."""
    sc = S.eval3d_scene(20_000, seed=98)
    f3 = S.filter_3d_values(20_000, seed=98)
    cam = S.look_at_camera((0.6, -0.3, -2.2), 160, 120, 65.0)
    cfg = S.render_config(False)
    cfg.eval_3D = True
    (a, ea), (b, eb) = (O.forward_eval3d(sc, cam, cfg, impl, filter_3d=f3) for impl in ("c", "ref"))
    vis = b.radii > 0
    assert U.bits_equal(a.radii, b.radii) and U.bits_equal(a.depths[vis], b.depths[vis])
    assert U.bits_equal(ea["gauss2screen"][vis], eb["gauss2screen"][vis])
    assert U.bits_equal(a.keys_unsorted, b.keys_unsorted)
    ka, va = U.canon(a.keys_sorted, a.vals_sorted)
    kb, vb = U.canon(b.keys_sorted, b.vals_sorted)
    assert U.bits_equal(ka, kb) and U.bits_equal(va, vb)
    assert U.bits_equal(a.ranges, b.ranges)
    assert U.bits_equal(a.image, b.image) and U.bits_equal(a.n_contrib, b.n_contrib)


@pytest.mark.parametrize("name", U.density_cases())
def test_density_oracle_matches_reference_fixture(name):
    """densify_and_prune and reset_opacity of the C restatement against the reference's."""
    sc, acc, cfg, extent, z = U.load_density(name)
    ora = O.DensityOracle()
    for d, r in acc:
        ora.accumulate(d, r, sc.count)
    new = ora.densify(sc, cfg, extent)
    assert new.count == int(z["out_count"])
    for k in ("positions", "scales", "rotations", "sh", "opacities"):
        assert U.bits_equal(getattr(new, k), z["out_" + k]), k
    O.DensityOracle.reset_opacity(new)
    assert U.bits_equal(new.opacities, z["out_reset_opacities"])


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the reference tree)")
def test_density_oracle_matches_reference_live():
    """Two rounds (the split sampler's state carries over) on a fresh seed, clones only in
    round 2, so that the reference's compaction reads stay inside its mask."""
    rng = np.random.default_rng(97)
    sc = S.random_scene(650, seed=97)
    sc.scales[:] = np.minimum(sc.scales, np.log(0.0105))
    big = rng.choice(650, 3, replace=False)
    sc.scales[big] = np.log(0.03)
    cfg = S.densify_config(enabled=True)
    ora, ref = O.DensityOracle(), O.DensityRef()
    ref.set_model(sc)
    cur = sc
    for rnd in range(2):
        n = cur.count
        for _ in range(2):
            d = rng.normal(0, 1e-5, (n, 2)).astype(np.float32)
            if rnd == 0:
                d[big] = 1e-3
            else:
                d[: n // 3] = rng.normal(0, 5e-4, (n // 3, 2)).astype(np.float32)
                d[np.exp(cur.scales).max(1) > 0.011] = 0.0   # no second-round splits
            r = rng.integers(0, 25, n).astype(np.int32)
            ora.accumulate(d, r, n)
            ref.accumulate(d, r, n)
        cur = ora.densify(cur, cfg, 1.1)
        assert cur.count == ref.densify(cfg, 1.1)
        got = ref.model()
        for k in ("positions", "scales", "rotations", "sh", "opacities"):
            assert U.bits_equal(getattr(cur, k), getattr(got, k)), (rnd, k)


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the reference tree)")
def test_oracle_matches_reference_live():
    """A fresh seed, both oracles side by side (forward of 20k Gaussians, 320x240)."""
    sc = S.random_scene(20_000, seed=99)
    cam = S.look_at_camera((0.7, -0.4, 2.6), 320, 240, 55.0)
    cfg = S.render_config(False)
    a, b = O.forward(sc, cam, cfg, "c"), O.forward(sc, cam, cfg, "ref")
    vis = b.radii > 0
    assert U.bits_equal(a.radii, b.radii) and U.bits_equal(a.depths[vis], b.depths[vis])
    assert U.bits_equal(a.keys_unsorted, b.keys_unsorted)
    ka, va = U.canon(a.keys_sorted, a.vals_sorted)
    kb, vb = U.canon(b.keys_sorted, b.vals_sorted)
    assert U.bits_equal(ka, kb) and U.bits_equal(va, vb)
    assert U.bits_equal(a.ranges, b.ranges)


# ---- known-answer unit tests of the reference, restated ----

def _sort(keys, vals, num_tiles):
    keys = np.ascontiguousarray(keys, np.uint64)
    vals = np.ascontiguousarray(vals, np.uint32)
    P = len(keys)
    ko, vo = np.zeros(max(P, 1), np.uint64), np.zeros(max(P, 1), np.uint32)
    rg = np.zeros(2 * num_tiles, np.uint32)
    u64, u32 = ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint32)
    O.lib_c().orc_sort(ctypes.c_int64(P), keys.ctypes.data_as(u64), vals.ctypes.data_as(u32),
                       ko.ctypes.data_as(u64), vo.ctypes.data_as(u32), ctypes.c_int(num_tiles), rg.ctypes.data_as(u32))
    return ko[:P], vo[:P], rg


SORTER_CASES = {
    # tests/test_sorter.cpp:6-102
    "basic": ([(1 << 32) | 3, 1, 2], [0, 1, 2], 2, [1, 2, 0], [0, 2, 2, 3]),
    "empty": ([], [], 1, [], [0, 0]),
    "single": ([42], [7], 1, [7], [0, 1]),
    "empty_tile_in_middle": ([1, (2 << 32) | 2], [0, 1], 3, [0, 1], [0, 1, 0, 0, 1, 2]),
}


@pytest.mark.parametrize("case", sorted(SORTER_CASES))
def test_sorter_known_answers(case):
    keys, vals, nt, exp_vals, exp_ranges = SORTER_CASES[case]
    ko, vo, rg = _sort(keys, vals, nt)
    assert list(vo) == exp_vals
    assert list(rg) == exp_ranges
    assert list(ko) == sorted(keys)


def test_binner_known_answers():
    """tests/test_tile_binner.cpp:7-105: tile of a centred Gaussian, zero radius, key = depth bits."""
    cam = S.Camera()
    cam.width, cam.height = 320, 240
    cfg = S.render_config(False)
    f = ctypes.POINTER(ctypes.c_float)
    i = ctypes.POINTER(ctypes.c_int)
    for radius, exp_pairs in ((5, 1), (0, 0)):
        m = np.array([8.0, 8.0], np.float32)
        d = np.array([5.0], np.float32)
        r = np.array([radius], np.int32)
        t = np.array([exp_pairs], np.int32)
        keys, vals = np.zeros(2, np.uint64), np.zeros(2, np.uint32)
        O.lib_c().orc_bin(1, m.ctypes.data_as(f), d.ctypes.data_as(f), r.ctypes.data_as(i), t.ctypes.data_as(i),
                          ctypes.byref(cam), ctypes.byref(cfg), keys.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                          vals.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        if exp_pairs:
            assert keys[0] >> np.uint64(32) == 0 and vals[0] == 0
            assert np.uint32(keys[0] & np.uint64(0xFFFFFFFF)) == np.float32(5.0).view(np.uint32)


def test_fp64_oracle_agrees_with_float_oracle():
    """The FP64 instantiation computes the same function: images within 1e-5,
    gradients with cosine > 0.9999 on a 2k-Gaussian, 128x128 step."""
    sc = S.random_scene(2000)
    cam = S.look_at_camera((0.0, 0.0, -3.0), 128, 128)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "c").image
    cfg = S.render_config(True)
    r = O.train_step(sc.copy(), cam, gt, cfg, _zero_lr(), 0, O.AdamOracle(sc.count, 48), "c")
    loss64, img64, g64 = O.step_f64(sc, cam, cfg, gt)
    assert np.abs(img64.reshape(-1) - r.image).max() < 1e-5
    assert abs(loss64 - r.loss_acc64) < 1e-6
    for k32, k64 in (("g_pos", "pos"), ("g_sc", "sc"), ("g_rot", "rot"), ("g_sh", "sh"), ("g_op", "op")):
        assert U.cosine(getattr(r, k32), g64[k64]) > 0.9999, k32

"""Regenerates the committed golden fixtures under tests/golden/.

    python tests/golden/make_golden.py

Two kinds of fixtures, both produced by the reference itself:

* ref_fixtures/  the reference repository's own golden vectors, copied verbatim
  (data files only): train/verify_grads_ext/<scene>/ (inputs, cpp_rendered.bin,
  cpp_loss.bin, cpp_grad_raw_*.bin), train/verify_forward/, and
  tests/test_data/l1_verify/.
* seeded/        outputs of the reference's CPU stages (oracle/_ref/libgs3d_ref.so,
  built from the reference sources by oracle/Makefile) on seeded synthetic
  scenes, including the edge cases the reference's unit tests cover: ragged
  tiles, non-black background, antialiasing and scale modifier, SH degrees 0-2,
  a single Gaussian, every Gaussian culled, oversized splats; and the 3D-evaluation
  mode (eval_3D) on scenes that reach its frustum culling, camera-inside test and
  view-space bounding box, with and without a 3D filter; and the density
  controller's densify_and_prune (clone, split, prune) and reset_opacity; and the
  drivers' file formats (cameras.json, PLY load / save, PPM).

It needs the reference tree (GS3D_REFERENCE_ROOT; only this script reads it);
the tests and the GPU runs read the committed copies.
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from aaags_claude_b200 import scenes as S  # noqa: E402
from oracle import pyoracle as O  # noqa: E402

REF = O.REF_ROOT


def copy_ref_fixtures():
    dst = os.path.join(HERE, "ref_fixtures")
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    os.makedirs(dst)
    srcs = {f"verify_grads_ext/{d}": os.path.join(REF, "train", "verify_grads_ext", d)
            for d in sorted(os.listdir(os.path.join(REF, "train", "verify_grads_ext")))}
    srcs["verify_forward"] = os.path.join(REF, "train", "verify_forward")
    srcs["l1_verify"] = os.path.join(REF, "tests", "test_data", "l1_verify")
    for name, src in srcs.items():
        out = os.path.join(dst, name)
        os.makedirs(out, exist_ok=True)
        for f in sorted(os.listdir(src)):
            if f.endswith((".bin", ".json")):
                shutil.copyfile(os.path.join(src, f), os.path.join(out, f))
    # the data files of the format tests: the repository's cameras.json and the
    # PLY of its loader test (tests/test_ply_loader.cpp)
    out = os.path.join(dst, "formats")
    os.makedirs(out, exist_ok=True)
    shutil.copyfile(os.path.join(REF, "cameras.json"), os.path.join(out, "cameras.json"))
    shutil.copyfile(os.path.join(REF, "tests", "test_data", "tiny_3gaussians.ply"),
                    os.path.join(out, "tiny_3gaussians.ply"))


# ---- seeded cases ----

def _single_scene():
    s = S.random_scene(1, sh_degree=3, seed=11)
    s.positions[:] = [[0.05, -0.02, 0.0]]
    s.scales[:] = -2.5
    s.opacities[:] = 2.0
    return s


def _culled_scene():
    s = S.random_scene(64, sh_degree=1, seed=12)
    s.positions[:, 2] = 10.0 + s.positions[:, 2]    # behind a camera at z=+3 that looks towards -z
    return s


def _big_scene():
    s = S.random_scene(200, sh_degree=2, seed=13)
    s.scales[:20] = 1.5       # screen radius > max(W, H): culled by the radius test
    s.scales[20:60] = -1.0    # large but kept
    return s


def _scene_with_degree(n, deg, seed):
    return S.random_scene(n, sh_degree=deg, seed=seed)


def render_cases():
    """(name, scene, camera, render config) of the forward fixtures."""
    cam128 = S.look_at_camera((0.0, 0.0, -3.0), 128, 128)
    cases = [
        ("render_2k_128x128", S.random_scene(2000), cam128, S.render_config(False)),
        ("render_ragged_100x37_bg", _scene_with_degree(500, 1, 21),
         S.look_at_camera((0.4, 0.3, -2.5), 100, 37, 50.0), S.render_config(False, 1, bg=(0.2, 0.5, 0.9))),
        ("render_deg0_64x48", _scene_with_degree(300, 0, 22), S.look_at_camera((0.0, 0.0, 3.0), 64, 48),
         S.render_config(False, 0)),
        ("render_deg2_train_80x80", _scene_with_degree(400, 2, 23), S.look_at_camera((1.0, 1.0, -2.5), 80, 80),
         S.render_config(True, 2)),
        ("render_single_33x17", _single_scene(), S.look_at_camera((0.0, 0.0, -3.0), 33, 17),
         S.render_config(False)),
        ("render_all_culled_64x64", _culled_scene(), S.look_at_camera((0.0, 0.0, 3.0), 64, 64),
         S.render_config(False, 1)),
        ("render_oversized_96x64", _big_scene(), S.look_at_camera((0.0, 0.5, -3.0), 96, 64),
         S.render_config(False, 2)),
    ]
    aa = S.render_config(False)
    aa.antialiasing = True
    aa.scale_modifier = 1.7
    cases.append(("render_aa_scale_64x48", S.random_scene(300, seed=24), S.look_at_camera((0.2, -0.1, -3.0), 64, 48),
                  aa))
    return cases


def eval3d_cases():
    """(name, scene, filter_3D or None, camera, render config) of the eval_3D forward fixtures."""
    def e3(cfg):
        cfg.eval_3D = True
        return cfg
    culled = S.eval3d_scene(300, seed=34)
    culled.positions[:, 2] = -6.0 - np.abs(culled.positions[:, 2])   # all behind the camera at z = -3
    bg = e3(S.render_config(True, 1, bg=(0.3, 0.1, 0.6)))
    bg.scale_modifier = 1.3
    return [
        ("eval3d_2k_128x96", S.eval3d_scene(2000, seed=31), S.filter_3d_values(2000, seed=31),
         S.look_at_camera((0.3, 0.2, -3.0), 128, 96), e3(S.render_config(False))),
        ("eval3d_near_96x64", S.eval3d_scene(1500, seed=32), S.filter_3d_values(1500, seed=32),
         S.look_at_camera((0.1, 0.0, -0.6), 96, 64, 70.0), e3(S.render_config(False))),
        ("eval3d_ragged_bg_100x37", S.random_scene(800, sh_degree=1, seed=33), None,
         S.look_at_camera((0.4, 0.3, -2.5), 100, 37, 50.0), bg),
        ("eval3d_all_culled_48x32", culled, None, S.look_at_camera((0.0, 0.0, -3.0), 48, 32),
         e3(S.render_config(False))),
    ]


def make_eval3d():
    dst = os.path.join(HERE, "seeded")
    os.makedirs(dst, exist_ok=True)
    for name, sc, f3, cam, cfg in eval3d_cases():
        r, ex = O.forward_eval3d(sc, cam, cfg, "ref", filter_3d=f3)
        ks, vs = _canon(r.keys_sorted, r.vals_sorted)
        vis = r.radii > 0
        np.savez_compressed(
            os.path.join(dst, name + ".npz"), **scene_arrays(sc), **cam_arrays(cam, cfg),
            filter_3d=np.zeros(0, np.float32) if f3 is None else f3,
            radii=r.radii, tiles=r.tiles, depths=r.depths, means2D=r.means2D, opac2d=r.opac2d, rgb=r.rgb,
            gauss2screen=np.where(vis[:, None], ex["gauss2screen"], 0).astype(np.float32),
            cov3D_inv=ex["cov3D_inv"], mean_offset=ex["mean_offset"],
            total_pairs=np.int64(r.total_pairs), keys_unsorted=r.keys_unsorted, vals_unsorted=r.vals_unsorted,
            keys_sorted=ks, vals_sorted=vs, ranges=r.ranges, image=r.image, T_final=r.T_final,
            n_contrib=r.n_contrib)
        print(name, "visible", int(vis.sum()), "P", r.total_pairs)


def density_cases():
    """(name, scene, accumulations [(d_means2D, radii)], DensifyConfig, extent) of the density fixtures.

    The reference's split compaction reads its removal mask past the end for
    the appended children (density_controller.cpp:78 with train_types.h:119-124);
    the cases keep those reads inside the mask's last 64-bit word, which its
    constructor zero-fills, so the reference's result is defined: either no
    split at all, or N + clones = 650 (bits 650.. of a 704-bit mask) with three
    splits."""
    out = []
    for name, seed, n, n_big, frac in (("density_clone_prune_3000", 41, 3000, 0, 0.3),
                                       ("density_split_650_a", 42, 650, 3, 0.0),
                                       ("density_split_650_b", 43, 650, 3, 0.0)):
        rng = np.random.default_rng(seed)
        sc = S.random_scene(n, seed=seed)
        sc.scales[:] = np.minimum(sc.scales, np.log(0.0105))
        big = rng.choice(n, n_big, replace=False)
        sc.scales[big] = np.log(0.03)
        sc.opacities[rng.random(n) < 0.03] = -7.0
        hot = rng.random(n) < frac
        hot[big] = True
        acc = []
        for _ in range(3):
            d = rng.normal(0, 1e-5, (n, 2)).astype(np.float32)
            d[hot] = rng.normal(0, 5e-4, (int(hot.sum()), 2)).astype(np.float32)
            acc.append((d, rng.integers(0, 25, n).astype(np.int32)))
        out.append((name, sc, acc, S.densify_config(enabled=True), 1.1))
    return out


def make_density():
    dst = os.path.join(HERE, "seeded")
    for name, sc, acc, cfg, extent in density_cases():
        ref = O.DensityRef()
        ref.set_model(sc)
        for d, r in acc:
            ref.accumulate(d, r, sc.count)
        k = ref.densify(cfg, extent)
        got = ref.model()
        ref.reset_opacity()
        reset_op = ref.model().opacities
        np.savez_compressed(
            os.path.join(dst, name + ".npz"), **scene_arrays(sc),
            acc_d_means2D=np.stack([d for d, _ in acc]), acc_radii=np.stack([r for _, r in acc]),
            cfg_bytes=np.frombuffer(bytes(cfg), np.uint8), extent=np.float32(extent), out_count=np.int32(k),
            out_positions=got.positions, out_scales=got.scales, out_rotations=got.rotations, out_sh=got.sh,
            out_opacities=got.opacities, out_reset_opacities=reset_op)
        print(name, sc.count, "->", k)


def make_formats():
    """The reference's loaders on the format fixtures: cameras.json -> cameras, the
    tiny PLY -> activated model and raw parameters, savePly of those raw
    parameters, and a writePPM / readPPM round trip of a seeded image."""
    import ctypes
    fx = os.path.join(HERE, "ref_fixtures", "formats")
    L = O.lib_ref()
    out = {}
    cams = (S.Camera * 256)()
    names = ctypes.create_string_buffer(256 * 64)
    n = L.ref_io_cameras(os.path.join(fx, "cameras.json").encode(), cams, names, 64, 256)
    out["cam_count"] = np.int32(n)
    out["cam_bytes"] = np.frombuffer(bytes(cams)[: n * ctypes.sizeof(S.Camera)], np.uint8)
    out["cam_names"] = np.array([names.raw[i * 64:(i + 1) * 64].split(b"\0")[0].decode() for i in range(n)])
    ply = os.path.join(fx, "tiny_3gaussians.ply").encode()
    cnt, deg, mc, hf = (ctypes.c_int() for _ in range(4))
    L.ref_io_ply_count(ply, ctypes.byref(cnt), ctypes.byref(deg), ctypes.byref(mc), ctypes.byref(hf))
    n, k = cnt.value, mc.value
    act = dict(positions=np.zeros(3 * n, np.float32), scales=np.zeros(3 * n, np.float32),
               rotations=np.zeros(4 * n, np.float32), sh_coeffs=np.zeros(3 * k * n, np.float32),
               opacities=np.zeros(n, np.float32))
    sc = S.Scene(np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
                 np.zeros((n, k, 3), np.float32), np.zeros(n, np.float32), deg.value)
    g = O.gaussians_struct(sc, act)
    L.ref_io_ply_load(ply, ctypes.byref(g))
    out.update({"ply_" + a: b for a, b in act.items()})
    out["ply_shape"] = np.array([n, deg.value, k, hf.value], np.int32)
    raw = sc.raw_struct()
    L.ref_io_raw_from_gaussians(ctypes.byref(g), ctypes.byref(raw))
    out.update(raw_positions=sc.positions.copy(), raw_scales=sc.scales.copy(), raw_rotations=sc.rotations.copy(),
               raw_sh=sc.sh.copy(), raw_opacities=sc.opacities.copy())
    tmp = os.path.join(HERE, "_tmp_saved.ply")
    L.ref_io_ply_save(tmp.encode(), ctypes.byref(raw))
    out["saved_ply_bytes"] = np.frombuffer(open(tmp, "rb").read(), np.uint8)
    os.remove(tmp)
    rng = np.random.default_rng(5)
    img = rng.uniform(-0.2, 1.2, (37, 23, 3)).astype(np.float32)
    tmp = os.path.join(HERE, "_tmp.ppm")
    L.ref_io_ppm_write(tmp.encode(), img.ctypes.data_as(ctypes.c_void_p), 23, 37)
    out["ppm_in"] = img
    out["ppm_bytes"] = np.frombuffer(open(tmp, "rb").read(), np.uint8)
    back = np.zeros(37 * 23 * 3, np.float32)
    w, h = ctypes.c_int(), ctypes.c_int()
    L.ref_io_ppm_read(tmp.encode(), back.ctypes.data_as(ctypes.c_void_p), ctypes.byref(w), ctypes.byref(h))
    os.remove(tmp)
    out["ppm_read"] = back
    np.savez_compressed(os.path.join(HERE, "seeded", "formats_ref.npz"), **out)
    print("formats: cameras", int(out["cam_count"]), "ply", n)


def _canon(keys, vals):
    o = np.lexsort((vals, keys))
    return keys[o], vals[o]


def scene_arrays(s):
    return dict(in_positions=s.positions, in_scales=s.scales, in_rotations=s.rotations, in_sh=s.sh,
                in_opacities=s.opacities, in_sh_degree=np.int32(s.sh_degree))


def cam_arrays(cam, cfg):
    return dict(cam_bytes=np.frombuffer(bytes(cam), np.uint8), cfg_bytes=np.frombuffer(bytes(cfg), np.uint8))


def make_seeded():
    dst = os.path.join(HERE, "seeded")
    os.makedirs(dst, exist_ok=True)
    for name, sc, cam, cfg in render_cases():
        r = O.forward(sc, cam, cfg, "ref")
        ks, vs = _canon(r.keys_sorted, r.vals_sorted)
        np.savez_compressed(
            os.path.join(dst, name + ".npz"), **scene_arrays(sc), **cam_arrays(cam, cfg),
            radii=r.radii, tiles=r.tiles, depths=r.depths, means2D=r.means2D, conics=r.conics,
            opac2d=r.opac2d, rgb=r.rgb, cov3D=r.cov3D, p_view=r.p_view, p_hom_w=r.p_hom_w, cov2D=r.cov2D,
            det=r.det, total_pairs=np.int64(r.total_pairs), keys_unsorted=r.keys_unsorted,
            vals_unsorted=r.vals_unsorted, keys_sorted=ks, vals_sorted=vs, ranges=r.ranges, image=r.image,
            T_final=r.T_final, n_contrib=r.n_contrib)
        print(name, "P", r.total_pairs)
    # training: two Adam steps of Trainer::step on the 2k scene
    sc = S.random_scene(2000)
    cam = S.look_at_camera((0.0, 0.0, -3.0), 128, 128)
    gt = O.forward(S.perturbed(sc), cam, S.render_config(False), "ref").image
    cfg, tc = S.render_config(True), S.train_config()
    work = sc.copy()
    adam = O.RefAdam()
    out = dict(**scene_arrays(sc), **cam_arrays(cam, cfg), tc_bytes=np.frombuffer(bytes(tc), np.uint8), gt=gt)
    for it in range(2):
        r = O.train_step(work, cam, gt, cfg, tc, it, adam, "ref")
        out.update({f"s{it}_loss": np.float32(r.loss), f"s{it}_loss_acc64": np.float64(r.loss_acc64),
                    f"s{it}_image": r.image, f"s{it}_d_means2D": r.d_means2D, f"s{it}_d_conics": r.d_conics,
                    f"s{it}_d_rgb": r.d_rgb, f"s{it}_d_opac": r.d_opac, f"s{it}_g_pos": r.g_pos,
                    f"s{it}_g_sc": r.g_sc, f"s{it}_g_rot": r.g_rot, f"s{it}_g_sh": r.g_sh, f"s{it}_g_op": r.g_op,
                    f"s{it}_positions": work.positions.copy(), f"s{it}_scales": work.scales.copy(),
                    f"s{it}_rotations": work.rotations.copy(), f"s{it}_sh": work.sh.copy(),
                    f"s{it}_opacities": work.opacities.copy()})
    np.savez_compressed(os.path.join(dst, "train_2k_128x128_adam.npz"), **out)
    print("train_2k_128x128_adam")


if __name__ == "__main__":
    O.ensure_built(ref=True)
    if not O.have_ref():
        sys.exit("oracle/_ref/libgs3d_ref.so is missing: `make -C oracle ref` needs the reference tree")
    copy_ref_fixtures()
    make_seeded()
    make_eval3d()
    make_density()
    make_formats()

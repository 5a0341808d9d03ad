"""GPU: the C++ stage adapters (aaags_claude_b200/host) driven through the
reference's abstract interfaces by tests/native/stages_demo.cpp -- the drop-in
boundary as a maintainer would wire it into Renderer / Trainer."""
import os
import subprocess

import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import build
from aaags_claude_b200 import scenes as S
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def _rd(d, name, dtype=np.float32):
    return np.fromfile(os.path.join(d, name), dtype=dtype)


HERE = os.path.dirname(os.path.abspath(__file__))


def _demo(tmp_path) -> str:
    """Compiles the driver with the adapters and links it against the in-tree library."""
    exe = os.path.join(str(tmp_path), "stages_demo")
    lib_dir = os.path.dirname(build.LIB)
    subprocess.run([os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", f"-I{build.INCLUDE}",
                    f"-I{build.HOST}", os.path.join(build.HOST, "gs3d_stages_cuda.cpp"),
                    os.path.join(HERE, "native", "stages_demo.cpp"), "-o", exe, f"-L{lib_dir}", "-lgs3d_cuda",
                    f"-Wl,-rpath,{lib_dir}"], check=True)
    return exe


def test_stage_adapters_match_the_reference(tmp_path):
    build.build()
    demo = _demo(tmp_path)
    z = np.load(os.path.join(U.SEEDED, "train_2k_128x128_adam.npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), 3)
    d = str(tmp_path)
    for name, arr in (("raw_positions", sc.positions), ("raw_scales", sc.scales), ("raw_rotations", sc.rotations),
                      ("raw_sh_coeffs", sc.sh), ("raw_opacities", sc.opacities), ("gt_image", z["gt"])):
        np.ascontiguousarray(arr, np.float32).tofile(os.path.join(d, name + ".bin"))
    z["cam_bytes"].tofile(os.path.join(d, "camera.bin"))
    z["cfg_bytes"].tofile(os.path.join(d, "render_config.bin"))
    z["tc_bytes"].tofile(os.path.join(d, "train_config.bin"))
    open(os.path.join(d, "meta.txt"), "w").write(f"{sc.count} 3 16 2\n")
    r = subprocess.run([demo, d], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    cam = S.Camera.from_buffer_copy(z["cam_bytes"].tobytes())
    cfg = S.RenderConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    ref = O.forward(sc, cam, cfg, "c")
    # forward through Preprocessor / TileBinner / Sorter / Rasterizer: integer outputs exact
    assert U.bits_equal(_rd(d, "out_radii.bin", np.int32), ref.radii)
    assert U.bits_equal(_rd(d, "out_tiles.bin", np.int32), ref.tiles)
    assert U.bits_equal(_rd(d, "out_keys_unsorted.bin", np.uint64), ref.keys_unsorted)
    assert U.bits_equal(_rd(d, "out_vals_unsorted.bin", np.uint32), ref.vals_unsorted)
    assert U.bits_equal(_rd(d, "out_keys_sorted.bin", np.uint64), ref.keys_sorted)
    assert U.bits_equal(_rd(d, "out_vals_sorted.bin", np.uint32), ref.vals_sorted)
    assert U.bits_equal(_rd(d, "out_ranges.bin", np.uint32), ref.ranges)
    assert np.abs(_rd(d, "out_image.bin") - z["s0_image"]).max() <= 1e-5
    assert U.bits_equal(_rd(d, "out_n_contrib.bin", np.int32), ref.n_contrib)
    # stage backward from the activated device model
    for k in ("g_pos", "g_sc", "g_rot", "g_sh", "g_op"):
        ok, worst = U.rel_close(_rd(d, f"out_{k}.bin"), z[f"s0_{k}"], 1e-4, 1e-5)
        assert ok, (k, worst)
    # TrainerCUDA::step, caller's parameters updated in place, two Adam steps
    losses = _rd(d, "out_losses.bin")
    for it in range(2):
        assert abs(losses[it] - z[f"s{it}_loss_acc64"]) <= 1e-6 * z[f"s{it}_loss_acc64"]
    for k, f in (("positions", "pos"), ("scales", "sc"), ("rotations", "rot"), ("sh", "sh"), ("opacities", "op")):
        assert np.abs(_rd(d, f"out_params_{f}.bin") - z[f"s1_{k}"].reshape(-1)).max() <= 1e-5, k
    assert np.abs(_rd(d, "out_last_rendered.bin") - z["s1_image"]).max() <= 1e-5

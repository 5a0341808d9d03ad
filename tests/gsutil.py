"""Helpers shared by the tests: fixture loading and comparisons."""
from __future__ import annotations

import json
import os

import numpy as np

from aaags_claude_b200 import scenes as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_FIXTURES = os.path.join(GOLDEN, "ref_fixtures")
SEEDED = os.path.join(GOLDEN, "seeded")

# The 4 "many_30g" scenes were pinned by an older reference build; the current
# reference sources reproduce them only to ~3e-6 (image) / 1e-4 (gradients).
STALE_GRAD_SCENES = {"many_30g_16x16_sh0", "many_30g_offset_0.1", "many_30g_offset_0.5", "many_30g_offset_2.0"}


def grads_ext_scenes():
    d = os.path.join(REF_FIXTURES, "verify_grads_ext")
    return sorted(os.listdir(d))


def _rd(path, dtype=np.float32):
    return np.fromfile(path, dtype=dtype)


def load_grads_fixture(path: str):
    """A reference gradient fixture: (scene, camera, cfg, gt, expected dict)."""
    meta = json.load(open(os.path.join(path, "meta.json")))
    n, W, H, deg, mc = meta["N"], meta["W"], meta["H"], meta["sh_degree"], meta["max_coeffs"]
    sc = S.Scene(_rd(os.path.join(path, "raw_positions.bin")).reshape(n, 3).copy(),
                 _rd(os.path.join(path, "raw_scales.bin")).reshape(n, 3).copy(),
                 _rd(os.path.join(path, "raw_rotations.bin")).reshape(n, 4).copy(),
                 _rd(os.path.join(path, "raw_sh_coeffs.bin")).reshape(n, mc, 3).copy(),
                 _rd(os.path.join(path, "raw_opacities.bin")).reshape(n).copy(), deg)
    cam = S.Camera()
    cam.view_matrix[:] = _rd(os.path.join(path, "view_matrix.bin")).tolist()
    cam.viewproj_matrix[:] = _rd(os.path.join(path, "viewproj_matrix.bin")).tolist()
    cam.cam_pos[:] = [0.0, 0.0, 0.0]   # the reference driver fixes cam_pos to 0 (verify_grads_main.cpp:109)
    cam.tan_fovx, cam.tan_fovy = float(meta["tan_fovx"]), float(meta["tan_fovy"])
    cam.width, cam.height = W, H
    cfg = S.render_config(True, deg)
    gt = _rd(os.path.join(path, "gt_image.bin"))
    exp = {}
    for k in ("rendered", "grad_raw_positions", "grad_raw_scales", "grad_raw_rotations", "grad_raw_sh_coeffs",
              "grad_raw_opacities"):
        p = os.path.join(path, f"cpp_{k}.bin")
        if os.path.exists(p):
            exp[k] = _rd(p)
    lp = os.path.join(path, "cpp_loss.bin")
    if os.path.exists(lp):
        exp["loss"] = float(_rd(lp, np.float64)[0])
    return sc, cam, cfg, gt, exp


def seeded_cases():
    return sorted(f[:-4] for f in os.listdir(SEEDED) if f.startswith("render_"))


def load_seeded(name: str):
    z = np.load(os.path.join(SEEDED, name + ".npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), int(z["in_sh_degree"]))
    cam = S.Camera.from_buffer_copy(z["cam_bytes"].tobytes())
    cfg = S.RenderConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    return sc, cam, cfg, z


def activate_cr(scene) -> dict:
    """RawGaussianParams::activate (train_types.cpp:6-36) in float32 with a correctly
    rounded exp -- the device's activation -- for checks of the raw-model path
    (glibc's expf, which the reference and the C oracle call, is 1 ulp off on a
    few inputs in 1e5)."""
    f = np.float32
    q = np.ascontiguousarray(scene.rotations, f).reshape(-1, 4)
    ln = np.sqrt(((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3])
    ln = np.where(ln < f(1e-12), f(1e-12), ln).astype(f)
    inv = (f(1.0) / ln).astype(f)
    e = np.exp(-np.asarray(scene.opacities, np.float64)).astype(f)
    return dict(positions=np.ascontiguousarray(scene.positions, f).reshape(-1),
                scales=np.exp(np.asarray(scene.scales, np.float64)).astype(f).reshape(-1),
                rotations=(q * inv[:, None]).astype(f).reshape(-1),
                sh_coeffs=np.ascontiguousarray(scene.sh, f).reshape(-1),
                opacities=(f(1.0) / (f(1.0) + e)).astype(f))


def eval3d_cases():
    return sorted(f[:-4] for f in os.listdir(SEEDED) if f.startswith("eval3d_"))


def load_eval3d(name: str):
    """(scene, filter_3D or None, camera, render config, fixture) of an eval_3D golden case."""
    sc, cam, cfg, z = load_seeded(name)
    f3 = z["filter_3d"] if z["filter_3d"].size else None
    return sc, f3, cam, cfg, z


def density_cases():
    return sorted(f[:-4] for f in os.listdir(SEEDED) if f.startswith("density_"))


def load_density(name: str):
    """(scene, accumulations [(d_means2D, radii)], DensifyConfig, extent, fixture) of a density case."""
    z = np.load(os.path.join(SEEDED, name + ".npz"))
    sc = S.Scene(z["in_positions"].copy(), z["in_scales"].copy(), z["in_rotations"].copy(), z["in_sh"].copy(),
                 z["in_opacities"].copy(), int(z["in_sh_degree"]))
    acc = list(zip(z["acc_d_means2D"], z["acc_radii"]))
    cfg = S.DensifyConfig.from_buffer_copy(z["cfg_bytes"].tobytes())
    return sc, acc, cfg, float(z["extent"]), z


def canon(keys, vals):
    """(key, value)-sorted order: the reference's std::sort leaves equal keys unordered."""
    o = np.lexsort((vals, keys))
    return keys[o], vals[o]


def bits_equal(a, b) -> bool:
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64),
                              b.view(np.uint32 if b.dtype.itemsize == 4 else np.uint64))
    return np.array_equal(a, b)


def rel_close(a, b, rtol: float, atol_frac: float = 0.0) -> tuple[bool, float]:
    """|a-b| <= rtol*|b| + atol_frac*max|b| elementwise; returns (ok, worst ratio)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    tol = rtol * np.abs(b) + atol_frac * scale + 1e-30
    r = np.abs(a - b) / tol
    return bool((r <= 1.0).all()), float(r.max() if r.size else 0.0)


def cosine(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-300))


def fd_picks(lengths, n: int = 200, seed: int = 3):
    """(group, index) of n random raw parameters, groups drawn uniformly."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        grp = int(rng.integers(len(lengths)))
        out.append((grp, int(rng.integers(lengths[grp]))))
    return out


def fd_within(fd, ana):
    """The reference's finite-difference tolerance (tools/verify_gradients_extended.py:455-490)."""
    fd, ana = np.asarray(fd), np.asarray(ana)
    return np.abs(fd - ana) <= 5e-5 * np.abs(fd).max() + 0.10 * np.maximum(np.abs(fd), np.abs(ana))

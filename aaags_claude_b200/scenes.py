"""Seeded synthetic scenes and cameras for the 3DGS render/train workloads.

The reference measures on real PLY scenes that are not available here; these
generators stand in for them with the distributions of the benchmark configs:

* ``random_scene``     means ~ N(0, 0.5^2 I3), log-scales ~ N(-4.5, 0.5^2),
                       rotations = normalised N(0, I4) quaternions,
                       opacity logits ~ N(0, 1), SH degree 3 with DC ~ N(0, 0.5^2)
                       and higher bands ~ N(0, 0.05^2);
* ``clustered_scene``  the same attributes, means from 64 isotropic clusters
                       (centres uniform in [-2, 2]^3, sigma 0.15);
* ``perturbed``        the target scene: means + N(0, 0.01^2), DC colours +
                       N(0, 0.05^2), opacity logits + N(0, 0.2^2);
* ``look_at_camera``   a pinhole camera built like the reference's render CLI
                       (harmonyos_3dgs src/main.cpp:28-74 look-at + perspective,
                       viewproj = proj * view as at src/main.cpp:133-138).

Seeds follow one convention: 0 = scene, 1 = target perturbation, 2 = cameras,
3 = finite-difference parameter choice.  All arrays are float32 in the
reference layouts (``include/gs3d_types.h``).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

SEED_SCENE, SEED_TARGET, SEED_CAMERA, SEED_FD = 0, 1, 2, 3


class Camera(ctypes.Structure):
    """Layout of ``gs3d_camera`` (= the reference's ``Camera``)."""

    _fields_ = [
        ("view_matrix", ctypes.c_float * 16),
        ("viewproj_matrix", ctypes.c_float * 16),
        ("cam_pos", ctypes.c_float * 3),
        ("tan_fovx", ctypes.c_float),
        ("tan_fovy", ctypes.c_float),
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
    ]


class RenderConfig(ctypes.Structure):
    """Layout of ``gs3d_render_config`` (= the reference's ``RenderConfig``)."""

    _fields_ = [
        ("bg_color", ctypes.c_float * 3),
        ("scale_modifier", ctypes.c_float),
        ("antialiasing", ctypes.c_bool),
        ("eval_3D", ctypes.c_bool),
        ("training", ctypes.c_bool),
        ("sh_degree", ctypes.c_int),
        ("tile_w", ctypes.c_int),
        ("tile_h", ctypes.c_int),
    ]


class TrainConfig(ctypes.Structure):
    """Layout of ``gs3d_train_config`` (= the reference's ``TrainConfig``)."""

    _fields_ = [
        ("lr_position_init", ctypes.c_float),
        ("lr_position_final", ctypes.c_float),
        ("lr_feature", ctypes.c_float),
        ("lr_opacity", ctypes.c_float),
        ("lr_scaling", ctypes.c_float),
        ("lr_rotation", ctypes.c_float),
        ("max_steps", ctypes.c_int),
        ("use_adam", ctypes.c_bool),
        ("adam_beta1", ctypes.c_float),
        ("adam_beta2", ctypes.c_float),
        ("adam_eps", ctypes.c_float),
    ]


class DensifyConfig(ctypes.Structure):
    """Layout of ``gs3d_densify_config`` (= the reference's ``DensifyConfig``)."""

    _fields_ = [
        ("densify_from_iter", ctypes.c_int),
        ("densify_until_iter", ctypes.c_int),
        ("densify_interval", ctypes.c_int),
        ("grad_threshold", ctypes.c_float),
        ("min_opacity", ctypes.c_float),
        ("percent_dense", ctypes.c_float),
        ("opacity_reset_interval", ctypes.c_int),
        ("max_screen_size", ctypes.c_int),
        ("enabled", ctypes.c_bool),
    ]


def densify_config(**kw) -> DensifyConfig:
    """DensifyConfig with the reference's defaults (train_types.h:71-81), overridden by kw."""
    d = DensifyConfig()
    vals = dict(densify_from_iter=500, densify_until_iter=15000, densify_interval=100, grad_threshold=0.0002,
                min_opacity=0.005, percent_dense=0.01, opacity_reset_interval=3000, max_screen_size=20,
                enabled=False)
    vals.update(kw)
    for k, v in vals.items():
        setattr(d, k, v)
    return d


class GaussianData(ctypes.Structure):
    """Layout of ``gs3d_gaussians`` (= the reference's ``GaussianData``)."""

    _fields_ = [
        ("count", ctypes.c_int),
        ("sh_degree", ctypes.c_int),
        ("max_coeffs", ctypes.c_int),
        ("positions", ctypes.POINTER(ctypes.c_float)),
        ("sh_coeffs", ctypes.POINTER(ctypes.c_float)),
        ("scales", ctypes.POINTER(ctypes.c_float)),
        ("rotations", ctypes.POINTER(ctypes.c_float)),
        ("opacities", ctypes.POINTER(ctypes.c_float)),
        ("filter_3D", ctypes.POINTER(ctypes.c_float)),
    ]


class RawParams(ctypes.Structure):
    """Layout of ``gs3d_raw_params`` (= the reference's ``RawGaussianParams``)."""

    _fields_ = [
        ("count", ctypes.c_int),
        ("sh_degree", ctypes.c_int),
        ("max_coeffs", ctypes.c_int),
        ("raw_positions", ctypes.POINTER(ctypes.c_float)),
        ("raw_scales", ctypes.POINTER(ctypes.c_float)),
        ("raw_rotations", ctypes.POINTER(ctypes.c_float)),
        ("raw_sh_coeffs", ctypes.POINTER(ctypes.c_float)),
        ("raw_opacities", ctypes.POINTER(ctypes.c_float)),
    ]


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


@dataclass
class Scene:
    """Raw (pre-activation) parameters in the reference layouts."""

    positions: np.ndarray   # [N,3]
    scales: np.ndarray      # [N,3] log scale
    rotations: np.ndarray   # [N,4] (r,x,y,z), not necessarily unit
    sh: np.ndarray          # [N,K,3]
    opacities: np.ndarray   # [N] logits
    sh_degree: int = 3

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])

    @property
    def max_coeffs(self) -> int:
        return int(self.sh.shape[1])

    def copy(self) -> "Scene":
        return Scene(self.positions.copy(), self.scales.copy(), self.rotations.copy(),
                     self.sh.copy(), self.opacities.copy(), self.sh_degree)

    def raw_struct(self) -> RawParams:
        """A ``gs3d_raw_params`` view over this scene's arrays (no copy)."""
        r = RawParams()
        r.count, r.sh_degree, r.max_coeffs = self.count, self.sh_degree, self.max_coeffs
        r.raw_positions = fptr(self.positions)
        r.raw_scales = fptr(self.scales)
        r.raw_rotations = fptr(self.rotations)
        r.raw_sh_coeffs = fptr(self.sh)
        r.raw_opacities = fptr(self.opacities)
        r._keep = self  # keep arrays alive with the struct
        return r


def _draw_attributes(rng: np.random.Generator, n: int, sh_degree: int):
    k = (sh_degree + 1) ** 2
    scales = rng.normal(-4.5, 0.5, size=(n, 3)).astype(np.float32)
    q = rng.normal(0.0, 1.0, size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    rotations = q.astype(np.float32)
    sh = np.empty((n, k, 3), np.float32)
    sh[:, 0, :] = rng.normal(0.0, 0.5, size=(n, 3))
    if k > 1:
        sh[:, 1:, :] = rng.normal(0.0, 0.05, size=(n, k - 1, 3))
    opac = rng.normal(0.0, 1.0, size=n).astype(np.float32)
    return scales, rotations, sh, opac


def random_scene(n: int, sh_degree: int = 3, seed: int = SEED_SCENE) -> Scene:
    rng = np.random.default_rng(seed)
    pos = rng.normal(0.0, 0.5, size=(n, 3)).astype(np.float32)
    sc, rot, sh, op = _draw_attributes(rng, n, sh_degree)
    return Scene(pos, sc, rot, sh, op, sh_degree)


def eval3d_scene(n: int, seed: int = SEED_SCENE, spread: float = 1.5, sh_degree: int = 3) -> Scene:
    """A scene that reaches every branch of the 3D-evaluation mode's preprocess:
    means ~ N(0, spread^2 I3) (many outside the view frustum, some behind or close to
    the camera), log-scales ~ N(-2.5, 1) (large Gaussians crossing the screen border and
    the near plane, so the view-space bounding box is used), and 5 % with opacity logits
    near -7 (below 1/255 once the mip filter dilates them)."""
    rng = np.random.default_rng(seed)
    pos = rng.normal(0.0, spread, size=(n, 3)).astype(np.float32)
    sc, rot, sh, op = _draw_attributes(rng, n, sh_degree)
    sc = rng.normal(-2.5, 1.0, size=(n, 3)).astype(np.float32)
    low = rng.random(n) < 0.05
    op[low] = rng.normal(-7.0, 0.5, size=int(low.sum())).astype(np.float32)
    return Scene(pos, sc, rot, sh, op, sh_degree)


def filter_3d_values(n: int, seed: int = SEED_SCENE) -> np.ndarray:
    """Per-Gaussian 3D mip filter sizes (GaussianData::filter_3D): |N(0, 0.01^2)|."""
    return np.abs(np.random.default_rng(seed + 1).normal(0.0, 0.01, size=n)).astype(np.float32)


def clustered_scene(n: int, clusters: int = 64, sigma: float = 0.15, sh_degree: int = 3,
                    seed: int = SEED_SCENE) -> Scene:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-2.0, 2.0, size=(clusters, 3))
    which = rng.integers(0, clusters, size=n)
    pos = (centres[which] + rng.normal(0.0, sigma, size=(n, 3))).astype(np.float32)
    sc, rot, sh, op = _draw_attributes(rng, n, sh_degree)
    return Scene(pos, sc, rot, sh, op, sh_degree)


def perturbed(scene: Scene, seed: int = SEED_TARGET) -> Scene:
    """The target scene of the training configs."""
    rng = np.random.default_rng(seed)
    t = scene.copy()
    n = scene.count
    t.positions += rng.normal(0.0, 0.01, size=(n, 3)).astype(np.float32)
    t.sh[:, 0, :] += rng.normal(0.0, 0.05, size=(n, 3)).astype(np.float32)
    t.opacities += rng.normal(0.0, 0.2, size=n).astype(np.float32)
    return t


def look_at_camera(eye, width: int, height: int, fovy_deg: float = 60.0,
                   center=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0),
                   znear: float = 0.2, zfar: float = 100.0) -> Camera:
    """Pinhole camera at ``eye`` looking at ``center``; ``fovy_deg`` is vertical."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(center, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    view = np.zeros(16, np.float64)   # column-major, rows = (r, u, f)
    view[0], view[4], view[8] = r
    view[1], view[5], view[9] = u
    view[2], view[6], view[10] = f
    view[12] = -r.dot(eye)
    view[13] = -u.dot(eye)
    view[14] = -f.dot(eye)
    view[15] = 1.0
    tan_fovy = math.tan(math.radians(fovy_deg) * 0.5)
    tan_fovx = tan_fovy * width / height
    proj = np.zeros(16, np.float64)
    proj[0] = 1.0 / tan_fovx
    proj[5] = 1.0 / tan_fovy
    proj[10] = zfar / (zfar - znear)
    proj[11] = 1.0
    proj[14] = -(zfar * znear) / (zfar - znear)
    P = proj.reshape(4, 4).T          # column-major -> math matrix
    V = view.reshape(4, 4).T
    vp = (P @ V).T.reshape(16)
    cam = Camera()
    cam.view_matrix[:] = [float(np.float32(x)) for x in view]
    cam.viewproj_matrix[:] = [float(np.float32(x)) for x in vp]
    cam.cam_pos[:] = [float(np.float32(x)) for x in eye]
    cam.tan_fovx = float(np.float32(tan_fovx))
    cam.tan_fovy = float(np.float32(tan_fovy))
    cam.width, cam.height = int(width), int(height)
    return cam


def sphere_cameras(count: int, radius: float = 3.0, seed: int = SEED_CAMERA,
                   resolutions=None, fov_range=None):
    """``count`` cameras at uniform random points of a sphere looking at the origin.

    ``resolutions`` (list of (W, H)) and ``fov_range`` ((lo, hi) degrees) are
    sampled uniformly when given; otherwise 1920x1080 at 60 degrees.
    """
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(count):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if abs(d[1]) > 0.99:   # keep the look-at up vector well defined
            d[1] = 0.99 * np.sign(d[1])
            d /= np.linalg.norm(d)
        w, h = (1920, 1080) if resolutions is None else resolutions[rng.integers(len(resolutions))]
        fov = 60.0 if fov_range is None else float(rng.uniform(*fov_range))
        cams.append(look_at_camera(d * radius, w, h, fov))
    return cams


def render_config(training: bool, sh_degree: int = 3, bg=(0.0, 0.0, 0.0)) -> RenderConfig:
    c = RenderConfig()
    c.bg_color[:] = bg
    c.scale_modifier = 1.0
    c.antialiasing = False
    c.eval_3D = False
    c.training = training
    c.sh_degree = sh_degree
    c.tile_w = 16
    c.tile_h = 16
    return c


def train_config(lr_pos: float = 1.6e-4, lr_rest: float = 1e-3, use_adam: bool = True,
                 max_steps: int = 30000) -> TrainConfig:
    """Adam with position lr fixed (init = final) and one lr for the other groups."""
    t = TrainConfig()
    t.lr_position_init = lr_pos
    t.lr_position_final = lr_pos
    t.lr_feature = lr_rest
    t.lr_opacity = lr_rest
    t.lr_scaling = lr_rest
    t.lr_rotation = lr_rest
    t.max_steps = max_steps
    t.use_adam = use_adam
    t.adam_beta1 = 0.9
    t.adam_beta2 = 0.999
    t.adam_eps = 1e-8
    return t


@dataclass
class Workload:
    """One benchmark configuration: scene, cameras and (for training) a target scene."""

    name: str
    scene: Scene
    cameras: list
    target_scene: Scene | None = None
    meta: dict = field(default_factory=dict)


def config_render_100k() -> Workload:
    """Plain forward render: N=100k, one 640x480 camera 3 units from the origin."""
    s = random_scene(100_000)
    cam = look_at_camera((0.0, 0.0, -3.0), 640, 480, 60.0)
    return Workload("render_100k_640x480", s, [cam])


def config_render_eval3d() -> Workload:
    """3D-evaluation render (eval_3D): N=100k random Gaussians, one 640x480 camera 3 units away."""
    s = random_scene(100_000)
    cam = look_at_camera((0.0, 0.0, -3.0), 640, 480, 60.0)
    return Workload("render_eval3d_100k_640x480", s, [cam])


def config_train_1m_1080p() -> Workload:
    """Plain training step: N=1M, one 1920x1080 camera on the radius-3 sphere."""
    s = random_scene(1_000_000)
    cams = sphere_cameras(1)
    return Workload("train_1M_1920x1080", s, cams, perturbed(s))


def config_fd_2k() -> Workload:
    """Differentiation check: N=2k, one 128x128 camera."""
    s = random_scene(2_000)
    cams = [look_at_camera((0.0, 0.0, -3.0), 128, 128, 60.0)]
    return Workload("fd_2k_128x128", s, cams, perturbed(s))


def config_clustered_3m() -> Workload:
    """Mixed precision: N=3M clustered Gaussians, one 1920x1080 camera."""
    s = clustered_scene(3_000_000)
    cams = sphere_cameras(1)
    return Workload("clustered_3M_1920x1080", s, cams, perturbed(s))


def config_batched_64(n: int = 1_000_000) -> Workload:
    """Batched training: N=1M (n for smaller profiling cases), 64 cameras of
    mixed resolution and FOV."""
    s = random_scene(n)
    res = [(320, 240), (640, 480), (1280, 720), (1920, 1080), (3840, 2160)]
    cams = sphere_cameras(64, resolutions=res, fov_range=(45.0, 75.0))
    return Workload("batched_64views_1M" if n == 1_000_000 else f"batched_64views_{n}", s, cams, perturbed(s))

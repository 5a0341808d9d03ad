"""TEST INFRASTRUCTURE: Python access to the two CPU oracles of the 3DGS path.

* ``C``   -- oracle/liboracle.so, the C restatement (gs3d_oracle.c);
* ``REF`` -- oracle/_ref/libgs3d_ref.so, the reference's own CPU stages compiled
            from their sources plus ref_shim.cpp (present when it was built in a
            container that had the reference tree).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_C = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libgs3d_ref.so")

_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_u32 = ctypes.POINTER(ctypes.c_uint32)
_d = ctypes.POINTER(ctypes.c_double)


class StepIO(ctypes.Structure):
    """Mirror of ``orc_step_io`` (oracle/gs3d_oracle.h)."""

    _fields_ = [
        ("means2D", _f), ("depths", _f), ("conics", _f), ("opac2d", _f), ("rgb", _f),
        ("radii", _i), ("tiles", _i),
        ("cov3D", _f), ("p_view", _f), ("p_hom_w", _f), ("cov2D", _f), ("det", _f),
        ("pair_capacity", ctypes.c_int64), ("total_pairs", ctypes.c_int64),
        ("keys_unsorted", _u64), ("keys_sorted", _u64),
        ("vals_unsorted", _u32), ("vals_sorted", _u32), ("ranges", _u32),
        ("image", _f), ("T_final", _f), ("n_contrib", _i), ("d_image", _f),
        ("d_means2D", _f), ("d_conics", _f), ("d_rgb", _f), ("d_opac", _f),
        ("g_pos", _f), ("g_sc", _f), ("g_rot", _f), ("g_sh", _f), ("g_op", _f),
        ("loss", ctypes.c_float), ("loss_acc64", ctypes.c_double),
    ]


class AdamState(ctypes.Structure):
    """Mirror of ``orc_adam_state``."""

    _fields_ = [(n, _f) for n in ("m_pos", "v_pos", "m_sc", "v_sc", "m_rot", "v_rot",
                                  "m_sh", "v_sh", "m_op", "v_op")] + [("step_count", ctypes.c_int)]


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


# The reference project's root (harmonyos_3dgs/): only the build recipe of
# oracle/_ref and the fixture generator read it; the tests use the built
# library and the committed fixtures.
REF_ROOT = os.environ.get("GS3D_REFERENCE_ROOT", "/root/reference/harmonyos_3dgs")


def ensure_built(ref: bool = False) -> None:
    """Build liboracle.so (and, if asked and the reference tree exists, _ref)."""
    if not os.path.exists(LIB_C):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and not os.path.exists(LIB_REF) and os.path.isdir(REF_ROOT):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "-j8"], check=True)


_LIBS: dict = {}


def lib_c():
    if "c" not in _LIBS:
        ensure_built()
        L = ctypes.CDLL(LIB_C)
        L.orc_forward.restype = ctypes.c_int
        L.orc_train_step.restype = ctypes.c_int
        L.orc_step_f64.restype = ctypes.c_double
        L.orc_scan_tiles.restype = ctypes.c_int64
        L.orc_l1_loss_f32.restype = ctypes.c_float
        _LIBS["c"] = L
    return _LIBS["c"]


def have_ref() -> bool:
    return os.path.exists(LIB_REF)


def lib_ref():
    if "ref" not in _LIBS:
        if not have_ref():
            raise FileNotFoundError(LIB_REF)
        L = ctypes.CDLL(LIB_REF)
        L.ref_forward.restype = ctypes.c_int
        L.ref_train_step.restype = ctypes.c_int
        L.ref_adam_create.restype = ctypes.c_void_p
        L.ref_adam_destroy.argtypes = [ctypes.c_void_p]
        L.ref_train_step.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int, ctypes.c_void_p]
        L.ref_trainer_create.restype = ctypes.c_void_p
        L.ref_trainer_create.argtypes = [ctypes.c_size_t]
        L.ref_trainer_destroy.argtypes = [ctypes.c_void_p]
        L.ref_trainer_step.restype = ctypes.c_int
        L.ref_trainer_step.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int, ctypes.c_void_p]
        L.ref_renderer_create.restype = ctypes.c_void_p
        L.ref_renderer_create.argtypes = [ctypes.c_size_t]
        L.ref_renderer_destroy.argtypes = [ctypes.c_void_p]
        L.ref_renderer_render.restype = ctypes.c_int
        L.ref_renderer_render.argtypes = [ctypes.c_void_p] * 5
        L.ref_activate.argtypes = [ctypes.c_void_p] * 2
        _LIBS["ref"] = L
    return _LIBS["ref"]


@dataclass
class StepResult:
    """Every intermediate of one forward (and, for a train step, backward)."""

    means2D: np.ndarray
    depths: np.ndarray
    conics: np.ndarray
    opac2d: np.ndarray
    rgb: np.ndarray
    radii: np.ndarray
    tiles: np.ndarray
    cov3D: np.ndarray
    p_view: np.ndarray
    p_hom_w: np.ndarray
    cov2D: np.ndarray
    det: np.ndarray
    total_pairs: int
    keys_unsorted: np.ndarray
    vals_unsorted: np.ndarray
    keys_sorted: np.ndarray
    vals_sorted: np.ndarray
    ranges: np.ndarray
    image: np.ndarray
    T_final: np.ndarray
    n_contrib: np.ndarray
    d_image: np.ndarray | None = None
    d_means2D: np.ndarray | None = None
    d_conics: np.ndarray | None = None
    d_rgb: np.ndarray | None = None
    d_opac: np.ndarray | None = None
    g_pos: np.ndarray | None = None
    g_sc: np.ndarray | None = None
    g_rot: np.ndarray | None = None
    g_sh: np.ndarray | None = None
    g_op: np.ndarray | None = None
    loss: float | None = None
    loss_acc64: float | None = None


def _alloc_io(n: int, mc3: int, npx: int, ntiles: int, cap: int, train: bool):
    z = np.zeros
    a = dict(
        means2D=z(2 * n, np.float32), depths=z(n, np.float32), conics=z(3 * n, np.float32),
        opac2d=z(n, np.float32), rgb=z(3 * n, np.float32), radii=z(n, np.int32),
        tiles=z(n, np.int32), cov3D=z(6 * n, np.float32), p_view=z(3 * n, np.float32),
        p_hom_w=z(n, np.float32), cov2D=z(3 * n, np.float32), det=z(n, np.float32),
        keys_unsorted=z(max(cap, 1), np.uint64), keys_sorted=z(max(cap, 1), np.uint64),
        vals_unsorted=z(max(cap, 1), np.uint32), vals_sorted=z(max(cap, 1), np.uint32),
        ranges=z(2 * ntiles, np.uint32), image=z(3 * npx, np.float32),
        T_final=z(npx, np.float32), n_contrib=z(npx, np.int32),
    )
    if train:
        a.update(d_image=z(3 * npx, np.float32), d_means2D=z(2 * n, np.float32),
                 d_conics=z(3 * n, np.float32), d_rgb=z(3 * n, np.float32), d_opac=z(n, np.float32),
                 g_pos=z(3 * n, np.float32), g_sc=z(3 * n, np.float32), g_rot=z(4 * n, np.float32),
                 g_sh=z(mc3 * n, np.float32), g_op=z(n, np.float32))
    io = StepIO()
    for k, v in a.items():
        t = {np.float32: _f, np.int32: _i, np.uint64: _u64, np.uint32: _u32}[v.dtype.type]
        setattr(io, k, _ptr(v, t))
    io.pair_capacity = cap
    return io, a


def _result(io, a, train: bool) -> StepResult:
    P = int(io.total_pairs)
    kw = {k: v for k, v in a.items()}
    for k in ("keys_unsorted", "keys_sorted", "vals_unsorted", "vals_sorted"):
        kw[k] = kw[k][:P].copy()
    kw["total_pairs"] = P
    if train:
        kw["loss"] = float(io.loss)
        kw["loss_acc64"] = float(io.loss_acc64)
    return StepResult(**kw)


def _grid(cam, cfg):
    gx = (cam.width + cfg.tile_w - 1) // cfg.tile_w
    gy = (cam.height + cfg.tile_h - 1) // cfg.tile_h
    return gx * gy


def activate(scene):
    """Activated model arrays (float32, the reference's activate()) via the C oracle."""
    L = lib_c()
    n, mc3 = scene.count, scene.max_coeffs * 3
    out = [np.empty(3 * n, np.float32), np.empty(3 * n, np.float32), np.empty(4 * n, np.float32),
           np.empty(mc3 * n, np.float32), np.empty(n, np.float32)]
    L.orc_activate_f32(ctypes.c_int(n), ctypes.c_int(mc3),
                       *[_ptr(np.ascontiguousarray(x, np.float32).reshape(-1), _f)
                         for x in (scene.positions, scene.scales, scene.rotations, scene.sh,
                                   scene.opacities)],
                       *[_ptr(x, _f) for x in out])
    return dict(positions=out[0], scales=out[1], rotations=out[2], sh_coeffs=out[3], opacities=out[4])


def activate_ref(scene):
    """The reference's own RawGaussianParams::activate (oracle/_ref)."""
    n, mc3 = scene.count, scene.max_coeffs * 3
    act = dict(positions=np.empty(3 * n, np.float32), scales=np.empty(3 * n, np.float32),
               rotations=np.empty(4 * n, np.float32), sh_coeffs=np.empty(mc3 * n, np.float32),
               opacities=np.empty(n, np.float32))
    g = gaussians_struct(scene, act)
    raw = scene.raw_struct()
    lib_ref().ref_activate(ctypes.addressof(raw), ctypes.addressof(g))
    return act


def gaussians_struct(scene, act: dict):
    from aaags_claude_b200.scenes import GaussianData
    g = GaussianData()
    g.count, g.sh_degree, g.max_coeffs = scene.count, scene.sh_degree, scene.max_coeffs
    for k in ("positions", "sh_coeffs", "scales", "rotations", "opacities"):
        setattr(g, k, _ptr(act[k], _f))
    g.filter_3D = None
    g._keep = act
    return g


def forward(scene, cam, cfg, impl: str = "c", act: dict | None = None, cap: int | None = None) -> StepResult:
    """Plain-FP32 forward (preprocess, bin, sort, rasterise) of an activated scene."""
    act = act if act is not None else activate(scene)
    g = gaussians_struct(scene, act)
    n, mc3 = scene.count, scene.max_coeffs * 3
    npx, nt = cam.width * cam.height, _grid(cam, cfg)
    cap = cap if cap is not None else max(16, 8 * n)
    for _ in range(2):
        io, a = _alloc_io(n, mc3, npx, nt, cap, False)
        if impl == "c":
            rc = lib_c().orc_forward(ctypes.byref(g), ctypes.byref(cam), ctypes.byref(cfg), ctypes.byref(io))
        else:
            rc = lib_ref().ref_forward(ctypes.byref(g), ctypes.byref(cam), ctypes.byref(cfg), ctypes.byref(io))
        if rc == 0:
            return _result(io, a, False)
        cap = int(io.total_pairs)
    raise RuntimeError("oracle forward: pair capacity retry failed")


def forward_eval3d(scene, cam, cfg, impl: str = "c", act: dict | None = None, cap: int | None = None,
                   filter_3d: np.ndarray | None = None):
    """Forward of the 3D-evaluation mode (cfg.eval_3D) of an activated scene.

    Returns (StepResult, extras) with extras = dict(gauss2screen [N,16],
    cov3D_inv [N,6], mean_offset [N,3]); conics and the 2D cache stay zero.
    impl "c" is the C restatement, "ref" the reference's own stages.
    """
    act = act if act is not None else activate(scene)
    g = gaussians_struct(scene, act)
    if filter_3d is not None:
        f3 = np.ascontiguousarray(filter_3d, np.float32)
        g.filter_3D = _ptr(f3, _f)
        g._keep_f3 = f3
    n, mc3 = scene.count, scene.max_coeffs * 3
    npx, nt = cam.width * cam.height, _grid(cam, cfg)
    cap = cap if cap is not None else max(16, 8 * n)
    for _ in range(2):
        io, a = _alloc_io(n, mc3, npx, nt, cap, False)
        io.cov3D = None
        ex = dict(gauss2screen=np.zeros(16 * n, np.float32), cov3D_inv=np.zeros(6 * n, np.float32),
                  mean_offset=np.zeros(3 * n, np.float32))
        args = (ctypes.byref(g), ctypes.byref(cam), ctypes.byref(cfg), ctypes.byref(io),
                *[_ptr(ex[k], _f) for k in ("gauss2screen", "cov3D_inv", "mean_offset")])
        rc = (lib_c().orc_forward_eval3d if impl == "c" else lib_ref().ref_forward_eval3d)(*args)
        if rc == 0:
            ex = {k: v.reshape(n, -1) for k, v in ex.items()}
            return _result(io, a, False), ex
        if rc != 1:
            raise RuntimeError(f"eval_3D forward failed ({rc})")
        cap = int(io.total_pairs)
    raise RuntimeError("oracle forward: pair capacity retry failed")


class DensityOracle:
    """DensityController state (density_controller.cpp) over the C restatement:
    per-Gaussian statistics, the split sampler's LCG state (12345 at start)."""

    def __init__(self):
        self.n = 0
        self.rng = ctypes.c_uint64(12345)
        self.reset(0)

    def reset(self, n: int):
        self.n = n
        self.accum = np.zeros(n, np.float32)
        self.denom = np.zeros(n, np.float32)
        self.max_radii = np.zeros(n, np.int32)

    def accumulate(self, d_means2D: np.ndarray, radii: np.ndarray | None, n: int):
        if n != self.n:
            self.reset(n)
        d = np.ascontiguousarray(d_means2D, np.float32).reshape(-1)
        r = None if radii is None else np.ascontiguousarray(radii, np.int32)
        lib_c().orc_dc_accumulate(ctypes.c_int(n), _ptr(d, _f), None if r is None else _ptr(r, _i),
                                  _ptr(self.accum, _f), _ptr(self.denom, _f), _ptr(self.max_radii, _i))

    def densify(self, scene, cfg, extent: float):
        """densify_and_prune on a Scene of raw parameters; returns the new Scene."""
        from aaags_claude_b200.scenes import Scene
        n, k = scene.count, scene.max_coeffs
        mc3 = 3 * k
        if self.n != n:
            self.reset(n)
        o = [np.zeros((2 * n, 3), np.float32), np.zeros((2 * n, 3), np.float32), np.zeros((2 * n, 4), np.float32),
             np.zeros((2 * n, k, 3), np.float32), np.zeros(2 * n, np.float32)]
        ins = [np.ascontiguousarray(x, np.float32) for x in
               (scene.positions, scene.scales, scene.rotations, scene.sh, scene.opacities)]
        m = lib_c().orc_dc_densify(ctypes.c_int(n), ctypes.c_int(mc3), *[_ptr(x, _f) for x in ins],
                                   _ptr(self.accum, _f), _ptr(self.denom, _f), _ptr(self.max_radii, _i),
                                   ctypes.c_float(cfg.grad_threshold), ctypes.c_float(cfg.min_opacity),
                                   ctypes.c_int(cfg.max_screen_size), ctypes.c_float(extent),
                                   ctypes.byref(self.rng), *[_ptr(x, _f) for x in o])
        self.reset(m)
        return Scene(o[0][:m].copy(), o[1][:m].copy(), o[2][:m].copy(), o[3][:m].copy(), o[4][:m].copy(),
                     scene.sh_degree)

    @staticmethod
    def reset_opacity(scene):
        op = np.ascontiguousarray(scene.opacities, np.float32)
        lib_c().orc_dc_reset_opacity(ctypes.c_int(scene.count), _ptr(op, _f))
        scene.opacities[:] = op


class DensityRef:
    """The reference's own DensityController on an OwnedRawParams (oracle/_ref)."""

    def __init__(self):
        L = lib_ref()
        L.ref_dc_create.restype = ctypes.c_void_p
        L.ref_dc_destroy.argtypes = [ctypes.c_void_p]
        L.ref_dc_set_model.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.ref_dc_accumulate.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.ref_dc_densify.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float]
        L.ref_dc_densify.restype = ctypes.c_int
        L.ref_dc_reset_opacity.argtypes = [ctypes.c_void_p]
        L.ref_dc_get_model.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.ref_dc_get_model.restype = ctypes.c_int
        self.L = L
        self.h = L.ref_dc_create()
        self.count, self.k, self.deg = 0, 1, 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_dc_destroy(self.h)
            self.h = None

    def set_model(self, scene):
        raw = scene.raw_struct()
        self.L.ref_dc_set_model(self.h, ctypes.addressof(raw))
        self.count, self.k, self.deg = scene.count, scene.max_coeffs, scene.sh_degree

    def accumulate(self, d_means2D: np.ndarray, radii: np.ndarray | None, n: int):
        d = np.ascontiguousarray(d_means2D, np.float32).reshape(-1)
        r = None if radii is None else np.ascontiguousarray(radii, np.int32)
        self.L.ref_dc_accumulate(self.h, d.ctypes.data, None if r is None else r.ctypes.data, n)

    def densify(self, cfg, extent: float) -> int:
        self.count = self.L.ref_dc_densify(self.h, ctypes.addressof(cfg), ctypes.c_float(extent))
        return self.count

    def reset_opacity(self):
        self.L.ref_dc_reset_opacity(self.h)

    def model(self):
        from aaags_claude_b200.scenes import Scene
        n, k = self.count, self.k
        sc = Scene(np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
                   np.zeros((n, k, 3), np.float32), np.zeros(n, np.float32), self.deg)
        raw = sc.raw_struct()
        self.L.ref_dc_get_model(self.h, ctypes.addressof(raw))
        return sc


class AdamOracle:
    """Adam moments for the C oracle's train step (zero-initialised)."""

    def __init__(self, n: int, mc3: int):
        self.arrays = {k: np.zeros(s * n, np.float32) for k, s in
                       (("m_pos", 3), ("v_pos", 3), ("m_sc", 3), ("v_sc", 3), ("m_rot", 4),
                        ("v_rot", 4), ("m_sh", mc3), ("v_sh", mc3), ("m_op", 1), ("v_op", 1))}
        self.st = AdamState()
        for k, v in self.arrays.items():
            setattr(self.st, k, _ptr(v, _f))
        self.st.step_count = 0


class RefAdam:
    def __init__(self):
        self.h = lib_ref().ref_adam_create()

    def __del__(self):
        try:
            lib_ref().ref_adam_destroy(self.h)
        except Exception:
            pass


def train_step(scene, cam, gt: np.ndarray, cfg, tcfg, iteration: int, state,
               impl: str = "c", cap: int | None = None) -> StepResult:
    """One Trainer::step (Adam or SGD per tcfg); ``scene`` is updated in place."""
    n, mc3 = scene.count, scene.max_coeffs * 3
    npx, nt = cam.width * cam.height, _grid(cam, cfg)
    raw = scene.raw_struct()
    gt = np.ascontiguousarray(gt, np.float32).reshape(-1)
    cap = cap if cap is not None else max(16, 8 * n)
    for _ in range(2):
        io, a = _alloc_io(n, mc3, npx, nt, cap, True)
        if impl == "c":
            act = [np.empty(s, np.float32) for s in (3 * n, 3 * n, 4 * n, mc3 * n, n)]
            rc = lib_c().orc_train_step(ctypes.byref(raw), ctypes.byref(cam), _ptr(gt, _f), ctypes.byref(cfg),
                                        ctypes.byref(tcfg), ctypes.c_int(iteration), ctypes.byref(state.st),
                                        *[_ptr(x, _f) for x in act], ctypes.byref(io))
        else:
            rc = lib_ref().ref_train_step(state.h, ctypes.addressof(raw), ctypes.addressof(cam),
                                          gt.ctypes.data, ctypes.addressof(cfg), ctypes.addressof(tcfg),
                                          iteration, ctypes.addressof(io))
        if rc == 0:
            return _result(io, a, True)
        cap = int(io.total_pairs)
    raise RuntimeError("oracle train step: pair capacity retry failed")


def step_f64(scene, cam, cfg, gt: np.ndarray | None, want_grads: bool = True, params64=None):
    """FP64 evaluation: (loss, image[H,W,3], grads dict or None).

    ``params64`` optionally overrides the raw parameters with float64 arrays
    (pos, scales, rotations, sh, opacities), as the finite-difference driver does.
    """
    L = lib_c()
    n, mc3 = scene.count, scene.max_coeffs * 3
    if params64 is None:
        params64 = [np.ascontiguousarray(x, np.float64).reshape(-1) for x in
                    (scene.positions, scene.scales, scene.rotations, scene.sh, scene.opacities)]
    img = np.zeros(cam.width * cam.height * 3, np.float64)
    grads = None
    gptr = [None] * 5
    if want_grads:
        grads = dict(pos=np.zeros(3 * n), sc=np.zeros(3 * n), rot=np.zeros(4 * n),
                     sh=np.zeros(mc3 * n), op=np.zeros(n))
        gptr = [_ptr(grads[k], _d) for k in ("pos", "sc", "rot", "sh", "op")]
    gtp = _ptr(np.ascontiguousarray(gt, np.float32).reshape(-1), _f) if gt is not None else None
    loss = L.orc_step_f64(ctypes.c_int(n), ctypes.c_int(scene.sh_degree), ctypes.c_int(scene.max_coeffs),
                          *[_ptr(p, _d) for p in params64], ctypes.byref(cam), ctypes.byref(cfg), gtp,
                          _ptr(img, _d), *gptr)
    return float(loss), img.reshape(cam.height, cam.width, 3), grads

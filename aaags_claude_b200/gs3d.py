"""Python binding of the gs3dc_* C ABI (include/gs3d_cuda.h) over ctypes.

The product path is libgs3d_cuda.so (CUDA, sm_100a).  Nothing here computes on
the CPU: if the library or a B200-class device is missing, ``Context`` raises.

    ctx = Context(0)
    ctx.set_raw_params(scene)                 # RawGaussianParams -> device
    loss = ctx.train_step(cam, gt, cfg, tcfg, iteration)   # Trainer::step
    img = ctx.render(cam, cfg, gaussians=...) # Renderer::render
"""
from __future__ import annotations

import ctypes
import struct
import os

import numpy as np

from . import scenes as S

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgs3d_cuda.so")

OK = 0
ERR_INVALID_ARG, ERR_CUDA, ERR_PAIR_OVERFLOW, ERR_DEVICE_TIMEOUT, ERR_NO_MODEL, ERR_OOM, ERR_STATE = range(1, 8)
OPT_PAIR_CAPACITY, OPT_USE_GRAPH, OPT_FORM, OPT_SPIN_LIMIT, OPT_STAGE_TIMING, OPT_FUSED_ADAM = 1, 2, 3, 4, 5, 6
NUM_STAGES = 8
STAT_TOTAL_PAIRS, STAT_PAIR_CAPACITY, STAT_KERNELS_LAST, STAT_SORT_PASSES, STAT_GRAPH_REPLAYS, STAT_ADAM_STEP = range(1, 7)
STAT_NUM_GAUSSIANS = 9
STAT_SCREEN_GAUSSIANS = 10
STAT_GRAPH_CAPTURES = 11
STAT_FWD_BATCH, STAT_BWD_BATCH = 12, 13
STAT_FWD_PPT, STAT_BWD_PPT = 7, 8
FORM_PLAIN_FP32, FORM_BF16, FORM_FP16 = 0, 1, 2
OPT_SORT = 7
OPT_KEEP_GRADIENTS = 8
OPT_AUTOTUNE = 9
OPT_DENSITY_SEED = 10
OPT_RASTER_PPT = 11
OPT_RASTER_BATCH = 12
SORT_DEPTH_FIRST, SORT_FULL_KEY = 0, 1

_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int)


class ScreenArrays(ctypes.Structure):
    """Layout of ``gs3dc_screen_arrays``."""

    _fields_ = [(n, _f) for n in ("means2D", "depths", "conics", "opacities_2d", "rgb")] + \
               [("radii", _i), ("tiles_touched", _i)] + \
               [(n, _f) for n in ("cov3D", "p_view", "p_hom_w", "cov2D", "cov2D_det",
                                  "gauss2screen", "cov3D_inv", "mean_offset")]


class Gs3dError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gs3dc status {status}: {message}")
        self.status = status


_LIB = None


def load_library(path: str = LIB_PATH):
    """Loads libgs3d_cuda.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: run `python -m aaags_claude_b200.build`")
    L = ctypes.CDLL(path)
    vp, i64 = ctypes.c_void_p, ctypes.c_int64
    sig = {
        "gs3dc_create": ([ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "gs3dc_destroy": ([vp], None),
        "gs3dc_last_error": ([vp], ctypes.c_char_p),
        "gs3dc_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "gs3dc_get_stream": ([vp, ctypes.POINTER(vp)], ctypes.c_int),
        "gs3dc_set_option": ([vp, ctypes.c_int, i64], ctypes.c_int),
        "gs3dc_get_stat": ([vp, ctypes.c_int, ctypes.POINTER(i64)], ctypes.c_int),
        "gs3dc_set_gaussians": ([vp, vp], ctypes.c_int),
        "gs3dc_set_raw_params": ([vp, vp], ctypes.c_int),
        "gs3dc_get_raw_params": ([vp, vp], ctypes.c_int),
        "gs3dc_preprocess": ([vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_bin": ([vp, ctypes.c_int, vp, vp, vp, ctypes.POINTER(i64), vp, vp], ctypes.c_int),
        "gs3dc_sort": ([vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_sort_pairs": ([vp, i64, vp, vp, ctypes.c_int, vp, vp, vp], ctypes.c_int),
        "gs3dc_rasterize": ([vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_render": ([vp, vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_raster_backward": ([vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_preprocess_backward": ([vp, vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_update_raw_params": ([vp, vp], ctypes.c_int),
        "gs3dc_get_image": ([vp, vp], ctypes.c_int),
        "gs3dc_raster_backward_lists": ([vp, vp, vp, vp, vp, vp, vp, vp, ctypes.POINTER(i64)], ctypes.c_int),
        "gs3dc_get_batch_image": ([vp, ctypes.c_int, vp], ctypes.c_int),
        "gs3dc_optimizer_step": ([vp, vp, ctypes.c_int], ctypes.c_int),
        "gs3dc_train_step": ([vp, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int, vp], ctypes.c_int),
        "gs3dc_synchronize": ([vp], ctypes.c_int),
        "gs3dc_get_stage_times": ([vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int], ctypes.c_int),
        "gs3dc_selftest_bounded_wait": ([vp, ctypes.c_uint32], ctypes.c_int),
        "gs3dc_get_gradients": ([vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_save_state": ([vp, ctypes.c_char_p], ctypes.c_int),
        "gs3dc_density_accumulate": ([vp, vp, vp], ctypes.c_int),
        "gs3dc_rasterize_arrays": ([vp, ctypes.c_int, vp, i64, vp, ctypes.c_int, vp, vp, vp, vp, vp, vp],
                                   ctypes.c_int),
        "gs3dc_ply_info": ([ctypes.c_char_p, vp, vp, vp, vp], ctypes.c_int),
        "gs3dc_ply_read": ([ctypes.c_char_p, ctypes.c_int, vp], ctypes.c_int),
        "gs3dc_ply_write": ([ctypes.c_char_p, vp], ctypes.c_int),
        "gs3dc_raw_from_gaussians": ([vp, vp], ctypes.c_int),
        "gs3dc_cameras_read": ([ctypes.c_char_p, vp, vp, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
        "gs3dc_ppm_read": ([ctypes.c_char_p, vp, vp, vp], ctypes.c_int),
        "gs3dc_ppm_write": ([ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "gs3dc_image_resize_nearest": ([vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int],
                                       ctypes.c_int),
        "gs3dc_io_last_error": ([], ctypes.c_char_p),
        "gs3dc_densify_and_prune": ([vp, vp, ctypes.c_float, vp], ctypes.c_int),
        "gs3dc_reset_opacity": ([vp], ctypes.c_int),
        "gs3dc_train_step_densify": ([vp, vp, vp, ctypes.c_int, vp, vp, vp, ctypes.c_float, ctypes.c_int, vp, vp],
                                     ctypes.c_int),
        "gs3dc_load_state": ([vp, ctypes.c_char_p], ctypes.c_int),
        "gs3dc_train_step_batch": ([vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int, vp],
                                   ctypes.c_int),
        "gs3dc_sort_pairs_static": ([i64, vp, vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_char_p, ctypes.c_size_t],
                                    ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def exported_symbols() -> list[str]:
    """The gs3dc_* names include/gs3d_cuda.h declares."""
    import re
    hdr = os.path.join(os.path.dirname(PKG), "include", "gs3d_cuda.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"\b(gs3dc_[a-z_0-9]+)\s*\(", txt)))


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _ref(s):
    return None if s is None else ctypes.cast(ctypes.pointer(s), ctypes.c_void_p)


# ---- on-disk formats (host functions: no context, no GPU needed) ----

def _io(rc: int):
    if rc != 0:
        raise Gs3dError(rc, load_library().gs3dc_io_last_error().decode(errors="replace"))


def ply_info(path: str) -> dict:
    """count, sh_degree, max_coeffs, has_filter_3D of a 3DGS PLY."""
    L = load_library()
    v = [ctypes.c_int() for _ in range(4)]
    _io(L.gs3dc_ply_info(str(path).encode(), *[ctypes.byref(x) for x in v]))
    return dict(count=v[0].value, sh_degree=v[1].value, max_coeffs=v[2].value, has_filter_3D=bool(v[3].value))


def load_ply(path: str, activate: bool = True):
    """loadPly: (Scene of the arrays, filter_3D or None).  activate: the loader's
    activations (the arrays are a GaussianData model: opacities, scales,
    normalised rotations); otherwise the stored raw values (a trainable Scene)."""
    L = load_library()
    info = ply_info(path)
    n, k = info["count"], info["max_coeffs"]
    sc = S.Scene(np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
                 np.zeros((n, k, 3), np.float32), np.zeros(n, np.float32), info["sh_degree"])
    g = S.GaussianData()
    g.count, g.sh_degree, g.max_coeffs = n, info["sh_degree"], k
    for fld, arr in (("positions", sc.positions), ("scales", sc.scales), ("rotations", sc.rotations),
                     ("sh_coeffs", sc.sh), ("opacities", sc.opacities)):
        setattr(g, fld, S.fptr(arr))
    f3 = np.zeros(n, np.float32) if info["has_filter_3D"] else None
    if f3 is not None:
        g.filter_3D = S.fptr(f3)
    _io(L.gs3dc_ply_read(str(path).encode(), 1 if activate else 0, _ref(g)))
    return sc, f3


def save_ply(path: str, scene: S.Scene):
    """savePly of the train driver (raw parameters)."""
    r = scene.raw_struct()
    _io(load_library().gs3dc_ply_write(str(path).encode(), _ref(r)))


def raw_from_gaussians(model: S.Scene) -> S.Scene:
    """initRawFromGaussianData: a loaded (activated) model -> trainable raw parameters."""
    n, k = model.count, model.max_coeffs
    g = S.GaussianData()
    g.count, g.sh_degree, g.max_coeffs = n, model.sh_degree, k
    arrs = [np.ascontiguousarray(x, np.float32) for x in
            (model.positions, model.scales, model.rotations, model.sh, model.opacities)]
    for fld, arr in zip(("positions", "scales", "rotations", "sh_coeffs", "opacities"), arrs):
        setattr(g, fld, S.fptr(arr))
    out = S.Scene(np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
                  np.zeros((n, k, 3), np.float32), np.zeros(n, np.float32), model.sh_degree)
    r = out.raw_struct()
    _io(load_library().gs3dc_raw_from_gaussians(_ref(g), _ref(r)))
    return out


def load_cameras(path: str, name_len: int = 256) -> list:
    """loadCamerasJson: [(Camera, img_name)] in file order."""
    L = load_library()
    n = ctypes.c_int()
    _io(L.gs3dc_cameras_read(str(path).encode(), None, None, 0, 0, ctypes.byref(n)))
    cams = (S.Camera * max(n.value, 1))()
    names = ctypes.create_string_buffer(max(n.value, 1) * name_len)
    _io(L.gs3dc_cameras_read(str(path).encode(), ctypes.cast(cams, ctypes.c_void_p), ctypes.cast(names, ctypes.c_void_p),
                             name_len, n.value, ctypes.byref(n)))
    out = []
    for i in range(n.value):
        raw = names.raw[i * name_len:(i + 1) * name_len]
        out.append((S.Camera.from_buffer_copy(cams[i]), raw.split(b"\0")[0].decode(errors="replace")))
    return out


def read_ppm(path: str):
    """readPPM: (float32 image [H*W*3] in [0, 1], width, height)."""
    L = load_library()
    w, h = ctypes.c_int(), ctypes.c_int()
    _io(L.gs3dc_ppm_read(str(path).encode(), None, ctypes.byref(w), ctypes.byref(h)))
    img = np.zeros(w.value * h.value * 3, np.float32)
    _io(L.gs3dc_ppm_read(str(path).encode(), _p(img), ctypes.byref(w), ctypes.byref(h)))
    return img, w.value, h.value


def write_ppm(path: str, image: np.ndarray, width: int, height: int):
    img = np.ascontiguousarray(image, np.float32).reshape(-1)
    _io(load_library().gs3dc_ppm_write(str(path).encode(), _p(img), int(width), int(height)))


def resize_nearest(image: np.ndarray, sw: int, sh: int, dw: int, dh: int) -> np.ndarray:
    src = np.ascontiguousarray(image, np.float32).reshape(-1)
    dst = np.zeros(dw * dh * 3, np.float32)
    _io(load_library().gs3dc_image_resize_nearest(_p(src), sw, sh, _p(dst), dw, dh))
    return dst


def load_views(cameras_json: str, gt_dir: str) -> list:
    """The train driver's multi-view data (train_main.cpp:515-563): every camera of
    cameras.json whose <gt_dir>/<img_name>{.ppm,.PPM,} loads, with its target
    resized (nearest) to the camera when the sizes differ.  [(Camera, target)]."""
    views = []
    for cam, name in load_cameras(cameras_json):
        if not name:
            continue
        for ext in (".ppm", ".PPM", ""):
            path = os.path.join(gt_dir, name + ext)
            if not os.path.exists(path):
                continue
            try:
                img, w, h = read_ppm(path)
            except Gs3dError:
                continue
            if (w, h) != (cam.width, cam.height):
                img = resize_nearest(img, w, h, cam.width, cam.height)
            views.append((cam, img))
            break
    return views


class Context:
    """One gs3dc context: a CUDA stream and the device buffers of the path."""

    def __init__(self, device: int = 0):
        self.L = load_library()
        h = ctypes.c_void_p()
        rc = self.L.gs3dc_create(device, ctypes.byref(h))
        if rc != OK:
            raise Gs3dError(rc, f"gs3dc_create(device={device}) failed: "
                                f"{self.L.gs3dc_status_string(rc).decode()} (needs an sm_100 GPU)")
        self.h = h
        self._model = None

    def close(self):
        if getattr(self, "h", None):
            self.L.gs3dc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc: int):
        if rc != OK:
            raise Gs3dError(rc, self.L.gs3dc_last_error(self.h).decode())

    # ---- context ----
    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._chk(self.L.gs3dc_get_stream(self.h, ctypes.byref(s)))
        return int(s.value or 0)

    def set_option(self, opt: int, value: int):
        self._chk(self.L.gs3dc_set_option(self.h, opt, int(value)))

    def stat(self, which: int) -> int:
        v = ctypes.c_int64()
        self._chk(self.L.gs3dc_get_stat(self.h, which, ctypes.byref(v)))
        return int(v.value)

    def synchronize(self):
        self._chk(self.L.gs3dc_synchronize(self.h))

    def selftest_bounded_wait(self, spin_limit: int) -> int:
        """Status of a device wait on a flag nothing sets (expected: ERR_DEVICE_TIMEOUT)."""
        return int(self.L.gs3dc_selftest_bounded_wait(self.h, int(spin_limit)))

    def stage_times(self) -> list[float]:
        """Per-stage device ms of the last train step run with OPT_STAGE_TIMING."""
        a = (ctypes.c_float * NUM_STAGES)()
        self._chk(self.L.gs3dc_get_stage_times(self.h, a, NUM_STAGES))
        return list(a)

    # ---- model ----
    def set_gaussians(self, scene: S.Scene, act: dict, filter_3d: np.ndarray | None = None):
        """Uploads an activated model (act: positions/scales/rotations/sh_coeffs/opacities);
        filter_3d: GaussianData::filter_3D of the eval_3D mode, or None."""
        g = S.GaussianData()
        g.count, g.sh_degree, g.max_coeffs = scene.count, scene.sh_degree, scene.max_coeffs
        arrs = {k: np.ascontiguousarray(act[k], np.float32) for k in
                ("positions", "sh_coeffs", "scales", "rotations", "opacities")}
        for k, v in arrs.items():
            setattr(g, k, S.fptr(v))
        f3 = None
        if filter_3d is not None:
            f3 = np.ascontiguousarray(filter_3d, np.float32)
            g.filter_3D = S.fptr(f3)
        self._keep = (arrs, f3, g)
        self._chk(self.L.gs3dc_set_gaussians(self.h, _ref(g)))
        self._model = ("act", scene.count, scene.max_coeffs)

    def set_raw_params(self, scene: S.Scene):
        r = scene.raw_struct()
        self._chk(self.L.gs3dc_set_raw_params(self.h, _ref(r)))
        self._model = ("raw", scene.count, scene.max_coeffs)

    def get_raw_params(self, scene: S.Scene):
        """Copies the device parameters into scene's arrays (in place)."""
        r = scene.raw_struct()
        self._chk(self.L.gs3dc_get_raw_params(self.h, _ref(r)))
        return scene

    # ---- stages ----
    def preprocess(self, cam, cfg, want_cache: bool = False) -> dict:
        """Preprocessor::process; with cfg.eval_3D also gauss2screen / cov3D_inv / mean_offset."""
        n = self._model[1]
        out = dict(means2D=np.zeros(2 * n, np.float32), depths=np.zeros(n, np.float32),
                   conics=np.zeros(3 * n, np.float32), opacities_2d=np.zeros(n, np.float32),
                   rgb=np.zeros(3 * n, np.float32), radii=np.zeros(n, np.int32),
                   tiles_touched=np.zeros(n, np.int32))
        if cfg.eval_3D:
            out.update(gauss2screen=np.zeros(16 * n, np.float32), cov3D_inv=np.zeros(6 * n, np.float32),
                       mean_offset=np.zeros(3 * n, np.float32))
        if want_cache:
            out.update(cov3D=np.zeros(6 * n, np.float32), p_view=np.zeros(3 * n, np.float32),
                       p_hom_w=np.zeros(n, np.float32), cov2D=np.zeros(3 * n, np.float32),
                       cov2D_det=np.zeros(n, np.float32))
        sa = ScreenArrays()
        for k, v in out.items():
            setattr(sa, k, v.ctypes.data_as(_i if v.dtype == np.int32 else _f))
        self._chk(self.L.gs3dc_preprocess(self.h, _ref(cam), _ref(cfg), _ref(sa)))
        return out

    def bin(self, cam, cfg, arrays: dict | None = None):
        """TileBinner::bin: (total_pairs, keys_unsorted, values_unsorted).

        Without ``arrays`` the pairs of the last preprocess are returned; with
        host arrays (means2D, depths, radii, tiles_touched) those are binned.
        """
        P = ctypes.c_int64()
        if arrays is not None:
            sa = ScreenArrays()
            keep = {}
            names = ("means2D", "depths", "radii", "tiles_touched") + (
                ("cov3D_inv", "mean_offset") if cfg.eval_3D else ())
            for k in names:
                v = np.ascontiguousarray(arrays[k], np.int32 if k in ("radii", "tiles_touched") else np.float32)
                v = v.reshape(-1)
                keep[k] = v
                setattr(sa, k, v.ctypes.data_as(_i if v.dtype == np.int32 else _f))
            n = int(keep["radii"].shape[0])
            total = int(keep["tiles_touched"].astype(np.int64).sum())
            keys = np.zeros(max(total, 1), np.uint64)
            vals = np.zeros(max(total, 1), np.uint32)
            self._chk(self.L.gs3dc_bin(self.h, n, _ref(sa), _ref(cam), _ref(cfg), ctypes.byref(P), _p(keys), _p(vals)))
            return int(P.value), keys[:P.value], vals[:P.value]
        n = self._model[1]
        self._chk(self.L.gs3dc_bin(self.h, n, None, _ref(cam), _ref(cfg), ctypes.byref(P), None, None))
        keys = np.zeros(max(P.value, 1), np.uint64)
        vals = np.zeros(max(P.value, 1), np.uint32)
        self._chk(self.L.gs3dc_bin(self.h, n, None, _ref(cam), _ref(cfg), ctypes.byref(P), _p(keys), _p(vals)))
        return int(P.value), keys[:P.value], vals[:P.value]

    def sort(self, total_pairs: int, num_tiles: int):
        keys = np.zeros(max(total_pairs, 1), np.uint64)
        vals = np.zeros(max(total_pairs, 1), np.uint32)
        ranges = np.zeros(2 * num_tiles, np.uint32)
        self._chk(self.L.gs3dc_sort(self.h, _p(keys), _p(vals), _p(ranges)))
        return keys[:total_pairs], vals[:total_pairs], ranges

    def sort_pairs(self, keys: np.ndarray, vals: np.ndarray, num_tiles: int):
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = np.ascontiguousarray(vals, np.uint32)
        P = int(keys.shape[0])
        ko = np.zeros(max(P, 1), np.uint64)
        vo = np.zeros(max(P, 1), np.uint32)
        ranges = np.zeros(2 * num_tiles, np.uint32)
        self._chk(self.L.gs3dc_sort_pairs(self.h, P, _p(keys) if P else None, _p(vals) if P else None,
                                          int(num_tiles), _p(ko), _p(vo), _p(ranges)))
        return ko[:P], vo[:P], ranges

    def rasterize(self, cam, cfg):
        npx = cam.width * cam.height
        img = np.zeros(3 * npx, np.float32)
        T = np.zeros(npx, np.float32)
        nc = np.zeros(npx, np.int32)
        self._chk(self.L.gs3dc_rasterize(self.h, _ref(cam), _ref(cfg), _p(img), _p(T), _p(nc)))
        return img, T, nc

    def rasterize_arrays(self, cam, cfg, means2D, conics, opacities_2d, rgb, values_sorted, tile_ranges):
        """Rasterizer::rasterize on host PreprocessOutput / BinningOutput arrays: (image, T_final, n_contrib)."""
        arrs = [np.ascontiguousarray(x, np.float32).reshape(-1) for x in (means2D, conics, opacities_2d, rgb)]
        n = int(arrs[2].shape[0])
        sa = ScreenArrays()
        for k, v in zip(("means2D", "conics", "opacities_2d", "rgb"), arrs):
            setattr(sa, k, v.ctypes.data_as(_f))
        vals = np.ascontiguousarray(values_sorted, np.uint32).reshape(-1)
        rg = np.ascontiguousarray(tile_ranges, np.uint32).reshape(-1)
        npx = cam.width * cam.height
        img, T, nc = np.zeros(3 * npx, np.float32), np.zeros(npx, np.float32), np.zeros(npx, np.int32)
        self._chk(self.L.gs3dc_rasterize_arrays(self.h, n, _ref(sa), int(vals.shape[0]), _p(vals) if vals.size else None,
                                                int(rg.shape[0] // 2), _p(rg), _ref(cam), _ref(cfg), _p(img), _p(T),
                                                _p(nc)))
        return img, T, nc

    def render(self, cam, cfg, download: bool = True) -> np.ndarray | None:
        """Renderer::render of the device model; download=False leaves the image on the device."""
        img = np.zeros(3 * cam.width * cam.height, np.float32) if download else None
        self._chk(self.L.gs3dc_render(self.h, None, _ref(cam), _ref(cfg), _p(img) if download else None))
        return img

    def raster_backward(self, cam, cfg, d_image: np.ndarray) -> dict:
        n = self.stat(STAT_SCREEN_GAUSSIANS)   # the screen records' Gaussians (model or imported arrays)
        out = dict(d_means2D=np.zeros(2 * n, np.float32), d_conics=np.zeros(3 * n, np.float32),
                   d_rgb=np.zeros(3 * n, np.float32), d_opac=np.zeros(n, np.float32))
        d = np.ascontiguousarray(d_image, np.float32).reshape(-1)
        self._chk(self.L.gs3dc_raster_backward(self.h, _ref(cam), _ref(cfg), _p(d), _p(out["d_means2D"]),
                                               _p(out["d_conics"]), _p(out["d_rgb"]), _p(out["d_opac"])))
        return out

    def raster_backward_lists(self, cam, cfg, d_image: np.ndarray) -> tuple[dict, int]:
        """raster_backward with stored per-pixel contributor lists; returns (gradients, list bytes)."""
        n = self.stat(STAT_SCREEN_GAUSSIANS)
        out = dict(d_means2D=np.zeros(2 * n, np.float32), d_conics=np.zeros(3 * n, np.float32),
                   d_rgb=np.zeros(3 * n, np.float32), d_opac=np.zeros(n, np.float32))
        d = np.ascontiguousarray(d_image, np.float32).reshape(-1)
        nb = ctypes.c_int64()
        self._chk(self.L.gs3dc_raster_backward_lists(self.h, _ref(cam), _ref(cfg), _p(d), _p(out["d_means2D"]),
                                                     _p(out["d_conics"]), _p(out["d_rgb"]), _p(out["d_opac"]),
                                                     ctypes.byref(nb)))
        return out, int(nb.value)

    def preprocess_backward(self, cam, cfg, raw_rotations: np.ndarray | None = None) -> dict:
        """PreprocessorBackward; raw_rotations is needed when the device model is activated."""
        n, mc = self._model[1], self._model[2]
        out = dict(g_pos=np.zeros(3 * n, np.float32), g_sc=np.zeros(3 * n, np.float32),
                   g_rot=np.zeros(4 * n, np.float32), g_sh=np.zeros(3 * mc * n, np.float32),
                   g_op=np.zeros(n, np.float32))
        rr = None if raw_rotations is None else np.ascontiguousarray(raw_rotations, np.float32).reshape(-1)
        self._chk(self.L.gs3dc_preprocess_backward(self.h, _ref(cam), _ref(cfg), _p(rr), *[_p(out[k]) for k in
                                                   ("g_pos", "g_sc", "g_rot", "g_sh", "g_op")]))
        return out

    def update_raw_params(self, scene: S.Scene):
        r = scene.raw_struct()
        self._chk(self.L.gs3dc_update_raw_params(self.h, _ref(r)))

    def train_step_batch(self, cams, gt, cfg, tcfg, iteration: int, want_loss: bool = True,
                         gt_device_ptr: int | None = None) -> float | None:
        """One step over several views (reduced-storage form); gt = targets concatenated view-major."""
        arr = (S.Camera * len(cams))(*cams)
        loss = ctypes.c_float()
        if gt_device_ptr is not None:
            gp, on_dev = ctypes.c_void_p(gt_device_ptr), 1
        else:
            gt = np.ascontiguousarray(gt, np.float32)
            gp, on_dev = _p(gt), 0
        self._chk(self.L.gs3dc_train_step_batch(self.h, len(cams), ctypes.byref(arr), gp, on_dev, _ref(cfg), _ref(tcfg),
                                                int(iteration), ctypes.byref(loss) if want_loss else None))
        return float(loss.value) if want_loss else None

    # ---- adaptive density control ----
    def density_accumulate(self, d_means2D: np.ndarray | None = None, radii: np.ndarray | None = None):
        """DensityController::accumulate_stats (host arrays, or None: the device's last raster backward)."""
        d = None if d_means2D is None else np.ascontiguousarray(d_means2D, np.float32).reshape(-1)
        r = None if radii is None else np.ascontiguousarray(radii, np.int32).reshape(-1)
        self._chk(self.L.gs3dc_density_accumulate(self.h, _p(d), _p(r)))

    def densify_and_prune(self, dcfg, scene_extent: float) -> int:
        """DensityController::densify_and_prune on the device model; returns the new count."""
        n = ctypes.c_int()
        self._chk(self.L.gs3dc_densify_and_prune(self.h, _ref(dcfg), ctypes.c_float(scene_extent), ctypes.byref(n)))
        self._model = ("raw", n.value, self._model[2])
        return n.value

    def reset_opacity(self):
        self._chk(self.L.gs3dc_reset_opacity(self.h))

    def train_step_densify(self, cam, gt, cfg, tcfg, dcfg, scene_extent: float, iteration: int,
                           gt_device_ptr: int | None = None):
        """Trainer::step_with_densify: (loss, Gaussian count afterwards)."""
        loss, n = ctypes.c_float(), ctypes.c_int()
        if gt_device_ptr is not None:
            gptr, on_dev = ctypes.c_void_p(int(gt_device_ptr)), 1
        else:
            gt = np.ascontiguousarray(gt, np.float32)
            gptr, on_dev = _p(gt), 0
        self._chk(self.L.gs3dc_train_step_densify(self.h, _ref(cam), gptr, on_dev, _ref(cfg), _ref(tcfg), _ref(dcfg),
                                                  ctypes.c_float(scene_extent), int(iteration), ctypes.byref(loss),
                                                  ctypes.byref(n)))
        self._model = ("raw", n.value, self._model[2])
        return float(loss.value), n.value

    def get_model(self, sh_degree: int = 3) -> S.Scene:
        """The device's raw model as a new Scene (its current count)."""
        n, k = self._model[1], self._model[2]
        sc = S.Scene(np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
                     np.zeros((n, k, 3), np.float32), np.zeros(n, np.float32), sh_degree)
        return self.get_raw_params(sc)

    def save_state(self, path: str):
        """Model, optimiser moments and step counter to a file (gs3dc_save_state)."""
        self._chk(self.L.gs3dc_save_state(self.h, str(path).encode()))

    def load_state(self, path: str):
        """Restores a saved training state; the context takes the saved form and shape."""
        self._chk(self.L.gs3dc_load_state(self.h, str(path).encode()))
        with open(path, "rb") as f:
            _, _, _, count, _, max_coeffs, _ = struct.unpack("<8sIiiiii", f.read(32))
        self._model = ("raw", count, max_coeffs)

    def get_gradients(self) -> dict:
        """Raw-parameter gradients of the last train step (GS3DC_OPT_KEEP_GRADIENTS)."""
        n, mc3 = self._model[1], self._model[2] * 3
        g = dict(pos=np.zeros(3 * n, np.float32), sc=np.zeros(3 * n, np.float32), rot=np.zeros(4 * n, np.float32),
                 sh=np.zeros(mc3 * n, np.float32), op=np.zeros(n, np.float32))
        self._chk(self.L.gs3dc_get_gradients(self.h, *[_p(g[k]) for k in ("pos", "sc", "rot", "sh", "op")]))
        return g

    def get_image(self, cam) -> np.ndarray:
        img = np.zeros(3 * cam.width * cam.height, np.float32)
        self._chk(self.L.gs3dc_get_image(self.h, _p(img)))
        return img

    def get_batch_image(self, view: int, cam) -> np.ndarray:
        """View `view`'s image (H*W*3) of the last multi-view step; cam = that view's camera."""
        img = np.zeros(3 * cam.width * cam.height, np.float32)
        self._chk(self.L.gs3dc_get_batch_image(self.h, int(view), _p(img)))
        return img

    def optimizer_step(self, tcfg, iteration: int):
        self._chk(self.L.gs3dc_optimizer_step(self.h, _ref(tcfg), int(iteration)))

    def train_step(self, cam, gt, cfg, tcfg, iteration: int, want_loss: bool = True,
                   gt_device_ptr: int | None = None) -> float | None:
        """Trainer::step on the device-resident parameters.

        gt is a host float32 array (H*W*3) or, with gt_device_ptr, ignored in
        favour of that device address.
        """
        loss = ctypes.c_float()
        if gt_device_ptr is not None:
            gptr, on_dev = ctypes.c_void_p(int(gt_device_ptr)), 1
        else:
            gt = np.ascontiguousarray(gt, np.float32)
            gptr, on_dev = _p(gt), 0
        self._chk(self.L.gs3dc_train_step(self.h, _ref(cam), gptr, on_dev, _ref(cfg), _ref(tcfg), int(iteration),
                                          ctypes.byref(loss) if want_loss else None))
        return float(loss.value) if want_loss else None

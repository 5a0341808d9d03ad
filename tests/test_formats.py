"""The drivers' file formats through the C ABI (host functions, no GPU).

Against the reference's own loaders run on the reference's data files
(tests/golden/seeded/formats_ref.npz, made by tests/golden/make_golden.py):
cameras.json -> cameras (every matrix bit-exact, names), the PLY of the
reference's loader test -> activated model and raw parameters (bit-exact),
savePly (byte-identical file), writePPM / readPPM (byte-identical, bit-exact);
plus the known answers of the reference's tests/test_ply_loader.cpp, round
trips, the nearest resize and the refusals of malformed files.
"""
import os

import numpy as np
import pytest

import gsutil as U
from aaags_claude_b200 import gs3d
from aaags_claude_b200 import scenes as S

FX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_fixtures", "formats")
REF = np.load(os.path.join(U.SEEDED, "formats_ref.npz"))


def test_cameras_match_reference_loader():
    cams = gs3d.load_cameras(os.path.join(FX, "cameras.json"))
    assert len(cams) == int(REF["cam_count"]) == 76
    got = b"".join(bytes(c) for c, _ in cams)
    assert got == REF["cam_bytes"].tobytes()
    assert [n for _, n in cams] == list(REF["cam_names"])
    c0 = cams[0][0]
    assert (c0.width, c0.height) == (720, 960)


def test_ply_load_matches_reference_loader():
    sc, f3 = gs3d.load_ply(os.path.join(FX, "tiny_3gaussians.ply"))
    n, deg, k, hf = REF["ply_shape"]
    assert (sc.count, sc.sh_degree, sc.max_coeffs, f3 is not None) == (n, deg, k, bool(hf))
    assert U.bits_equal(sc.positions.reshape(-1), REF["ply_positions"])
    assert U.bits_equal(sc.scales.reshape(-1), REF["ply_scales"])
    assert U.bits_equal(sc.rotations.reshape(-1), REF["ply_rotations"])
    assert U.bits_equal(sc.sh.reshape(-1), REF["ply_sh_coeffs"])
    assert U.bits_equal(sc.opacities, REF["ply_opacities"])


def test_ply_known_answers():
    """tests/test_ply_loader.cpp of the reference, restated."""
    sc, _ = gs3d.load_ply(os.path.join(FX, "tiny_3gaussians.ply"))
    assert (sc.count, sc.sh_degree, sc.max_coeffs) == (3, 3, 16)
    assert np.allclose(sc.positions[0], [0.0, 0.0, 5.0], atol=1e-5) and abs(sc.positions[1, 0] - 1.0) < 1e-5
    assert np.allclose(sc.opacities, [0.5, 1 / (1 + np.exp(-2.0)), 1 / (1 + np.exp(2.0))], atol=1e-4)
    assert np.allclose(sc.scales[0], 1.0, atol=1e-5) and abs(sc.scales[1, 0] - np.e) < 1e-4
    assert np.allclose(sc.rotations[0], [1, 0, 0, 0], atol=1e-5)
    assert np.allclose(sc.rotations[2], [2 ** -0.5, 2 ** -0.5, 0, 0], atol=1e-4)
    assert sc.sh[0, 0, 0] != 0.0


def test_raw_from_gaussians_and_save_match_reference(tmp_path):
    model, _ = gs3d.load_ply(os.path.join(FX, "tiny_3gaussians.ply"))
    raw = gs3d.raw_from_gaussians(model)
    for k, f in (("raw_positions", "positions"), ("raw_scales", "scales"), ("raw_rotations", "rotations"),
                 ("raw_sh", "sh"), ("raw_opacities", "opacities")):
        assert U.bits_equal(getattr(raw, f), REF[k]), k
    out = tmp_path / "saved.ply"
    gs3d.save_ply(out, raw)
    assert out.read_bytes() == REF["saved_ply_bytes"].tobytes()
    back, _ = gs3d.load_ply(out, activate=False)   # the stored raw values, unchanged
    for f in ("positions", "scales", "rotations", "sh", "opacities"):
        assert U.bits_equal(getattr(back, f), getattr(raw, f)), f


@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_ply_round_trip_every_degree(tmp_path, deg):
    sc = S.random_scene(5000, sh_degree=deg, seed=80 + deg)
    path = tmp_path / f"deg{deg}.ply"
    gs3d.save_ply(path, sc)
    info = gs3d.ply_info(path)
    assert info == dict(count=5000, sh_degree=deg, max_coeffs=(deg + 1) ** 2, has_filter_3D=False)
    back, _ = gs3d.load_ply(path, activate=False)
    for f in ("positions", "scales", "rotations", "sh", "opacities"):
        assert U.bits_equal(getattr(back, f), getattr(sc, f)), f


def test_ppm_matches_reference(tmp_path):
    img = REF["ppm_in"]
    h, w = img.shape[:2]
    path = tmp_path / "x.ppm"
    gs3d.write_ppm(path, img, w, h)
    assert path.read_bytes() == REF["ppm_bytes"].tobytes()
    back, bw, bh = gs3d.read_ppm(path)
    assert (bw, bh) == (w, h)
    assert U.bits_equal(back, REF["ppm_read"])


def test_ppm_comments_and_resize(tmp_path):
    rng = np.random.default_rng(9)
    px = rng.integers(0, 256, (7, 5, 3), dtype=np.uint8)
    path = tmp_path / "c.ppm"
    # comments before the size, as the reference's reader takes them (image_io.cpp:33-42)
    path.write_bytes(b"P6\n# a comment\n# another\n5 7\n255\n" + px.tobytes())
    img, w, h = gs3d.read_ppm(path)
    assert (w, h) == (5, 7)
    assert U.bits_equal(img, px.reshape(-1).astype(np.float32) * np.float32(1.0 / 255.0))
    r = gs3d.resize_nearest(img, 5, 7, 3, 11).reshape(11, 3, 3)
    src = img.reshape(7, 5, 3)
    want = np.stack([np.stack([src[y * 7 // 11, x * 5 // 3] for x in range(3)]) for y in range(11)])
    assert U.bits_equal(r, want)


def test_load_views(tmp_path):
    cams = gs3d.load_cameras(os.path.join(FX, "cameras.json"))[:3]
    for i, (cam, name) in enumerate(cams):
        w, h = (cam.width, cam.height) if i else (cam.width // 2, cam.height // 2)   # one needs a resize
        gs3d.write_ppm(tmp_path / f"{name}.ppm", np.full(w * h * 3, 0.25 * (i + 1), np.float32), w, h)
    views = gs3d.load_views(os.path.join(FX, "cameras.json"), str(tmp_path))
    assert len(views) == 3
    for i, (cam, img) in enumerate(views):
        assert img.size == cam.width * cam.height * 3
        q = np.float32(int(np.float32(0.25 * (i + 1)) * np.float32(255.0) + np.float32(0.5)))   # writePPM's byte
        assert np.all(img == q * np.float32(1.0 / 255.0))


def test_malformed_files_are_refused(tmp_path):
    bad = tmp_path / "bad.ply"
    bad.write_bytes(b"not a ply\n")
    with pytest.raises(gs3d.Gs3dError):
        gs3d.ply_info(bad)
    good = tmp_path / "good.ply"
    gs3d.save_ply(good, S.random_scene(10, seed=1))
    cut = tmp_path / "cut.ply"
    cut.write_bytes(good.read_bytes()[:-8])
    with pytest.raises(gs3d.Gs3dError):
        gs3d.load_ply(cut)
    ascii_ply = tmp_path / "ascii.ply"
    ascii_ply.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n0\n")
    with pytest.raises(gs3d.Gs3dError):
        gs3d.ply_info(ascii_ply)
    with pytest.raises(gs3d.Gs3dError):
        gs3d.read_ppm(tmp_path / "missing.ppm")
    p16 = tmp_path / "p16.ppm"
    p16.write_bytes(b"P6\n1 1\n65535\n" + bytes(6))
    with pytest.raises(gs3d.Gs3dError):
        gs3d.read_ppm(p16)
    js = tmp_path / "c.json"
    js.write_text("{not json")
    with pytest.raises(gs3d.Gs3dError):
        gs3d.load_cameras(js)
    js.write_text('[{"id": 0, "width": 10, "height": 10, "fx": 0, "fy": 5, "position": [0, 0, 0],'
                  ' "rotation": [[1, 0, 0], [0, 1, 0], [0, 0, 1]]}]')
    assert gs3d.load_cameras(js) == []     # fx <= 0: not a camera, skipped like the reference

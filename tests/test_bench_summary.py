"""bench.py host logic, on CPU: the per-stage algorithmic bytes and the
roofline block of a measured form, fed with made-up timings.  The DRAM-traffic
figure comes from the committed ncu table of the same form (both 16-bit forms
run the same rasterisers), scaled by tile pairs."""
import json
import os
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _fake_result(form, P):
    stage_ms = [0.01, 0.04, 0.15, 0.13, 0.02, 0.21, 0.42, 0.29]   # bench.STAGES order
    return {"form": form, "tile_pairs": P, "sort_passes": 6, "stage_ms": stage_ms, "ms_total": 200 * 1.3,
            "e2e_s": 0.3, "launches": 6000, "loss_first": 1.0, "loss_last": 0.5, "clocks": {}, "graph": True,
            "raster_pixels_per_thread": {"forward": 2, "backward": 2},
            "raster_staging_batch": {"forward": 128, "backward": 128}}


def test_traffic_table_has_both_forms():
    t = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))
    for form in ("bf16", "plain"):
        for k in ("raster_fwd", "raster_bwd"):
            e = t["forms"][form][k]
            assert e["bytes_per_launch"] == e["read"] + e["write"] and e["pairs"] > 0 and e["scale"] == "pairs"


def test_summary_roofline_uses_the_forms_own_traffic():
    a = types.SimpleNamespace(steps=200)
    X, N, T, P = 1920 * 1080, 1_000_000, 8160, 7_280_000
    t = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))["forms"]
    for form, key in (("bf16", "bf16"), ("fp16", "bf16"), ("plain", "plain")):
        s = bench._summary(a, _fake_result(form, P), 1, X, N, T, True, (6455.3, "measured"))
        rf = s["roofline"]
        assert rf["kernel"] == "raster_bwd"   # the longest stage of the fake timings
        want = t[key]["raster_bwd"]["bytes_per_launch"] * P / t[key]["raster_bwd"]["pairs"]
        assert abs(rf["traffic"] - want) <= 1e-6 * want
        assert abs(rf["frac"] - rf["achieved"] / 6455.3) < 1e-3
        assert s["value"] > 0 and s["ms_per_step"] == 1.3


def test_reduced_form_counts_three_depth_passes():
    X, N, T, P = 1920 * 1080, 1_000_000, 8160, 7_280_000
    b16 = bench.stage_bytes(N, P, X, T, 6, form="bf16")
    assert b16["sort_hist"] == N * 4 + 3 * N * 16 + N * 32 + P * 8 + P * 4
    plain = bench.stage_bytes(N, P, X, T, 6, form="plain")
    assert plain["preprocess"] > b16["preprocess"]   # FP32 parameters against 16-bit storage

"""GPU: gs3dc_sort_pairs_static, the pair sort that allocates no device memory.

It sorts caller-owned device buffers with its scratch in a static device
array.  Its output must equal gs3dc_sort_pairs' (keys, values and tile ranges
bit-exact) on consecutive calls that reuse the shared scratch: an even and an
odd number of radix passes, a smaller sort after a larger one, and a sort of
exactly the maximum size, in place with an even and an odd number of passes.
Oversized, non-device, partly overlapping and out-of-grid inputs and a
capturing stream are rejected with a message.  This file is collected last so that it also runs after every other
GPU test of the session; it passes on its own as well.
"""
import ctypes

import numpy as np
import pytest

from aaags_claude_b200 import gs3d

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1048576   # GS3DC_STATIC_SORT_MAX_PAIRS


def _pairs(P: int, num_tiles: int, seed: int):
    rng = np.random.default_rng(seed)
    tiles = rng.integers(0, num_tiles, P, dtype=np.uint64)
    # depths rounded to 1/64 so that many keys are equal and stability shows
    depth = (np.round(rng.uniform(0.2, 20.0, P) * 64) / 64).astype(np.float32)
    keys = (tiles << np.uint64(32)) | depth.view(np.uint32).astype(np.uint64)
    # non-decreasing values (Gaussian indices in emission order, as the binner
    # writes them): equal keys then have one order however the sort breaks ties
    vals = np.sort(rng.integers(0, 1 << 20, P, dtype=np.uint32))
    return keys, vals


def _static_sort(keys: np.ndarray, vals: np.ndarray, num_tiles: int, in_place: bool = False):
    import torch
    L = gs3d.load_library()
    P = int(keys.shape[0])
    k_in = torch.from_numpy(keys.view(np.int64)).cuda()
    v_in = torch.from_numpy(vals.view(np.int32)).cuda()
    k_out = k_in if in_place else torch.full((max(P, 1),), -1, dtype=torch.int64, device="cuda")
    v_out = v_in if in_place else torch.full((max(P, 1),), -1, dtype=torch.int32, device="cuda")
    ranges = torch.full((2 * num_tiles,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    err = ctypes.create_string_buffer(512)
    rc = L.gs3dc_sort_pairs_static(P, k_in.data_ptr(), v_in.data_ptr(), num_tiles, k_out.data_ptr(),
                                   v_out.data_ptr(), ranges.data_ptr(), None, err, len(err))
    assert rc == gs3d.OK, err.value.decode()
    return (k_out[:P].cpu().numpy().view(np.uint64), v_out[:P].cpu().numpy().view(np.uint32),
            ranges.cpu().numpy().view(np.uint32))


def _check_against_sort_pairs(ctx, P, num_tiles, seed, in_place=False):
    keys, vals = _pairs(P, num_tiles, seed)
    ks, vs, rs = _static_sort(keys, vals, num_tiles, in_place)
    k_ref, v_ref, r_ref = ctx.sort_pairs(keys, vals, num_tiles)
    assert np.array_equal(ks, k_ref)
    assert np.array_equal(vs, v_ref)
    assert np.array_equal(rs, r_ref)
    assert np.all(ks[1:] >= ks[:-1])


def test_two_calls_in_a_row_match_sort_pairs(ctx):
    # 1920x1080 tiles: 45 key bits, 6 passes (even); then 200 tiles: 40 bits,
    # 5 passes (odd), a smaller sort over the larger one's leftover scratch
    _check_against_sort_pairs(ctx, 400_000, 8160, seed=11)
    _check_against_sort_pairs(ctx, 70_000, 200, seed=12)


def test_maximum_size_and_in_place(ctx):
    _check_against_sort_pairs(ctx, MAX_PAIRS, 8160, seed=13)
    _check_against_sort_pairs(ctx, 123_457, 8160, seed=14, in_place=True)   # 6 passes (even)
    _check_against_sort_pairs(ctx, 98_765, 200, seed=16, in_place=True)     # 5 passes (odd)
    _check_against_sort_pairs(ctx, 5_000, 1, seed=15)   # one tile: 4 passes


def test_rejects_a_key_outside_the_tile_grid(ctx):
    import torch
    L = gs3d.load_library()
    keys, vals = _pairs(10_000, 64, seed=17)
    keys[1234] = (np.uint64(64) << np.uint64(32)) | (keys[1234] & np.uint64(0xFFFFFFFF))   # tile 64 of 0..63
    k_in = torch.from_numpy(keys.view(np.int64)).cuda()
    v_in = torch.from_numpy(vals.view(np.int32)).cuda()
    k_out = torch.empty_like(k_in)
    v_out = torch.empty_like(v_in)
    ranges = torch.full((2 * 64,), -1, dtype=torch.int32, device="cuda")
    err = ctypes.create_string_buffer(512)
    rc = L.gs3dc_sort_pairs_static(keys.shape[0], k_in.data_ptr(), v_in.data_ptr(), 64, k_out.data_ptr(),
                                   v_out.data_ptr(), ranges.data_ptr(), None, err, len(err))
    assert rc == gs3d.ERR_INVALID_ARG and b"tile field" in err.value
    # nothing was indexed with the bad key: the ranges stay cleared
    assert int(ranges.abs().sum()) == 0
    # the shared scratch is usable by the next call
    _check_against_sort_pairs(ctx, 50_000, 64, seed=18)


def test_rejects_partial_overlap_and_a_capturing_stream():
    import torch
    L = gs3d.load_library()
    err = ctypes.create_string_buffer(512)
    P = 1000
    buf = torch.zeros(4 * P, dtype=torch.int64, device="cuda")
    vals = torch.zeros(P, dtype=torch.int32, device="cuda")
    vout = torch.zeros(P, dtype=torch.int32, device="cuda")
    ranges = torch.zeros(8, dtype=torch.int32, device="cuda")
    base = buf.data_ptr()
    # keys_sorted starts inside keys (not the same buffer)
    rc = L.gs3dc_sort_pairs_static(P, base, vals.data_ptr(), 4, base + 8 * 10, vout.data_ptr(), ranges.data_ptr(),
                                   None, err, len(err))
    assert rc == gs3d.ERR_INVALID_ARG and b"overlap" in err.value
    # tile ranges inside the sorted keys
    rc = L.gs3dc_sort_pairs_static(P, base, vals.data_ptr(), 4, base + 8 * P, vout.data_ptr(), base + 8 * (P + 5),
                                   None, err, len(err))
    assert rc == gs3d.ERR_INVALID_ARG and b"overlap" in err.value
    # a capturing stream is refused before anything is enqueued
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    x = torch.zeros(4, device="cuda")
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        x.add_(1.0)
        rc = L.gs3dc_sort_pairs_static(P, base, vals.data_ptr(), 4, base + 8 * P, vout.data_ptr(),
                                       ranges.data_ptr(), ctypes.c_void_p(s.cuda_stream), err, len(err))
    assert rc == gs3d.ERR_INVALID_ARG and b"captured" in err.value
    g.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 4.0


def test_rejects_oversized_and_host_inputs():
    import torch
    L = gs3d.load_library()
    err = ctypes.create_string_buffer(512)
    d = torch.zeros(16, dtype=torch.int64, device="cuda")
    rc = L.gs3dc_sort_pairs_static(MAX_PAIRS + 1, d.data_ptr(), d.data_ptr(), 4, d.data_ptr(), d.data_ptr(),
                                   d.data_ptr(), None, err, len(err))
    assert rc == gs3d.ERR_INVALID_ARG and b"exceed the static sort scratch" in err.value
    h = np.zeros(16, np.uint64)
    rc = L.gs3dc_sort_pairs_static(4, h.ctypes.data, h.ctypes.data, 4, d.data_ptr(), d.data_ptr(), d.data_ptr(),
                                   None, err, len(err))
    assert rc == gs3d.ERR_INVALID_ARG and b"device memory" in err.value
    # empty input: ranges cleared, nothing else touched
    r = torch.full((8,), 7, dtype=torch.int32, device="cuda")
    rc = L.gs3dc_sort_pairs_static(0, None, None, 4, None, None, r.data_ptr(), None, err, len(err))
    assert rc == gs3d.OK and int(r.abs().sum()) == 0

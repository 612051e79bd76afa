"""Uneven SSIMULACRA2 batches (VshipExt_SSIMU2Batch*): pairs of mixed resolutions and formats
in one persistent launch.

The batch path must give the per-pair handler path's results (the same front and map tile
code; with 32-row tiles the same tiles, shift constants and partial sums, so scores agree to
within one float rounding of the final reduction), stay within the engine's accuracy bar
(|dSSIMU2| <= 1e-3) against the FP64 oracle for every tile height, give exactly 100 on
identical inputs, and reject what it does not support with the reference's error codes.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

SCORE_TOL = 1e-3

# (format, width, height, seed): small odd sizes, both fast paths and the generic one, and
# one frame wider than a single map tile row of every level.
MIX = [
    ("rgb8", 97, 61, 1), ("yuv420p10", 160, 96, 2), ("rgb8", 333, 211, 3), ("yuv420p10", 640, 360, 4),
    ("rgb8", 256, 256, 5), ("yuv420p10", 98, 66, 6), ("rgb8", 640, 360, 7), ("yuv444p8", 200, 120, 8),
    ("rgb8", 97, 61, 9), ("yuv420p10", 160, 96, 10), ("rgb8", 1280, 720, 11),
]


def _cs(fmt, w, h):
    if fmt == "rgb8":
        return abi.srgb8(w, h)
    if fmt == "yuv420p10":
        return abi.yuv420_10bit_bt709(w, h)
    # 8-bit 4:4:4 limited-range BT.709: the generic front path
    return abi.colorspace(w, h, sample=abi.SampleUINT8, range_=abi.RangeLimited, subw=0, subh=0,
                          family=abi.ColorYUV, matrix=abi.MATRIX_BT709, transfer=abi.TRC_BT709,
                          primaries=abi.PRIMARIES_BT709)


def _planes(fmt, w, h, seed):
    if fmt == "yuv444p8":
        p1, p2, _ = synth.make_pairs(1, w, h, fmt="rgb8", seed=seed)[0]
        return p1, p2, [w, w, w]
    return synth.make_pairs(1, w, h, fmt=fmt, seed=seed)[0]


def _dev(planes):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(p).view(np.uint8).copy()).cuda() for p in planes]


@pytest.fixture(scope="module")
def mix():
    out = []
    for fmt, w, h, seed in MIX:
        p1, p2, ls = _planes(fmt, w, h, seed)
        out.append(dict(fmt=fmt, w=w, h=h, cs=_cs(fmt, w, h), p1=p1, p2=p2, ls=ls, d1=_dev(p1), d2=_dev(p2)))
    return out


def _device_items(mix):
    return [(m["cs"], m["cs"], [t.data_ptr() for t in m["d1"]], [t.data_ptr() for t in m["d2"]], m["ls"], m["ls"])
            for m in mix]


def _handler_scores(mix):
    import torch
    scores, feats = [], []
    for m in mix:
        s = torch.zeros(1, dtype=torch.float64, device="cuda")
        f = torch.zeros(108, dtype=torch.float32, device="cuda")
        with api.SSIMU2(m["cs"]) as h:
            h.compute_device(1, [t.data_ptr() for t in m["d1"]], [t.data_ptr() for t in m["d2"]], m["ls"], m["ls"],
                             s.data_ptr(), f.data_ptr(), 0)
            torch.cuda.synchronize()
        scores.append(s.item())
        feats.append(f.cpu().numpy())
    return np.array(scores), np.stack(feats)


def _batch_scores(mix, rows):
    import torch
    n = len(mix)
    s = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
    f = torch.full((n, 108), -1.0, dtype=torch.float32, device="cuda")
    with api.SSIMU2Batch() as b:
        b.set_tile_rows(rows)
        b.compute_device(_device_items(mix), s.data_ptr(), f.data_ptr())
        torch.cuda.synchronize()
        assert b.tile_rows() == rows
    return s.cpu().numpy(), f.cpu().numpy()


def test_batch_equals_handler_path_with_32_row_tiles(gpu, mix):
    ref_s, ref_f = _handler_scores(mix)
    got_s, got_f = _batch_scores(mix, 32)
    np.testing.assert_allclose(got_s, ref_s, rtol=0, atol=1e-5)
    np.testing.assert_allclose(got_f, ref_f, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("rows", [16, 32, 64])
def test_batch_matches_oracle_for_each_tile_height(gpu, oracle_lib, mix, rows):
    got_s, got_f = _batch_scores(mix, rows)
    for i, m in enumerate(mix):
        q, d, f = oracle_lib.ssimu2(oracle_lib.convert(m["p1"], m["ls"], m["cs"]),
                                    oracle_lib.convert(m["p2"], m["ls"], m["cs"]))
        assert abs(got_s[i] - d) <= SCORE_TOL, (rows, m["fmt"], m["w"], m["h"], got_s[i], d)
        np.testing.assert_allclose(got_f[i], f, rtol=2e-3, atol=1e-5)


def test_batch_host_api_matches_device_api(gpu, mix):
    dev_s, dev_f = _batch_scores(mix, 32)
    items = [(m["cs"], m["cs"], m["p1"], m["p2"], m["ls"], m["ls"]) for m in mix]
    with api.SSIMU2Batch() as b:
        b.set_tile_rows(32)
        s, f = b.compute(items, features=True)
    np.testing.assert_array_equal(s, dev_s)
    np.testing.assert_array_equal(f, dev_f)


def test_batch_identity_is_exactly_100(gpu, mix):
    import torch
    items = [(m["cs"], m["cs"], [t.data_ptr() for t in m["d1"]], [t.data_ptr() for t in m["d1"]], m["ls"], m["ls"])
             for m in mix]
    s = torch.zeros(len(items), dtype=torch.float64, device="cuda")
    for rows in (16, 32, 64):
        with api.SSIMU2Batch() as b:
            b.set_tile_rows(rows)
            b.compute_device(items, s.data_ptr())
            torch.cuda.synchronize()
        assert (s.cpu().numpy() == 100.0).all(), rows


def test_batch_repeated_calls_reuse_graphs_and_buffers(gpu, mix):
    import torch
    ref_s, _ = _batch_scores(mix, 32)
    items = _device_items(mix)
    s = torch.zeros(len(items), dtype=torch.float64, device="cuda")
    with api.SSIMU2Batch() as b:
        b.set_tile_rows(32)
        # growing and shrinking batches, then the full one again
        for k in (3, len(items), 1, len(items)):
            s.fill_(-1.0)
            b.compute_device(items[:k], s.data_ptr())
            torch.cuda.synchronize()
            np.testing.assert_array_equal(s.cpu().numpy()[:k], ref_s[:k])


def test_batch_autotune_writes_its_cache(gpu, mix, tmp_path, monkeypatch):
    import torch
    path = tmp_path / "tiles.json"
    monkeypatch.setenv("VSHIP_TUNE_CACHE", str(path))
    items = _device_items(mix)
    s = torch.zeros(len(items), dtype=torch.float64, device="cuda")
    with api.SSIMU2Batch() as b:
        b.compute_device(items, s.data_ptr())
        torch.cuda.synchronize()
        chosen = b.tile_rows()
    assert chosen in (16, 32, 64)
    entries = json.loads(path.read_text())
    assert len(entries) == 1
    (key, val), = entries.items()
    assert val == chosen and "ssimu2_batch" in key
    with api.SSIMU2Batch() as b:  # a new handler takes the cached choice
        b.compute_device(items, s.data_ptr())
        torch.cuda.synchronize()
        assert b.tile_rows() == chosen


def test_batch_errors(gpu, mix):
    import torch
    m = mix[0]
    s = torch.zeros(2, dtype=torch.float64, device="cuda")
    ptrs = [t.data_ptr() for t in m["d1"]]
    with api.SSIMU2Batch() as b:
        with pytest.raises(api.VshipError) as e:
            b.set_tile_rows(24)
        assert e.value.code == abi.BadErrorType
        resized = _cs(m["fmt"], m["w"], m["h"])
        resized.target_width, resized.target_height = 2 * m["w"], 2 * m["h"]
        with pytest.raises(api.VshipError) as e:
            b.compute_device([(resized, resized, ptrs, ptrs, m["ls"], m["ls"])], s.data_ptr())
        assert e.value.code == abi.BadErrorType
        other = _cs(m["fmt"], m["w"] + 2, m["h"])
        with pytest.raises(api.VshipError) as e:
            b.compute_device([(m["cs"], other, ptrs, ptrs, m["ls"], m["ls"])], s.data_ptr())
        assert e.value.code == abi.DifferingInputType
        with pytest.raises(api.VshipError) as e:
            b.compute_device([(m["cs"], m["cs"], [ptrs[0], 0, ptrs[2]], ptrs, m["ls"], m["ls"])], s.data_ptr())
        assert e.value.code == abi.BadPointer
        with pytest.raises(api.VshipError) as e:
            b.compute_device([(m["cs"], m["cs"], ptrs, ptrs, [1, 1, 1], m["ls"])], s.data_ptr())
        assert e.value.code == abi.BadPointer
        # the handler is still usable after errors
        b.set_tile_rows(32)
        b.compute_device([(m["cs"], m["cs"], ptrs, ptrs, m["ls"], m["ls"])], s.data_ptr())
        torch.cuda.synchronize()
        assert s[0].item() == 100.0
    L = api.load()
    assert L.VshipExt_SSIMU2BatchFree(abi.SSIMU2BatchHandler(12345)) == abi.BadHandler


def test_batch_wait_limit_reports_error_and_recovers(gpu, mix):
    """A launch whose last front tile is held back: the map tiles of that pair wait for a
    pyramid that is never finished, the bounded wait gives up after its 2 s limit and sets the
    launch's error word, and the call reports Vship_HIPError.  The wait ends, nothing faults,
    and the next launches give the scores of launches without the hold, through both entries."""
    import time
    import torch
    items = [(m["cs"], m["cs"], m["p1"], m["p2"], m["ls"], m["ls"]) for m in mix[:5]]
    with api.SSIMU2Batch() as b:
        b.set_tile_rows(32)
        want = b.compute(items)
        b.hold_front_tile()
        t0 = time.perf_counter()
        with pytest.raises(api.VshipError) as e:
            b.compute(items)
        waited = time.perf_counter() - t0
        assert e.value.code == abi.HIPError
        assert "time limit" in str(e.value)
        assert 1.9 < waited < 30.0, waited
        np.testing.assert_array_equal(b.compute(items), want)
        # device entry: the launch is queued without waiting, so the next call reports it
        dev = _device_items(mix[:5])
        s = torch.zeros(len(dev), dtype=torch.float64, device="cuda")
        b.hold_front_tile()
        b.compute_device(dev, s.data_ptr())
        torch.cuda.synchronize()
        with pytest.raises(api.VshipError) as e:
            b.compute_device(dev, s.data_ptr())
        assert e.value.code == abi.HIPError
        b.compute_device(dev, s.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(s.cpu().numpy(), want)


def test_batch_uneven_1080p_and_4k(gpu):
    """Large frames of the uneven workload: batch scores equal the per-pair handler path."""
    import torch
    specs = [("rgb8", 3840, 2160, 31), ("rgb8", 1920, 1080, 32), ("rgb8", 640, 360, 33), ("rgb8", 1280, 720, 34),
             ("rgb8", 1920, 1080, 35)]
    mix = []
    for fmt, w, h, seed in specs:
        p1, p2, ls = _planes(fmt, w, h, seed)
        mix.append(dict(fmt=fmt, w=w, h=h, cs=_cs(fmt, w, h), p1=p1, p2=p2, ls=ls, d1=_dev(p1), d2=_dev(p2)))
    ref_s, ref_f = _handler_scores(mix)
    got_s, got_f = _batch_scores(mix, 32)
    np.testing.assert_allclose(got_s, ref_s, rtol=0, atol=1e-5)
    for rows in (16, 64):
        s, _ = _batch_scores(mix, rows)
        np.testing.assert_allclose(s, ref_s, rtol=0, atol=2e-4)
    del mix
    torch.cuda.empty_cache()

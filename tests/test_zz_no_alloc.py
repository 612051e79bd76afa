"""VshipExt_ComputeSSIMU2NoAlloc: scoring without any GPU allocation.

Callers that cannot call cudaMalloc (processes whose GPU memory is a fixed budget handed out
up front, real-time loops that must not block in the allocator) use this entry point; its
scratch lives in a fixed array inside the library and is reused by every call.  It runs the
same kernels on the same data as the handler-based device entry point, so it must give the
same results bit for bit on consecutive calls that reuse that array, including calls of
different sizes, and must refuse frames larger than the array with an error.

This file is collected last so that a stop-at-first-failure run has already run every other
test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

def _to_device(planes):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(p).view(np.uint8).copy()).cuda() for p in planes]


def _no_alloc(L, cs, d1, d2, ls, d_score, d_feat):
    a1 = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in d1])
    a2 = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in d2])
    return L.VshipExt_ComputeSSIMU2NoAlloc(cs, cs, d_score.data_ptr(), d_feat.data_ptr(), a1, a2,
                                           abi.LineSizes(*ls), abi.LineSizes(*ls), None)


def test_no_alloc_matches_handler_path_on_consecutive_calls(gpu):
    import torch
    L = gpu
    cases = [
        ("yuv420p10", 640, 360, 11),
        ("yuv420p10", 640, 360, 12),     # same size again: the array keeps the previous call's data
        ("rgb8", 1920, 1080, 13),        # larger frame and another format in the same array
        ("rgb8", 97, 61, 14),            # then a small odd-sized one
    ]
    for fmt, w, h, seed in cases:
        p1, p2, ls = synth.make_pairs(1, w, h, fmt=fmt, seed=seed)[0]
        cs = abi.srgb8(w, h) if fmt == "rgb8" else abi.yuv420_10bit_bt709(w, h)
        d1, d2 = _to_device(p1), _to_device(p2)
        ref_score = torch.zeros(1, dtype=torch.float64, device="cuda")
        ref_feat = torch.zeros(108, dtype=torch.float32, device="cuda")
        with api.SSIMU2(cs) as hd:
            hd.compute_device(1, [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls,
                              ref_score.data_ptr(), ref_feat.data_ptr(), 0)
        torch.cuda.synchronize()
        score = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        feat = torch.full((108,), -1.0, dtype=torch.float32, device="cuda")
        assert _no_alloc(L, cs, d1, d2, ls, score, feat) == abi.NoError
        torch.cuda.synchronize()
        assert score.item() == ref_score.item(), (fmt, w, h, score.item(), ref_score.item())
        np.testing.assert_array_equal(feat.cpu().numpy(), ref_feat.cpu().numpy())
        assert 0.0 < score.item() < 100.0


def test_no_alloc_with_odd_plane_addresses(gpu):
    """16-bit samples at odd device addresses (even strides) take byte loads and score exactly
    as the handler's host path, which stages the frames at aligned addresses."""
    import torch
    L = gpu
    w, h = 130, 98
    p1, p2, ls = synth.make_pairs(1, w, h, fmt="yuv420p10", seed=32)[0]
    cs = abi.yuv420_10bit_bt709(w, h)
    keep = []

    def odd(planes):
        ptrs = []
        for p in planes:
            raw = np.ascontiguousarray(p).view(np.uint8).reshape(-1)
            buf = torch.zeros(raw.size + 16, dtype=torch.uint8, device="cuda")
            buf[1:1 + raw.size] = torch.from_numpy(raw).cuda()
            keep.append(buf)
            ptrs.append(buf.data_ptr() + 1)
        return (ctypes.c_void_p * 3)(*ptrs)

    with api.SSIMU2(cs) as hd:
        want = hd.compute(p1, p2, ls)
    score = torch.zeros(1, dtype=torch.float64, device="cuda")
    feat = torch.zeros(108, dtype=torch.float32, device="cuda")
    rc = L.VshipExt_ComputeSSIMU2NoAlloc(cs, cs, score.data_ptr(), feat.data_ptr(), odd(p1), odd(p2),
                                         abi.LineSizes(*ls), abi.LineSizes(*ls), None)
    assert rc == abi.NoError
    torch.cuda.synchronize()
    assert score.item() == want, (score.item(), want)


def test_no_alloc_rejects_frames_beyond_its_scratch(gpu):
    import torch
    L = gpu
    w, h = 3840, 2160
    cs = abi.srgb8(w, h)
    planes = [np.zeros((h, w), np.uint8)] * 3
    d1, d2 = _to_device(planes), _to_device(planes)
    score = torch.zeros(1, dtype=torch.float64, device="cuda")
    feat = torch.zeros(108, dtype=torch.float32, device="cuda")
    rc = _no_alloc(L, cs, d1, d2, [w] * 3, score, feat)
    assert rc == abi.OutOfVRAM
    n = L.Vship_GetDetailedLastError(None, 0)
    buf = ctypes.create_string_buffer(n)
    L.Vship_GetDetailedLastError(buf, n)
    assert "bytes of scratch" in buf.value.decode()

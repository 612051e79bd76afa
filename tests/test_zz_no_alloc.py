"""VshipExt_ComputeSSIMU2NoAlloc: scoring without any GPU allocation.

Callers that cannot call cudaMalloc (work captured into a CUDA graph, processes with a fixed
GPU memory budget, real-time loops) use this entry point; its scratch lives in a fixed array
inside the library and is reused by every call.  It must give the same results as the
handler-based device entry point on consecutive calls that reuse that array, including calls
of different sizes, and must refuse frames larger than the array with an error.

This file is collected last so that a stop-at-first-failure run has already run every other
test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

SCORE_TOL = 1e-3  # the engine's parity tolerance on SSIMULACRA2 scores


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
        assert abs(score.item() - ref_score.item()) <= SCORE_TOL, (fmt, w, h, score.item(), ref_score.item())
        np.testing.assert_allclose(feat.cpu().numpy(), ref_feat.cpu().numpy(), rtol=2e-4, atol=1e-6)
        assert 0.0 < score.item() < 100.0


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

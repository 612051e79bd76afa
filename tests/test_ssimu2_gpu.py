"""GPU parity of the SSIMULACRA2 path through the C ABI against the FP64 oracle.

Tolerance: |dSSIMU2| <= 1e-3 against FP64 (the accuracy bar of the engine); features within
2e-4 relative (+1e-6 absolute).  Identical inputs must give exactly 100, as the reference's identity test
requires (test/libvshipTestIdentity.cpp:357-384).
"""
import numpy as np
import pytest

from tests.golden.cases import CASES, build_case
from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

SCORE_TOL = 1e-3


def _oracle_score(oracle, a, b):
    (p1, ls1, cs1), (p2, ls2, cs2) = a, b
    return oracle.ssimu2(oracle.convert(p1, ls1, cs1), oracle.convert(p2, ls2, cs2))


@pytest.mark.parametrize("case", [c for c in CASES if c["metric"] == "ssimu2"], ids=lambda c: c["name"])
def test_cases_match_oracle(gpu, oracle_lib, case):
    a, b = build_case(case)
    with api.SSIMU2(a[2], b[2]) as h:
        got = h.compute(a[0], b[0], a[1], b[1])
        feats = h.last_features()
    q, d, f = _oracle_score(oracle_lib, a, b)
    if case.get("identical"):
        assert got == 100.0
        return
    assert abs(got - d) <= SCORE_TOL, (got, d)
    np.testing.assert_allclose(feats, f, rtol=2e-4, atol=1e-6)


@pytest.mark.parametrize("fmt,w,h", [("rgb8", 64, 64), ("yuv420p10", 130, 98), ("rgb8", 1920, 1080)])
def test_identity_exact(gpu, fmt, w, h):
    p1, _, ls = synth.make_pairs(1, w, h, fmt=fmt, seed=9)[0]
    cs = abi.srgb8(w, h) if fmt == "rgb8" else abi.yuv420_10bit_bt709(w, h)
    padded, pls = synth.with_padding(p1, ls, [13, 5, 9])
    with api.SSIMU2(cs) as hd:
        assert hd.compute(p1, padded, ls, pls) == 100.0


def test_1080p_workloads(gpu, oracle_lib):
    for fmt, cs in (("rgb8", abi.srgb8(1920, 1080)), ("yuv420p10", abi.yuv420_10bit_bt709(1920, 1080))):
        pairs = synth.make_pairs(2, 1920, 1080, fmt=fmt, seed=21)
        with api.SSIMU2(cs) as h:
            for p1, p2, ls in pairs:
                got = h.compute(p1, p2, ls)
                _, d, _ = oracle_lib.ssimu2(oracle_lib.convert(p1, ls, cs), oracle_lib.convert(p2, ls, cs))
                assert abs(got - d) <= SCORE_TOL, (fmt, got, d)


def test_device_batch_matches_host_api(gpu):
    import torch
    w, h = 640, 360
    pairs = synth.make_pairs(5, w, h, fmt="yuv420p10", seed=4, unique=2)
    cs = abi.yuv420_10bit_bt709(w, h)
    with api.SSIMU2(cs) as hd:
        host = [hd.compute(p1, p2, ls) for p1, p2, ls in pairs]
        dev = [([torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in p1],
                [torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in p2]) for p1, p2, _ in pairs]
        ptr1 = [t.data_ptr() for d in dev for t in d[0]]
        ptr2 = [t.data_ptr() for d in dev for t in d[1]]
        scores = torch.zeros(len(pairs), dtype=torch.float64, device="cuda")
        feats = torch.zeros(len(pairs), 108, dtype=torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        hd.compute_device(len(pairs), ptr1, ptr2, pairs[0][2], pairs[0][2], scores.data_ptr(), feats.data_ptr(), stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(scores.cpu().numpy(), np.array(host))
        assert torch.all(feats.sum(dim=1) > 0)


def test_device_api_strided_and_misaligned(gpu):
    import torch
    w, h = 97, 61
    cs = abi.colorspace(w, h, sample=abi.SampleUINT16, range_=abi.RangeFull, family=abi.ColorRGB,
                        matrix=abi.MATRIX_RGB, transfer=abi.TRC_sRGB)
    rng = np.random.default_rng(2)
    planes = [rng.integers(0, 65536, (h, w), dtype=np.uint16) for _ in range(3)]
    dist = [np.clip(p.astype(np.int64) + rng.integers(-900, 900, p.shape), 0, 65535).astype(np.uint16) for p in planes]
    with api.SSIMU2(cs) as hd:
        ref = hd.compute(planes, dist, [2 * w] * 3)
        # odd byte strides force the byte-wise sample loads
        pp, pls = synth.with_padding(planes, [2 * w] * 3, [3, 5, 7])
        dd, dls = synth.with_padding(dist, [2 * w] * 3, [1, 1, 1])
        d1 = [torch.from_numpy(p).cuda() for p in pp]
        d2 = [torch.from_numpy(p).cuda() for p in dd]
        s = torch.zeros(1, dtype=torch.float64, device="cuda")
        hd.compute_device(1, [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], pls, dls, s.data_ptr())
        torch.cuda.synchronize()
        assert abs(s.item() - ref) <= 1e-9


def test_errors(gpu):
    cs1, cs2 = abi.srgb8(64, 64), abi.srgb8(64, 65)
    with pytest.raises(api.VshipError) as e:
        api.SSIMU2(cs1, cs2)
    assert e.value.code == abi.DifferingInputType
    assert "DifferingInputType" in str(e.value)
    with api.SSIMU2(cs1) as h:
        p = [np.zeros((64, 64), np.uint8)] * 3
        with pytest.raises(api.VshipError) as e:
            h.compute(p, p, [32, 64, 64])
        assert e.value.code == abi.BadPointer
        assert h.compute(p, p, [64] * 3) == 100.0


def test_contiguous_frame_single_copy_matches_separate_planes(gpu):
    # FFVship lays a frame's planes back to back in one pinned buffer; the engine then copies
    # the frame in one transfer and reads it with the caller's strides.
    w, h = 333, 201
    p1, p2, ls = synth.make_pairs(1, w, h, fmt="yuv420p10", seed=17)[0]
    cs = abi.yuv420_10bit_bt709(w, h)
    with api.SSIMU2(cs) as hd:
        separate = hd.compute(p1, p2, ls)
        for pad in ([0, 0, 0], [6, 2, 10], [3, 1, 5]):   # the last one gives odd strides
            f1, pls = synth.with_padding(p1, ls, pad)
            f2, _ = synth.with_padding(p2, ls, pad)
            buf1 = np.concatenate([f.reshape(-1) for f in f1])
            buf2 = np.concatenate([f.reshape(-1) for f in f2])
            o = np.cumsum([0] + [f.nbytes for f in f1])
            ptr1 = [buf1.ctypes.data + int(o[i]) for i in range(3)]
            ptr2 = [buf2.ctypes.data + int(o[i]) for i in range(3)]
            assert hd.compute(ptr1, ptr2, pls) == separate
    with api.Butteraugli(cs, qnorm=5) as hb:
        sep, _ = hb.compute(p1, p2, ls)
        f1, pls = synth.with_padding(p1, ls, [6, 2, 10])
        f2, _ = synth.with_padding(p2, ls, [6, 2, 10])
        buf1 = np.concatenate([f.reshape(-1) for f in f1])
        buf2 = np.concatenate([f.reshape(-1) for f in f2])
        o = np.cumsum([0] + [f.nbytes for f in f1])
        got, _ = hb.compute([buf1.ctypes.data + int(o[i]) for i in range(3)],
                            [buf2.ctypes.data + int(o[i]) for i in range(3)], pls)
        assert got == sep


def _odd_device_planes(planes):
    """Each plane copied to device memory one byte past an even address: strides stay even
    but every plane pointer is odd."""
    import torch
    out, keep = [], []
    for p in planes:
        raw = np.ascontiguousarray(p).view(np.uint8).reshape(-1)
        buf = torch.zeros(raw.size + 16, dtype=torch.uint8, device="cuda")
        buf[1:1 + raw.size] = torch.from_numpy(raw).cuda()
        keep.append(buf)
        out.append(buf.data_ptr() + 1)
    return out, keep


def test_device_path_with_odd_plane_addresses(gpu):
    """16-bit samples at odd device addresses (even strides) take byte loads and score exactly
    as the host path, which stages the frames at aligned addresses."""
    import torch
    w, h = 130, 98
    p1, p2, ls = synth.make_pairs(1, w, h, fmt="yuv420p10", seed=31)[0]
    cs = abi.yuv420_10bit_bt709(w, h)
    a, ka = _odd_device_planes(p1)
    b, kb = _odd_device_planes(p2)
    assert all(x % 2 == 1 for x in a + b)
    score = torch.zeros(1, dtype=torch.float64, device="cuda")
    with api.SSIMU2(cs) as hd:
        want = hd.compute(p1, p2, ls)
        hd.compute_device(1, a, b, ls, ls, score.data_ptr(), 0, 0)
        torch.cuda.synchronize()
    assert score.item() == want, (score.item(), want)
    norms = torch.zeros(3, dtype=torch.float64, device="cuda")
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as hb:
        bwant, _ = hb.compute(p1, p2, ls)
        hb.compute_device(a, b, ls, ls, norms.data_ptr())
        torch.cuda.synchronize()
    assert tuple(norms.cpu().numpy()) == tuple(bwant), (norms.cpu().numpy(), bwant)


def test_concurrent_handlers_on_own_streams(gpu):
    """Single-pair device calls dealt round-robin over handlers, each on its own stream (the
    bench's device-throughput method for one pair per call): every score equals the host API's."""
    import torch
    w, h = 640, 360
    pairs = synth.make_pairs(6, w, h, fmt="rgb8", seed=21)
    cs = abi.srgb8(w, h)
    ls = pairs[0][2]
    with api.SSIMU2(cs) as hh:
        expect = [hh.compute(p1, p2, ls, ls) for p1, p2, _ in pairs]
    dev = [([torch.from_numpy(p.copy()).cuda() for p in p1], [torch.from_numpy(p.copy()).cuda() for p in p2])
           for p1, p2, _ in pairs]
    hs = [api.SSIMU2(cs) for _ in range(4)]
    streams = [torch.cuda.Stream() for _ in range(4)]
    try:
        out = torch.zeros(len(pairs), dtype=torch.float64, device="cuda")
        for rep in range(3):
            for i, (d1, d2) in enumerate(dev):
                k = (i + rep) % 4
                hs[k].compute_device(1, [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls,
                                     out[i:i + 1].data_ptr(), 0, streams[k].cuda_stream)
            torch.cuda.synchronize()
            assert out.cpu().numpy().tolist() == expect
    finally:
        for x in hs:
            x.close()

"""GPU parity of the Butteraugli path through the C ABI against the FP64 oracle.

Tolerance: relative 1e-4 on the Q-norm, 3-norm and inf-norm; the FP32 distortion map
element-wise within 2e-4 relative (+2e-6 absolute).  Identical inputs give norminf == 0
exactly, as the reference's identity test requires.
"""
import numpy as np
import pytest

from tests.golden.cases import CASES, build_case
from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

REL = 1e-4


@pytest.mark.parametrize("case", [c for c in CASES if c["metric"] == "butteraugli"], ids=lambda c: c["name"])
def test_cases_match_oracle(gpu, oracle_lib, case):
    (p1, ls1, cs1), (p2, ls2, cs2) = build_case(case)
    with api.Butteraugli(cs1, cs2, qnorm=case["qnorm"], intensity=case["intensity"]) as h:
        norms, dmap = h.compute(p1, p2, ls1, ls2, distmap=True)
    if case.get("identical"):
        assert norms[2] == 0.0 and norms[0] == 0.0
        assert np.all(dmap == 0)
        return
    onorms, odmap = oracle_lib.butteraugli(oracle_lib.convert(p1, ls1, cs1), oracle_lib.convert(p2, ls2, cs2),
                                           case["intensity"], case["qnorm"])
    for k in range(3):
        assert abs(norms[k] - onorms[k]) <= REL * abs(onorms[k]), (k, norms, onorms)
    np.testing.assert_allclose(dmap, odmap, rtol=2e-4, atol=2e-6)


def test_4k_pair(gpu, oracle_lib):
    p1, p2, ls = synth.make_pairs(1, 3840, 2160, fmt="rgb8", seed=40, blur=(0.0, 1.5))[0]
    cs = abi.srgb8(3840, 2160)
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as h:
        norms, _ = h.compute(p1, p2, ls)
    onorms, _ = oracle_lib.butteraugli(oracle_lib.convert(p1, ls, cs), oracle_lib.convert(p2, ls, cs), 203.0, 5)
    for k in range(3):
        assert abs(norms[k] - onorms[k]) <= REL * abs(onorms[k]), (k, norms, onorms)


def test_device_api_matches_host_api(gpu):
    import torch
    w, h = 300, 200
    p1, p2, ls = synth.make_pairs(1, w, h, fmt="yuv420p10", seed=6)[0]
    cs = abi.yuv420_10bit_bt709(w, h)
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as hd:
        host, hmap = hd.compute(p1, p2, ls, distmap=True)
        d1 = [torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in p1]
        d2 = [torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in p2]
        norms = torch.zeros(3, dtype=torch.float64, device="cuda")
        pitch = 320
        dmap = torch.zeros(h, pitch, dtype=torch.float32, device="cuda")
        hd.compute_device([t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls, norms.data_ptr(),
                          dmap.data_ptr(), pitch * 4, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(norms.cpu().numpy(), np.array(host))
        np.testing.assert_array_equal(dmap[:, :w].cpu().numpy(), hmap)


def test_concurrent_handlers_on_own_streams(gpu):
    """Several handlers, each on its own stream, calls interleaved from one thread (the bench's
    device-throughput method), and the legacy default stream: norms and distortion maps equal
    the host API's bit for bit.  Each handler also forks its distorted image onto a second
    stream internally, so this covers both levels of concurrency."""
    import torch
    w, h = 517, 301
    pairs = synth.make_pairs(4, w, h, fmt="rgb8", seed=12, blur=(0.0, 1.5))
    cs = abi.srgb8(w, h)
    ls = pairs[0][2]
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as hh:
        expect = [hh.compute(p1, p2, ls, distmap=True) for p1, p2, _ in pairs]
    dev = [([torch.from_numpy(p.copy()).cuda() for p in p1], [torch.from_numpy(p.copy()).cuda() for p in p2])
           for p1, p2, _ in pairs]
    hs = [api.Butteraugli(cs, qnorm=5, intensity=203.0) for _ in range(3)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream(), None]  # None: the legacy default stream
    try:
        norms = torch.zeros(len(pairs), 3, dtype=torch.float64, device="cuda")
        maps = torch.zeros(len(pairs), h, w, dtype=torch.float32, device="cuda")
        for rep in range(2):
            for i, (d1, d2) in enumerate(dev):
                k = (i + rep) % 3
                s = streams[k]
                hs[k].compute_device([t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls,
                                     norms[i].data_ptr(), maps[i].data_ptr(), w * 4, s.cuda_stream if s else 0)
            torch.cuda.synchronize()
            for i, (en, em) in enumerate(expect):
                np.testing.assert_array_equal(norms[i].cpu().numpy(), np.array(en))
                np.testing.assert_array_equal(maps[i].cpu().numpy(), em)
    finally:
        for x in hs:
            x.close()


def test_tma_wait_limit_reports_error_and_recovers(gpu):
    """The column pass's bounded tensor-map waits (widths a multiple of 4 take that pass): the
    test hook arms one box barrier with no copy behind it, the wait gives up, and the call fails
    with Vship_HIPError instead of hanging; the next call is whole again, through both APIs."""
    import torch
    w, h = 256, 128
    p1, p2, ls = synth.make_pairs(1, w, h, fmt="rgb8", seed=33, blur=(0.0, 1.5))[0]
    cs = abi.srgb8(w, h)
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as hb:
        good, gmap = hb.compute(p1, p2, ls, distmap=True)
        hb.test_tma_timeout()
        with pytest.raises(api.VshipError) as e:
            hb.compute(p1, p2, ls)
        assert e.value.code == abi.HIPError
        again, amap = hb.compute(p1, p2, ls, distmap=True)
        assert again == good
        np.testing.assert_array_equal(amap, gmap)
        # device API: the failure is reported by the call after the one that met it
        d1 = [torch.from_numpy(p.copy()).cuda() for p in p1]
        d2 = [torch.from_numpy(p.copy()).cuda() for p in p2]
        norms = torch.zeros(3, dtype=torch.float64, device="cuda")
        hb.test_tma_timeout()
        hb.compute_device([t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls, norms.data_ptr())
        torch.cuda.synchronize()
        with pytest.raises(api.VshipError):
            hb.compute_device([t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls, norms.data_ptr())
        hb.compute_device([t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls, norms.data_ptr())
        torch.cuda.synchronize()
        assert tuple(norms.cpu().numpy()) == tuple(good)
    odd = abi.srgb8(258, 128)
    with api.Butteraugli(odd, qnorm=5, intensity=203.0) as hb:
        with pytest.raises(api.VshipError) as e:
            hb.test_tma_timeout()
        assert e.value.code == abi.BadDeviceArgument

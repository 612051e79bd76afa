"""The bounds-check build on odd sizes (the stand-in for compute-sanitizer, which the GPU pool
does not offer).

vship_b200/libvship_bc.so is the same sources built with -DVSHIP_BOUNDS_CHECK: every device
buffer the engines allocate has a 64 KiB guard band on each side, buffer and guards start as
0xFF bytes (NaN in every float), and after each API call the guards are checked.  A kernel
that writes out of bounds makes the call fail with Vship_HIPError; one that reads out of
bounds or reads memory it never wrote turns the score into NaN.  Here every metric runs on
frame sizes whose tiles are ragged (1x1, 2x3, 17x9, 130x98, 1921x1081) in the two fast
formats and a generic one, through the host and device entry points and the uneven batch,
and must give finite results equal bit for bit to the product library's.
"""
import numpy as np
import pytest

from tests.golden.cases import build_case
from vship_b200 import abi, api, build, synth

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (2, 3), (17, 9), (130, 98), (1921, 1081)]


@pytest.fixture(scope="module")
def bc_lib(gpu):
    return api.load_library(build.build(bounds_check=True))


def test_guard_checker_finds_a_changed_guard_byte(bc_lib):
    assert bc_lib.VshipExt_BoundsCheckProbe(0) == abi.NoError
    assert bc_lib.VshipExt_BoundsCheckProbe(1) == abi.HIPError


def _frames(fmt, w, h, seed):
    if fmt == "generic":
        case = dict(name="bc", metric="ssimu2", w=w, h=h, seed=seed, step=12.0, sample=abi.SampleUINT12,
                    range=abi.RangeFull, subw=2, subh=1, loc=abi.ChromaLoc_TopLeft, matrix=abi.MATRIX_BT470_BG,
                    trc=abi.TRC_BT470_BG, prim=abi.PRIMARIES_BT470_BG, family=abi.ColorYUV, pad=[3, 5, 7])
        (p1, ls, cs), (p2, _, _) = build_case(case)
        return p1, p2, ls, cs
    p1, p2, ls = synth.make_pairs(1, w, h, fmt=fmt, seed=seed)[0]
    cs = abi.srgb8(w, h) if fmt == "rgb8" else abi.yuv420_10bit_bt709(w, h)
    return p1, p2, ls, cs


@pytest.mark.parametrize("fmt", ["rgb8", "yuv420p10", "generic"])
@pytest.mark.parametrize("size", SIZES, ids=lambda s: "%dx%d" % s)
def test_ssimu2_and_butteraugli_stay_in_bounds(bc_lib, fmt, size):
    import torch
    w, h = size
    p1, p2, ls, cs = _frames(fmt, w, h, seed=w * 3 + h)
    with api.SSIMU2(cs) as mine, api.SSIMU2(cs, lib=bc_lib) as bc:
        want = mine.compute(p1, p2, ls)
        got = bc.compute(p1, p2, ls)
        assert np.isfinite(got) and got == want, (got, want)
        d1 = [torch.from_numpy(np.ascontiguousarray(p).view(np.uint8).copy()).cuda() for p in p1]
        d2 = [torch.from_numpy(np.ascontiguousarray(p).view(np.uint8).copy()).cuda() for p in p2]
        score = torch.zeros(1, dtype=torch.float64, device="cuda")
        bc.compute_device(1, [t.data_ptr() for t in d1], [t.data_ptr() for t in d2], ls, ls, score.data_ptr(), 0, 0)
        torch.cuda.synchronize()
        assert score.item() == want
    with api.Butteraugli(cs, qnorm=5, intensity=203.0) as mine, \
            api.Butteraugli(cs, qnorm=5, intensity=203.0, lib=bc_lib) as bc:
        want, wmap = mine.compute(p1, p2, ls, distmap=True)
        got, gmap = bc.compute(p1, p2, ls, distmap=True)
        assert all(np.isfinite(got)) and tuple(got) == tuple(want), (got, want)
        assert np.array_equal(gmap, wmap)


def test_uneven_batch_stays_in_bounds(bc_lib):
    items, want = [], []
    for k, (w, h) in enumerate(SIZES):
        for fmt in ("rgb8", "yuv420p10", "generic"):
            p1, p2, ls, cs = _frames(fmt, w, h, seed=100 + k)
            items.append((cs, cs, p1, p2, ls, ls))
            with api.SSIMU2(cs) as mine:
                want.append(mine.compute(p1, p2, ls))
    b = api.SSIMU2Batch(lib=bc_lib)
    try:
        got = b.compute(items)
    finally:
        b.close()
    assert np.all(np.isfinite(got))
    np.testing.assert_array_equal(got, np.array(want))


@pytest.mark.parametrize("size", [(17, 9), (130, 98), (1921, 1081)], ids=lambda s: "%dx%d" % s)
def test_cvvdp_stays_in_bounds(bc_lib, size):
    w, h = size
    pairs = synth.make_pairs(3, w, h, fmt="yuv420p10", seed=w)
    cs = abi.yuv420_10bit_bt709(w, h)
    with api.CVVDP(cs, fps=24.0) as mine, api.CVVDP(cs, fps=24.0, lib=bc_lib) as bc:
        for p1, p2, ls in pairs:
            want = mine.compute(p1, p2, ls)
            got = bc.compute(p1, p2, ls)
            assert np.isfinite(got) and got == want, (got, want)

"""The reference's identity stress matrix on the GPU (test/libvshipTestIdentity.cpp:208-461).

Two copies of one random frame that differ only in their row padding must score exactly
SSIMULACRA2 100, Butteraugli inf-norm 0 and CVVDP JOD 10 (the reference's checks,
:357-384 and :416-456), across 7 sample types x 2 ranges x 6 chroma subsamplings x 4 chroma
sitings x 3 crops, on 720x480 and 1920x1080 frames, with and without a resize to 720x480.
The colourspace is the reference's: Y'CbCr family, RGB matrix, BT.709 transfer, XYZ
("internal") primaries.  Every plane row carries padding bytes (47 / 38 / 97, as the
reference) filled with different garbage in the two copies; beyond the reference, the unused
high bits of 9- to 14-bit samples also hold different garbage in the two copies, which the
decode must mask, and integer samples span their whole bit range (the reference draws only
0-3 for them).
"""
import itertools

import numpy as np
import pytest

from vship_b200 import abi, api

pytestmark = pytest.mark.gpu

SAMPLES = [abi.SampleFLOAT, abi.SampleUINT16, abi.SampleUINT14, abi.SampleUINT12, abi.SampleUINT10,
           abi.SampleUINT9, abi.SampleUINT8]
RANGES = [abi.RangeLimited, abi.RangeFull]
SUBSAMPLINGS = [(0, 0), (1, 0), (2, 0), (0, 1), (1, 1), (2, 1)]
SITINGS = [abi.ChromaLoc_Left, abi.ChromaLoc_Center, abi.ChromaLoc_Top, abi.ChromaLoc_TopLeft]
CROPS = [(0, 0, 0, 0), (10, 10, 10, 10), (1, 3, 5, 7)]
PADDING = (47, 38, 97)


def _pair(rng, cs):
    """Two copies of one random frame: same samples, different padding bytes and (for 9-14
    bit samples) different garbage in the unused high bits."""
    bits = abi.SAMPLE_BITS.get(cs.sample)
    planes = [[], []]
    ls = []
    for (pw, ph), pad in zip(cs.plane_dims(), PADDING):
        if cs.sample == abi.SampleFLOAT:
            vals = rng.random((ph, pw), dtype=np.float32)
            raw = [vals.view(np.uint8).reshape(ph, -1)] * 2
        elif cs.sample == abi.SampleUINT8:
            vals = rng.integers(0, 256, (ph, pw), dtype=np.uint8)
            raw = [vals, vals]
        else:
            vals = rng.integers(0, 1 << bits, (ph, pw), dtype=np.uint16)
            raw = []
            for _ in range(2):
                junk = (rng.integers(0, 1 << 16, (ph, pw), dtype=np.uint16) >> bits) << bits if bits < 16 else 0
                raw.append((vals | junk).astype(np.uint16).view(np.uint8).reshape(ph, -1))
        row = raw[0].shape[1]
        for k in range(2):
            buf = rng.integers(0, 256, (ph, row + pad), dtype=np.uint8)
            buf[:, :row] = raw[k]
            planes[k].append(buf)
        ls.append(row + pad)
    return planes[0], planes[1], ls


def _colourspaces(w, h, target):
    for sample, rng_, (sw, sh), loc, crop in itertools.product(SAMPLES, RANGES, SUBSAMPLINGS, SITINGS, CROPS):
        tw, th = target
        yield abi.colorspace(w, h, sample=sample, range_=rng_, subw=sw, subh=sh, chroma_location=loc,
                             family=abi.ColorYUV, matrix=abi.MATRIX_RGB, transfer=abi.TRC_BT709,
                             primaries=abi.PRIMARIES_INTERNAL, target_width=tw, target_height=th, crop=crop)


def _describe(cs):
    return "sample=%d range=%d sub=%d/%d loc=%d crop=%s target=%dx%d size=%dx%d" % (
        cs.sample, cs.range, cs.subsampling.subw, cs.subsampling.subh, cs.chromaLocation,
        (cs.crop.top, cs.crop.bottom, cs.crop.left, cs.crop.right), cs.target_width, cs.target_height, cs.width, cs.height)


SIZES = [((720, 480), (-1, -1)), ((720, 480), (720, 480)), ((1920, 1080), (-1, -1)), ((1920, 1080), (720, 480))]


@pytest.mark.parametrize("size,target", SIZES, ids=["720x480", "720x480_target720x480", "1920x1080", "1920x1080_to_720x480"])
def test_identity_ssimu2_and_butteraugli(gpu, size, target):
    rng = np.random.default_rng(size[0] * 7 + target[0])
    bad = []
    count = 0
    for cs in _colourspaces(size[0], size[1], target):
        p1, p2, ls = _pair(rng, cs)
        with api.SSIMU2(cs, cs) as h:
            s = h.compute(p1, p2, ls, ls)
        with api.Butteraugli(cs, cs, qnorm=5, intensity=165.0) as hb:
            norms, _ = hb.compute(p1, p2, ls, ls)
        count += 1
        if s != 100.0 or norms[2] != 0.0:
            bad.append((_describe(cs), s, norms[2]))
    assert count == 7 * 2 * 6 * 4 * 3
    assert not bad, bad[:10]


@pytest.mark.parametrize("size,target", [SIZES[0], SIZES[3]], ids=["720x480", "1920x1080_to_720x480"])
def test_identity_cvvdp(gpu, size, target):
    rng = np.random.default_rng(size[0] * 11 + target[0])
    bad = []
    for cs in _colourspaces(size[0], size[1], target):
        p1, p2, ls = _pair(rng, cs)
        with api.CVVDP(cs, cs, fps=48.0, resize_to_display=False, model="standard_hdr_pq") as hc:
            j = hc.compute(p1, p2, ls, ls)
        if j != 10.0:
            bad.append((_describe(cs), j))
    assert not bad, bad[:10]


def test_identity_batch_path(gpu):
    """The uneven-batch entry point on a mix of the matrix's colourspaces (no resize or crop,
    which the batch path leaves to handlers): every pair scores exactly 100."""
    rng = np.random.default_rng(5)
    items = []
    for cs in _colourspaces(720, 480, (-1, -1)):
        if cs.crop.top or cs.chromaLocation not in (abi.ChromaLoc_Left, abi.ChromaLoc_TopLeft):
            continue
        p1, p2, ls = _pair(rng, cs)
        items.append((cs, cs, p1, p2, ls, ls))
    b = api.SSIMU2Batch()
    try:
        scores = b.compute(items)
    finally:
        b.close()
    assert len(scores) == 7 * 2 * 6 * 2
    assert all(s == 100.0 for s in scores), [(i, s) for i, s in enumerate(scores) if s != 100.0][:10]

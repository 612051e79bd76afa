"""The compile-time 10-bit 4:2:0 BT.709 pixel path equals the generic path bit for bit.

Frames whose planes sit back to back in one host buffer keep the caller's strides on the
device.  Odd byte strides then make the view misaligned for 16-bit samples, which routes the
clip to the generic runtime-dispatched path: byte loads, and chroma interpolated pixel by
pixel. The same frames given as separate planes are copied densely and take the fast path.
That path reads 2x2 quads, shares chroma tap rows, and interpolates two columns with one
packed spline. The SSIMULACRA2 score, through the per-handler and batch entries, and the
CVVDP score and distortion map must not change by a single bit. Odd sizes cover quads
without a right column or a bottom row.
"""
import numpy as np
import pytest

from vship_b200 import abi, api, synth

pytestmark = pytest.mark.gpu

SIZES = [(97, 61), (66, 34), (333, 211), (1281, 721)]
ODD_PADS = [3, 1, 5]


def _one_buffer(planes, line_sizes, pad):
    """The planes back to back in one buffer with rows padded by `pad` bytes; returns the
    buffer (keep it alive), the three plane addresses and the strides."""
    padded, strides = synth.with_padding(planes, line_sizes, pad)
    buf = np.concatenate([p.reshape(-1) for p in padded])
    off = np.cumsum([0] + [p.nbytes for p in padded])
    return buf, [buf.ctypes.data + int(off[i]) for i in range(3)], strides


@pytest.mark.parametrize("w,h", SIZES)
def test_ssimu2_fast_path_equals_generic_path(gpu, w, h):
    p1, p2, ls = synth.make_pairs(1, w, h, fmt="yuv420p10", seed=w + 7 * h)[0]
    cs = abi.yuv420_10bit_bt709(w, h)
    b1, q1, strides = _one_buffer(p1, ls, ODD_PADS)
    b2, q2, _ = _one_buffer(p2, ls, ODD_PADS)
    assert all(s % 2 for s in strides)
    with api.SSIMU2(cs) as hd:
        fast = hd.compute(p1, p2, ls)
        fast_features = hd.last_features()
        generic = hd.compute(q1, q2, strides)
        generic_features = hd.last_features()
    assert generic == fast
    np.testing.assert_array_equal(generic_features, fast_features)


def test_batch_fast_and_generic_classes_agree(gpu):
    items, keep = [], []
    for w, h in SIZES[:3]:
        p1, p2, ls = synth.make_pairs(1, w, h, fmt="yuv420p10", seed=3 * w + h)[0]
        cs = abi.yuv420_10bit_bt709(w, h)
        b1, q1, strides = _one_buffer(p1, ls, ODD_PADS)
        b2, q2, _ = _one_buffer(p2, ls, ODD_PADS)
        keep += [b1, b2]
        items.append((cs, cs, p1, p2, ls, ls))
        items.append((cs, cs, q1, q2, strides, strides))
    with api.SSIMU2Batch() as b:
        b.set_tile_rows(32)
        scores = b.compute(items)
    np.testing.assert_array_equal(scores[0::2], scores[1::2])


@pytest.mark.parametrize("w,h", [(97, 61), (333, 211)])
def test_cvvdp_fast_path_equals_generic_path(gpu, w, h):
    frames = synth.make_pairs(3, w, h, fmt="yuv420p10", seed=w * h)
    cs = abi.yuv420_10bit_bt709(w, h)
    with api.CVVDP(cs, fps=24.0) as fast_h, api.CVVDP(cs, fps=24.0) as generic_h:
        for p1, p2, ls in frames:
            s_fast, m_fast = fast_h.compute(p1, p2, ls, distmap=True)
            b1, q1, strides = _one_buffer(p1, ls, ODD_PADS)
            b2, q2, _ = _one_buffer(p2, ls, ODD_PADS)
            s_generic, m_generic = generic_h.compute(q1, q2, strides, distmap=True)
            assert s_generic == s_fast
            np.testing.assert_array_equal(m_generic, m_fast)

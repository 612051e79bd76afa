"""Seeded test cases shared by the golden-vector generator and the parity tests.

Each case is a small dict (committed in reference_vectors.json next to the scores the
reference library produced for it) from which build_case() regenerates the exact input
bytes.  Planes are synthesised directly in the code domain of the sample type (smooth
sinusoid fields + noise, distorted by 8x8 DCT quantisation), so every colourspace of the
ABI can be exercised without an encoder; rows may carry random padding bytes.
"""
import numpy as np

from vship_b200 import abi, synth


def _plane_field(rng, w, h):
    f = synth.sinusoid_field(rng, w, h, count=12, pmin=3.0, pmax=max(8.0, float(max(w, h))))
    f = (f - f.min()) / max(f.max() - f.min(), 1e-9)
    f = 0.08 + 0.84 * f + rng.normal(0.0, 0.01, size=f.shape)
    return np.clip(f, 0.0, 1.0)


def _encode(v, cs, chroma):
    """Values in [0, 1] -> stored samples of the colourspace."""
    s = cs.sample
    yuv_chroma = chroma and cs.colorFamily == abi.ColorYUV
    if s in (abi.SampleFLOAT, abi.SampleHALF):
        x = v - 0.5 if yuv_chroma else v
        return x.astype(np.float32 if s == abi.SampleFLOAT else np.float16)
    bits = abi.SAMPLE_BITS[s]
    if cs.range == abi.RangeFull:
        q = np.round(v * ((1 << bits) - 1))
    elif yuv_chroma:
        q = np.round((128.0 + 224.0 * (v - 0.5)) * (1 << (bits - 8)))
    else:
        q = np.round((16.0 + 219.0 * v) * (1 << (bits - 8)))
    q = np.clip(q, 0, (1 << bits) - 1)
    return q.astype(np.uint8 if bits == 8 else np.uint16)


def colorspace_of(case):
    return abi.colorspace(case["w"], case["h"], sample=case.get("sample", abi.SampleUINT8),
                          range_=case.get("range", abi.RangeFull), subw=case.get("subw", 0),
                          subh=case.get("subh", 0), chroma_location=case.get("loc", abi.ChromaLoc_Left),
                          family=case.get("family", abi.ColorRGB), matrix=case.get("matrix", abi.MATRIX_RGB),
                          transfer=case.get("trc", abi.TRC_sRGB), primaries=case.get("prim", abi.PRIMARIES_BT709),
                          target_width=case.get("tw", -1), target_height=case.get("th", -1),
                          crop=tuple(case.get("crop", (0, 0, 0, 0))))


def build_case(case):
    """-> ((planes1, line_sizes1, cs), (planes2, line_sizes2, cs))."""
    rng = np.random.default_rng(case["seed"])
    cs = colorspace_of(case)
    dims = cs.plane_dims()
    ref, dist = [], []
    for c, (pw, ph) in enumerate(dims):
        f = _plane_field(rng, pw, ph)
        d = synth.dct_quantize(f[None] * 255.0, case.get("step", 16.0))[0] / 255.0
        if case.get("identical"):
            d = f
        ref.append(_encode(f, cs, c != 0))
        dist.append(_encode(d, cs, c != 0))
    pad = case.get("pad", [0, 0, 0])
    out = []
    for planes in (ref, dist):
        ls = [p.shape[1] * p.itemsize for p in planes]
        if any(pad):
            padded, ls = synth.with_padding(planes, ls, pad, rng=np.random.default_rng(case["seed"] + 7))
            planes = padded
        else:
            planes = [np.ascontiguousarray(p).view(np.uint8).reshape(p.shape[0], -1) for p in planes]
        out.append((planes, ls, cs))
    return out[0], out[1]


S, B = "ssimu2", "butteraugli"
YUV = dict(family=abi.ColorYUV)

CASES = [
    # SSIMULACRA2: sizes
    dict(name="s_rgb8_64x48", metric=S, w=64, h=48, seed=1, step=12.0),
    dict(name="s_rgb8_17x9", metric=S, w=17, h=9, seed=2, step=20.0),
    dict(name="s_rgb8_1x1", metric=S, w=1, h=1, seed=3, step=20.0),
    dict(name="s_rgb8_2x3", metric=S, w=2, h=3, seed=4, step=20.0),
    dict(name="s_rgb8_333x201_pad", metric=S, w=333, h=201, seed=5, step=8.0, pad=[47, 38, 97]),
    dict(name="s_rgb8_1920x1080", metric=S, w=1920, h=1080, seed=6, step=16.0),
    dict(name="s_rgb8_1921x1081", metric=S, w=1921, h=1081, seed=7, step=24.0),
    # SSIMULACRA2: colourspaces
    dict(name="s_yuv420p10_bt709_1920x1080", metric=S, w=1920, h=1080, seed=8, step=16.0, sample=abi.SampleUINT10,
         range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Left, matrix=abi.MATRIX_BT709, trc=abi.TRC_BT709, **YUV),
    dict(name="s_yuv420p10_129x67", metric=S, w=129, h=67, seed=9, step=16.0, sample=abi.SampleUINT10,
         range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Left, matrix=abi.MATRIX_BT709, trc=abi.TRC_BT709, **YUV),
    dict(name="s_yuv422p8_center_170m", metric=S, w=150, h=90, seed=10, step=12.0, sample=abi.SampleUINT8,
         range=abi.RangeLimited, subw=1, subh=0, loc=abi.ChromaLoc_Center, matrix=abi.MATRIX_ST170_M, trc=abi.TRC_BT601,
         prim=abi.PRIMARIES_ST170_M, **YUV),
    dict(name="s_yuv410_topleft_12bit", metric=S, w=130, h=70, seed=11, step=12.0, sample=abi.SampleUINT12,
         range=abi.RangeFull, subw=2, subh=1, loc=abi.ChromaLoc_TopLeft, matrix=abi.MATRIX_BT470_BG,
         trc=abi.TRC_BT470_BG, prim=abi.PRIMARIES_BT470_BG, **YUV),
    dict(name="s_yuv411_center_9bit", metric=S, w=101, h=77, seed=12, step=12.0, sample=abi.SampleUINT9,
         range=abi.RangeLimited, subw=2, subh=0, loc=abi.ChromaLoc_Center, matrix=abi.MATRIX_BT709, trc=abi.TRC_BT470_M,
         prim=abi.PRIMARIES_BT470_M, pad=[3, 1, 5], **YUV),
    dict(name="s_yuv420_top_14bit_2020cl", metric=S, w=96, h=80, seed=13, step=12.0, sample=abi.SampleUINT14,
         range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Top, matrix=abi.MATRIX_BT2020_CL,
         trc=abi.TRC_ST240_M, prim=abi.PRIMARIES_BT2020, **YUV),
    dict(name="s_yuv444p16_2020ncl_pq", metric=S, w=120, h=72, seed=14, step=12.0, sample=abi.SampleUINT16,
         range=abi.RangeFull, matrix=abi.MATRIX_BT2020_NCL, trc=abi.TRC_PQ, prim=abi.PRIMARIES_BT2020, **YUV),
    dict(name="s_ictcp_pq_half", metric=S, w=88, h=60, seed=15, step=12.0, sample=abi.SampleHALF,
         range=abi.RangeFull, matrix=abi.MATRIX_BT2100_ICTCP, trc=abi.TRC_PQ, prim=abi.PRIMARIES_BT2020, **YUV),
    dict(name="s_yuv_hlg_float", metric=S, w=88, h=60, seed=16, step=12.0, sample=abi.SampleFLOAT,
         range=abi.RangeFull, matrix=abi.MATRIX_BT2020_NCL, trc=abi.TRC_HLG, prim=abi.PRIMARIES_BT2020, **YUV),
    dict(name="s_rgb_float_linear_xyz", metric=S, w=70, h=50, seed=17, step=12.0, sample=abi.SampleFLOAT,
         range=abi.RangeFull, trc=abi.TRC_Linear, prim=abi.PRIMARIES_INTERNAL),
    dict(name="s_rgb16_st428", metric=S, w=70, h=50, seed=18, step=12.0, sample=abi.SampleUINT16,
         range=abi.RangeFull, trc=abi.TRC_ST428, prim=abi.PRIMARIES_ST240_M, pad=[2, 2, 6]),
    dict(name="s_rgb8_limited_srgb", metric=S, w=64, h=64, seed=19, step=12.0, range=abi.RangeLimited),
    # SSIMULACRA2: resize and crop
    dict(name="s_resize_crop", metric=S, w=200, h=120, seed=20, step=16.0, tw=160, th=100, crop=[1, 3, 5, 7]),
    dict(name="s_crop_only", metric=S, w=120, h=90, seed=21, step=16.0, crop=[10, 10, 10, 10]),
    dict(name="s_upscale", metric=S, w=90, h=60, seed=22, step=16.0, tw=128, th=96),
    # Identity (reference test/libvshipTestIdentity.cpp)
    dict(name="s_identity_yuv420p10_pad", metric=S, w=720, h=480, seed=23, identical=True, sample=abi.SampleUINT10,
         range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Left, matrix=abi.MATRIX_RGB, trc=abi.TRC_BT709,
         prim=abi.PRIMARIES_INTERNAL, pad=[47, 38, 97], **YUV),
    # Butteraugli
    dict(name="b_rgb8_64x48", metric=B, w=64, h=48, seed=31, step=12.0, qnorm=5, intensity=203.0),
    dict(name="b_rgb8_17x9", metric=B, w=17, h=9, seed=32, step=20.0, qnorm=2, intensity=80.0),
    dict(name="b_rgb8_333x201_pad", metric=B, w=333, h=201, seed=33, step=8.0, qnorm=5, intensity=203.0, pad=[5, 9, 1]),
    dict(name="b_yuv420p10_256x144", metric=B, w=256, h=144, seed=34, step=16.0, qnorm=3, intensity=203.0,
         sample=abi.SampleUINT10, range=abi.RangeLimited, subw=1, subh=1, loc=abi.ChromaLoc_Left,
         matrix=abi.MATRIX_BT709, trc=abi.TRC_BT709, **YUV),
    dict(name="b_rgb8_640x360", metric=B, w=640, h=360, seed=35, step=24.0, qnorm=5, intensity=203.0),
    dict(name="b_rgb8_1920x1080", metric=B, w=1920, h=1080, seed=36, step=16.0, qnorm=5, intensity=203.0),
    dict(name="b_crop_resize", metric=B, w=200, h=120, seed=37, step=16.0, qnorm=2, intensity=203.0, tw=180, th=110,
         crop=[2, 2, 4, 4]),
    dict(name="b_identity_pad", metric=B, w=160, h=96, seed=38, identical=True, qnorm=5, intensity=165.0, pad=[7, 7, 7]),
]


def _variant(base, **over):
    c = dict(next(c for c in CASES if c["name"] == base))
    c.update(over)
    return c


# Every SSIMULACRA2-only colour path again at >= 60k pixels (where the reference's float
# drift is small) and as Butteraugli cases (no cancellation: the colour path is pinned to
# the reference's own outputs at 1e-5).
_COLOUR_PATHS = ["s_yuv422p8_center_170m", "s_yuv410_topleft_12bit", "s_yuv411_center_9bit",
                 "s_yuv420_top_14bit_2020cl", "s_yuv444p16_2020ncl_pq", "s_ictcp_pq_half", "s_yuv_hlg_float",
                 "s_rgb_float_linear_xyz", "s_rgb16_st428", "s_rgb8_limited_srgb"]
_SIZES = {"s_yuv411_center_9bit": (301, 221), "s_yuv410_topleft_12bit": (340, 200), "s_yuv422p8_center_170m": (352, 240)}
CASES += [_variant(n, name=n + "_big", seed=100 + k, w=_SIZES.get(n, (320, 240))[0], h=_SIZES.get(n, (320, 240))[1])
          for k, n in enumerate(_COLOUR_PATHS)]
CASES += [
    dict(name="s_resize_crop_big", metric=S, w=400, h=260, seed=120, step=16.0, tw=360, th=220, crop=[2, 4, 6, 8]),
    dict(name="s_crop_only_big", metric=S, w=340, h=240, seed=121, step=16.0, crop=[10, 10, 10, 10]),
    dict(name="s_upscale_big", metric=S, w=256, h=192, seed=122, step=16.0, tw=384, th=256),
]
CASES += [_variant(n, name="b" + n[1:], metric=B, seed=140 + k, w=128, h=96, qnorm=5 if k % 2 else 3,
                   intensity=203.0 if k % 3 else 80.0)
          for k, n in enumerate(_COLOUR_PATHS + ["s_crop_only"])]
CASES += [_variant("s_upscale", name="b_upscale", metric=B, seed=152, w=90, h=64, tw=128, th=96, qnorm=5, intensity=203.0)]

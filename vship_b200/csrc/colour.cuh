// Colour front-end shared by both metrics: raw planes of any Vship_Colorspace_t -> linear
// BT.709 RGB in FP32, one pixel at a time, fused into the consumers (the SSIMULACRA2 pyramid
// kernel and the Butteraugli opsin kernel) so the intermediate float planes the reference
// materialises (src/gpuColorToLinear/vshipColor.hpp:62-146) never touch HBM.
//
// Arithmetic follows the reference stage by stage, including its float/double promotions,
// so that results agree to float rounding:
//   sample decode      src/gpuColorToLinear/anyDepthToFloat.hpp:24-68
//   range              src/gpuColorToLinear/rangeToFull.hpp:24-55
//   chroma upsampling  src/gpuColorToLinear/chromaUpsample.hpp:28-247 (cubic Hermite)
//   Y'CbCr -> R'G'B'   src/gpuColorToLinear/YUVToLinRGB.hpp:7-163
//   transfer           src/gpuColorToLinear/transferToLinear.hpp:19-184
//   primaries          src/gpuColorToLinear/primaries.hpp:9-158
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

#include "../../include/VshipColor.h"

namespace vship {

// Per-clip conversion parameters, resolved on the host at Init.
struct ColourParams {
    int sample;          // Vship_Sample_t
    int bytes;           // bytes per stored sample
    unsigned mask;       // low-bit mask for 16-bit integer containers
    int misaligned;      // some stride is not a multiple of `bytes`: use byte loads
    float full_scale;    // full range: 1 / (2^bits - 1), or 1 for float/half
    float lim_scale;     // limited range: 1 / 2^(bits-8), or 256 for float/half
    int full_range;
    int yuv_chroma;      // planes 1 and 2 are chroma (YUV family)
    int subw, subh;
    int hcenter, vcenter;
    int matrix, trc, primaries;
    int skip_yuv;        // Linear transfer + RGB matrix: no Y'CbCr/transfer stage
    int64_t W, H;        // luma plane size
    int64_t cw, ch;      // chroma plane size
};

// Device view of one input image: three plane base pointers and byte strides.
struct RawImage {
    const uint8_t* p[3];
    int64_t stride[3];
};

__device__ __forceinline__ int64_t clamp64(int64_t v, int64_t lo, int64_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// PickValue + FullRange for one stored sample.
__device__ __forceinline__ float load_norm(const uint8_t* plane, int64_t stride, int64_t x, int64_t y,
                                           const ColourParams& cp, bool chroma) {
    const uint8_t* a = plane + y * stride + x * cp.bytes;
    float v;
    if (cp.sample == Vship_SampleUINT8) {
        v = (float)__ldg(a);
    } else if (cp.sample == Vship_SampleFLOAT) {
        if (cp.misaligned) {
            uint32_t u = (uint32_t)__ldg(a) | ((uint32_t)__ldg(a + 1) << 8) | ((uint32_t)__ldg(a + 2) << 16) | ((uint32_t)__ldg(a + 3) << 24);
            v = __uint_as_float(u);
        } else {
            v = __ldg(reinterpret_cast<const float*>(a));
        }
    } else {
        unsigned short u;
        if (cp.misaligned) u = (unsigned short)(__ldg(a) | (__ldg(a + 1) << 8));
        else u = __ldg(reinterpret_cast<const unsigned short*>(a));
        if (cp.sample == Vship_SampleHALF) v = __half2float(__ushort_as_half(u));
        else v = (float)(u & cp.mask);
    }
    // FullRange (rangeToFull.hpp:24-55) with the divisions applied as reciprocal products
    // (at most one rounding apart from the reference's quotients).
    if (cp.full_range) {
        v *= cp.full_scale;
        if (chroma) v -= 0.5f;
        return v;
    }
    v *= cp.lim_scale;
    return chroma ? (v - 128.f) * (1.0f / 224.f) : (v - 16.f) * (1.0f / 219.f);
}

// CubicHermitSplineInterpolator (src/gpuColorToLinear/resize.hpp:5-24).  Every rounding is
// spelled out, so the value does not depend on how the compiler fuses multiply-adds in the
// surrounding code: the per-pixel, quad and staged paths, which share some of these terms,
// give bit-identical samples.  Products by +-2 are exact, so fma(+-2, x, y) rounds exactly as
// y +- 2x does, in one instruction.  At t = 0 the result is p0 exactly.
__device__ __forceinline__ float hermite(float p0, float m0, float p1, float m1, float t) {
    const float v1 = __fadd_rn(__fmaf_rn(-2.f, p1, __fmaf_rn(2.f, p0, m0)), m1);
    const float v2 = __fsub_rn(__fmaf_rn(-2.f, m0, __fmaf_rn(3.f, p1, __fmul_rn(-3.f, p0))), m1);
    float r = __fmaf_rn(v1, t, v2);
    r = __fmaf_rn(r, t, m0);
    return __fmaf_rn(r, t, p0);
}

// hermite() on two independent lanes with packed FP32x2 arithmetic of sm_100: every lane
// takes hermite()'s operations in hermite()'s order (x - y as x + (-y), which rounds the
// same), so each lane equals the scalar call bit for bit.
__device__ __forceinline__ float2 hermite2(float2 p0, float2 m0, float2 p1, float2 m1, float t) {
    const float2 two = make_float2(2.f, 2.f), mtwo = make_float2(-2.f, -2.f);
    const float2 v1 = __fadd2_rn(__ffma2_rn(mtwo, p1, __ffma2_rn(two, p0, m0)), m1);
    const float2 v2 = __fadd2_rn(
        __ffma2_rn(mtwo, m0, __ffma2_rn(make_float2(3.f, 3.f), p1, __fmul2_rn(make_float2(-3.f, -3.f), p0))),
        make_float2(-m1.x, -m1.y));
    const float2 tt = make_float2(t, t);
    float2 r = __ffma2_rn(v1, tt, v2);
    r = __ffma2_rn(r, tt, m0);
    return __ffma2_rn(r, tt, p0);
}

// Central-difference tangent (b - a) / 2 of two lanes, rounded as the scalar expression.
__device__ __forceinline__ float2 tangent2(float2 a, float2 b) {
    return __fmul2_rn(__fadd2_rn(b, make_float2(-a.x, -a.y)), make_float2(0.5f, 0.5f));
}

// Output sample X of an axis decimated by 2^sub -> interval start i and fraction t.
// Co-sited (Left/Top) kernels put sample i at X = f*i; centred ones at X = f*i + (f-1)/2.
__device__ __forceinline__ void upsample_phase(int64_t X, int sub, int centered, int64_t& i, float& t) {
    if (sub == 0) { i = X; t = 0.f; return; }
    const int64_t f = (int64_t)1 << sub;
    if (!centered) {
        i = X >> sub;
        t = (float)(X & (f - 1)) / (float)f;
    } else {
        const int64_t off = X - f / 2;
        const int64_t q = off >= 0 ? (off >> sub) : -((-off + f - 1) >> sub);
        i = q;
        t = ((float)(off - q * f) + 0.5f) / (float)f;
    }
}

// Chroma plane c (1 or 2) upsampled to luma position (X, Y): horizontal Hermite on up to
// four clamped chroma rows, then vertical Hermite (the reference's two passes, fused).
__device__ __forceinline__ float chroma_at(const RawImage& im, int c, int64_t X, int64_t Y, const ColourParams& cp) {
    const bool chroma = cp.yuv_chroma != 0;
    const uint8_t* pl = im.p[c];
    const int64_t st = im.stride[c];
    if (cp.subw == 0 && cp.subh == 0) return load_norm(pl, st, X, Y, cp, chroma);
    int64_t ix, iy;
    float tx, ty;
    upsample_phase(X, cp.subw, cp.hcenter, ix, tx);
    upsample_phase(Y, cp.subh, cp.vcenter, iy, ty);
    const int64_t c0 = clamp64(ix - 1, 0, cp.cw - 1), c1 = clamp64(ix, 0, cp.cw - 1);
    const int64_t c2 = clamp64(ix + 1, 0, cp.cw - 1), c3 = clamp64(ix + 2, 0, cp.cw - 1);
    auto hrow = [&](int64_t r) -> float {
        if (cp.subw == 0) return load_norm(pl, st, X, r, cp, chroma);
        const float em1 = load_norm(pl, st, c0, r, cp, chroma);
        const float e0 = load_norm(pl, st, c1, r, cp, chroma);
        const float e1 = load_norm(pl, st, c2, r, cp, chroma);
        const float e2 = load_norm(pl, st, c3, r, cp, chroma);
        return hermite(e0, (e1 - em1) / 2, e1, (e2 - e0) / 2, tx);
    };
    if (cp.subh == 0) return hrow(Y);
    const float h0 = hrow(clamp64(iy - 1, 0, cp.ch - 1));
    const float h1 = hrow(clamp64(iy, 0, cp.ch - 1));
    const float h2 = hrow(clamp64(iy + 1, 0, cp.ch - 1));
    const float h3 = hrow(clamp64(iy + 2, 0, cp.ch - 1));
    return hermite(h1, (h2 - h0) / 2, h2, (h3 - h1) / 2, ty);
}

// Non-constant-luminance Y'CbCr -> R'G'B' (YUVToLinRGB.hpp:7-18).
// The three divisors are constants of the matrix; they are applied as reciprocal products.
__device__ __forceinline__ float3 ncl_to_rgb(float3 v, const float kr, const float kb) {
    const float kg = 1.f - kb - kr;
    const float us = 0.5f / (1.f - kb);
    const float vs = 0.5f / (1.f - kr);
    float3 r;
    r.x = (v.z + v.x * vs) * (1.0f / (vs * kr + 0.5f));
    r.z = (v.y + v.x * us) * (1.0f / (us * kb + 0.5f));
    r.y = (v.x - kr * r.x - kb * r.z) * (1.0f / kg);
    return r;
}

__device__ __forceinline__ float3 gamma_light(float3 v, int matrix) {
    switch (matrix) {
    case Vship_MATRIX_BT709: return ncl_to_rgb(v, 0.2126f, 0.0722f);
    case Vship_MATRIX_BT470_BG:
    case Vship_MATRIX_ST170_M: return ncl_to_rgb(v, 0.299f, 0.114f);
    case Vship_MATRIX_BT2020_NCL: return ncl_to_rgb(v, 0.2627f, 0.0593f);
    case Vship_MATRIX_BT2020_CL: {
        const float kr = 0.2627f, kb = 0.0593f;
        const float us = 0.5f / (1.f - kb), vs = 0.5f / (1.f - kr);
        float3 r;
        r.x = (v.z + v.x * vs) / (vs * kr + 0.5f);
        r.z = (v.y + v.x * us) / (us * kb + 0.5f);
        r.y = v.x;
        return r;
    }
    case Vship_MATRIX_BT2100_ICTCP:
        v.x = fmaf(v.y, 0.0086090370379327566f, fmaf(v.z, 0.11102962500302595655f, v.x));
        v.y = fmaf(v.y, -0.01721807407586551f, fmaf(v.z, -0.22205925000605192f, v.x));
        v.z = fmaf(v.x, 33.025782688766114f, fmaf(v.y, -32.025782688766114f, -v.z * 7.543278084714549f));
        return v;
    default: return v;
    }
}

__device__ __forceinline__ float3 linear_light(float3 v, int matrix) {
    if (matrix == Vship_MATRIX_BT2020_CL) {
        const float kr = 0.2627f, kb = 0.0593f, kg = 1.f - kr - kb;
        v.y = (v.y - kr * v.x - kb * v.z) / kg;
    } else if (matrix == Vship_MATRIX_BT2100_ICTCP) {
        v.x = fmaf(v.x, 3.4366066943330784267f, fmaf(v.y, -2.5064521186562698975f, v.z * 0.069845424323191470954f));
        v.y = fmaf(v.x, -0.23026480071281397f, fmaf(v.y, 1.4064527541936944f, -v.z * 0.2083538389058436f));
        v.z = fmaf(v.x, -0.02684381778741865f, fmaf(v.y, -0.08378524945770065f, (float)((double)v.z * 1.106879231557486)));
    }
    return v;
}

// |a|^g with the sign of a, as exp2(g * log2|a|) on the special-function unit.  The relative
// error is ~3e-7 (log2 to 2^-21, exp2 to 2 ulp, times g), far below the metric's
// resolution; pow's exact corner cases are not needed for finite pixel values.
// 2^x on the special-function unit (PTX ex2.approx: relative error below 2^-22; results
// below 2^-126 flush to zero).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// log2 on the special-function unit without the subnormal-input fix-up (PTX
// lg2.approx.ftz: a subnormal input reads as 0 and gives -inf; normal inputs give the same
// value as lg2.approx).
__device__ __forceinline__ float lg2_ftz(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// x^g for x > 0 (0 otherwise) as exp2(g log2 x).  Every caller passes g >= 1, where a
// subnormal x gives 0 through the flushed log2 (-inf) just as through the exact one (the
// power underflows and exp2 flushes it), or an x that is never subnormal (sRGB above its
// knee, ST 240 above 0.0228); so the flushed log2 gives the same values with fewer
// instructions.
__device__ __forceinline__ float fast_pow(float x, float g) { return x > 0.f ? ex2_approx(g * lg2_ftz(x)) : 0.f; }
__device__ __forceinline__ float signed_powf(float a, float g) {
    const float r = fast_pow(fabsf(a), g);  // one power for either sign
    return a < 0 ? -r : r;
}

__device__ __forceinline__ float trc_one(float a, int trc) {
    switch (trc) {
    case Vship_TRC_sRGB:
        if (a < 0) {
            if (a < -0.04045f) return -fast_pow((-a + 0.055f) * (1.0f / 1.055f), 2.4f);
            return a * (1.0f / 12.92f);
        }
        if (a > 0.04045f) return fast_pow((a + 0.055f) * (1.0f / 1.055f), 2.4f);
        return a * (1.0f / 12.92f);
    case Vship_TRC_BT709: return signed_powf(a, 2.4f);
    case Vship_TRC_BT470_M: return signed_powf(a, 2.2f);
    case Vship_TRC_BT470_BG:
    case Vship_TRC_BT601: return signed_powf(a, 2.8f);
    case Vship_TRC_ST240_M:
        if (a >= 0) return a < 0.0228f ? 4 * a : 1.1115f * fast_pow(a, 0.45f) - 0.1115f;
        return a > -0.0228f ? 4 * a : -1.1115f * fast_pow(-a, 0.45f) + 0.1115f;
    case Vship_TRC_ST428: return signed_powf(a, 2.6f) * (float)(52.37 / 48.);
    case Vship_TRC_PQ: {
        // Evaluated in FP64: the EOTF subtracts c1 from a value near it and then raises to
        // 1/n ~ 6.3, which turns FP32 rounding into ~1e-3 score errors on dark content.
        const double m = 78.843750000000000, n = 0.15930175781250000;
        const double c1 = 0.83593750000000000, c2 = 18.851562500000000, c3 = 18.687500000000000;
        double x = fmax(0.0, (double)a);
        x = pow(x, 1.0 / m);
        return (float)(100.0 * pow(fmax(0.0, x - c1) / (c2 - c3 * x), 1.0 / n));
    }
    default: return a;
    }
}

__device__ __forceinline__ float3 transfer(float3 v, int trc) {
    if (trc == Vship_TRC_HLG) {
        // Inverse OETF and OOTF of HLG, in FP64 for the same reason as PQ.
        const double a = 0.17883277, b = 1.0 - 4.0 * a, c = 0.5 - a * -0.3350097945111627;
        double x = v.x, y = v.y, z = v.z;
        x = x <= 0.5 ? x * x / 3.0 : (exp((x - c) / a) + b) / 12.0;
        y = y <= 0.5 ? y * y / 3.0 : (exp((y - c) / a) + b) / 12.0;
        z = z <= 0.5 ? z * z / 3.0 : (exp((z - c) / a) + b) / 12.0;
        const double ys = 0.2627 * x + 0.6780 * y + 0.0593 * z;
        const double s = pow(ys, 1.2 - 1.0);
        return make_float3((float)(x * s), (float)(y * s), (float)(z * s));
    }
    v.x = trc_one(v.x, trc);
    v.y = trc_one(v.y, trc);
    v.z = trc_one(v.z, trc);
    return v;
}

__device__ __forceinline__ float3 mat3f(float3 a, float m0, float m1, float m2, float m3, float m4, float m5,
                                        float m6, float m7, float m8) {
    float3 r;
    r.x = fmaf(a.x, m0, fmaf(a.y, m1, a.z * m2));
    r.y = fmaf(a.x, m3, fmaf(a.y, m4, a.z * m5));
    r.z = fmaf(a.x, m6, fmaf(a.y, m7, a.z * m8));
    return r;
}

// Any supported primaries -> BT.709, through XYZ except for the direct BT.2020 matrix.
__device__ __forceinline__ float3 primaries_to_709(float3 v, int prim) {
    switch (prim) {
    case Vship_PRIMARIES_BT709: return v;
    case Vship_PRIMARIES_BT2020:
        return mat3f(v, 1.6605f, -0.5876f, -0.0728f, -0.1246f, 1.1329f, -0.0083f, -0.0182f, -0.1006f, 1.1187f);
    case Vship_PRIMARIES_ST170_M:
    case Vship_PRIMARIES_ST240_M:
        v = mat3f(v, 0.39349893f, 0.3652766f, 0.19162447f, 0.2123645f, 0.70109542f, 0.08654008f, 0.01873804f, 0.1119396f, 0.95812235f);
        break;
    case Vship_PRIMARIES_BT470_BG:
        v = mat3f(v, 0.4305f, 0.3416f, 0.1783f, 0.2220f, 0.7067f, 0.07132f, 0.0202f, 0.1296f, 0.9391f);
        break;
    case Vship_PRIMARIES_BT470_M:
        v = mat3f(v, 0.6068f, 0.1735f, 0.2003f, 0.2989f, 0.5866f, 0.1145f, 0.f, 0.06609f, 1.116f);
        break;
    default: break;  // INTERNAL: already XYZ
    }
    return mat3f(v, 3.2410f, -1.5374f, -0.4986f, -0.9692f, 1.8760f, 0.0416f, 0.0556f, -0.2040f, 1.0570f);
}

// ---------------------------------------------------------------------------------------
// Tile-staged chroma: a CTA working on luma tile [X0, X0+64) x [Y0, Y0+64) decodes each
// chroma sample it needs once, with the edge replication of the reference's clamped
// interpolators baked in (into shared memory S, or, on the 10-bit 4:2:0 path, into registers
// shared within a warp by shuffles), interpolates horizontally once per (chroma row, luma
// column) into HH, and every pixel then does only the vertical step.  Interval starts and
// fractions of the tile's 64 columns and rows come from small phase tables.
// ---------------------------------------------------------------------------------------
constexpr int kStageTile = 64;
// Front paths (see fast_path_of): the generic runtime-dispatched one and two compile-time ones.
constexpr int kFastGeneric = 0, kFastYuv420Bt709 = 1, kFastRgb8Srgb = 2;
constexpr int kStageMaxSpan = kStageTile + 4;  // staged rows/columns: interval range + 3 taps

struct ChromaStage {
    int cx_lo, cx_n;     // staged chroma columns [cx_lo, cx_lo + cx_n) (may start below 0)
    int cy_lo, cy_n;     // staged chroma rows
    float* S;            // [2][cy_n][kStageMaxSpan] decoded, range-normalised samples (not
                         // used by the 10-bit 4:2:0 path)
    float* HH;           // [2][cy_n][64] horizontally interpolated at each luma column
    short* hb;           // [64] S column of the first tap of luma column x
    float* ht;           // [64] horizontal fraction of luma column x
    short* vb;           // [64] HH row of the first tap of luma row y
    float* vt;           // [64] vertical fraction of luma row y
};

// Floats of shared memory chroma_stage() needs for a colourspace (0 when not subsampled).
__host__ __device__ inline int chroma_stage_floats(int subw, int subh) {
    if (subw == 0 && subh == 0) return 0;
    const int rows = subh ? (kStageTile >> subh) + 5 : kStageTile;
    return 2 * rows * kStageMaxSpan + 2 * rows * kStageTile + 4 * kStageTile;
}

// Interval start and fraction of output sample X on an axis decimated by 2^sub (int32).
__device__ __forceinline__ void phase32(int X, int sub, int centered, int& i, float& t) {
    if (sub == 0) { i = X; t = 0.f; return; }
    const int f = 1 << sub;
    if (!centered) {
        i = X >> sub;
        t = (float)(X & (f - 1)) * (1.0f / (float)f);
    } else {
        const int off = X - (f >> 1);
        i = off >> sub;  // arithmetic shift: floor division
        t = ((float)(off - (i << sub)) + 0.5f) * (1.0f / (float)f);
    }
}

// kFast names the front path: for 16-bit 4:2:0 samples (kFastYuv420Bt709) each thread owns
// one staged column and issues all its row loads before using any, so a tile waits for
// memory about once instead of once per row.  Both paths stage the same values.
template <int kFast = kFastGeneric>
__device__ __forceinline__ void chroma_stage(const RawImage& im, const ColourParams& cp, int X0, int Y0, float* smem,
                                             ChromaStage& st) {
    const int W = (int)cp.W, H = (int)cp.H, cw = (int)cp.cw, ch = (int)cp.ch;
    const int Xl = min(X0 + kStageTile - 1, W - 1), Yl = min(Y0 + kStageTile - 1, H - 1);
    int i0, i1;
    float t;
    if (cp.subw) {
        phase32(X0, cp.subw, cp.hcenter, i0, t);
        phase32(Xl, cp.subw, cp.hcenter, i1, t);
        st.cx_lo = i0 - 1;
        st.cx_n = i1 + 3 - st.cx_lo;
    } else {
        st.cx_lo = X0;
        st.cx_n = Xl - X0 + 1;
    }
    if (cp.subh) {
        phase32(Y0, cp.subh, cp.vcenter, i0, t);
        phase32(Yl, cp.subh, cp.vcenter, i1, t);
        st.cy_lo = i0 - 1;
        st.cy_n = i1 + 3 - st.cy_lo;
    } else {
        st.cy_lo = Y0;
        st.cy_n = Yl - Y0 + 1;
    }
    st.S = smem;
    st.HH = st.S + 2 * st.cy_n * kStageMaxSpan;
    st.ht = st.HH + 2 * st.cy_n * kStageTile;
    st.vt = st.ht + kStageTile;
    st.hb = reinterpret_cast<short*>(st.vt + kStageTile);
    st.vb = st.hb + kStageTile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    if (tid < kStageTile) {
        int i;
        float f;
        phase32(X0 + tid, cp.subw, cp.hcenter, i, f);
        st.hb[tid] = (short)(cp.subw ? i - 1 - st.cx_lo : i - st.cx_lo);
        st.ht[tid] = f;
    } else if (tid < 2 * kStageTile) {
        int i;
        float f;
        phase32(Y0 + tid - kStageTile, cp.subh, cp.vcenter, i, f);
        st.vb[tid - kStageTile] = (short)(cp.subh ? i - 1 - st.cy_lo : i - st.cy_lo);
        st.vt[tid - kStageTile] = f;
    }
    const bool chroma = cp.yuv_chroma != 0;
    if constexpr (kFast == kFastYuv420Bt709) {
        // Aligned 16-bit samples, co-sited columns (X0 is a multiple of 64): luma columns 2u and
        // 2u + 1 both start at staged column u with fractions 0 and 1/2, and at fraction 0 the
        // spline returns its first node exactly (finite samples, never -0).  Lane u of a warp
        // holds staged samples u and, for u < 3, 32 + u of each of its rows; it reads samples
        // u + 1 .. u + 3 from its neighbours by shuffles and writes HH columns (2u, 2u + 1) as
        // one pair.  Raw samples never pass through shared memory, and all of a warp's row
        // loads are issued before any is used.
        constexpr int kRowsPerWarp = 10;  // 2 x 37 staged rows over 8 warps
        const int rows = 2 * st.cy_n;
        const int gx_lo = min(max(st.cx_lo + lane, 0), cw - 1);
        const int gx_hi = min(max(st.cx_lo + 32 + min(lane, 2), 0), cw - 1);
        for (int base = warp; base < rows; base += nwarps * kRowsPerWarp) {
            unsigned lo[kRowsPerWarp], hi[kRowsPerWarp];
#pragma unroll
            for (int k = 0; k < kRowsPerWarp; k++) {
                const int r = base + k * nwarps;
                lo[k] = hi[k] = 0u;
                if (r < rows) {
                    const int p = r >= st.cy_n, rr = r - p * st.cy_n;
                    const int gy = min(max(st.cy_lo + rr, 0), ch - 1);
                    const unsigned short* src =
                        reinterpret_cast<const unsigned short*>(im.p[1 + p] + (int64_t)gy * im.stride[1 + p]);
                    lo[k] = __ldg(src + gx_lo);
                    hi[k] = __ldg(src + gx_hi);
                }
            }
#pragma unroll
            for (int k = 0; k < kRowsPerWarp; k++) {
                const int r = base + k * nwarps;
                if (r >= rows) break;  // the same for every lane of the warp
                float a = (float)(lo[k] & cp.mask), b = (float)(hi[k] & cp.mask);
                // FullRange of a chroma sample, as load_norm computes it.
                if (cp.full_range) {
                    a = a * cp.full_scale - 0.5f;
                    b = b * cp.full_scale - 0.5f;
                } else {
                    a = (a * cp.lim_scale - 128.f) * (1.0f / 224.f);
                    b = (b * cp.lim_scale - 128.f) * (1.0f / 224.f);
                }
                float e[4];
                e[0] = a;
#pragma unroll
                for (int d = 1; d < 4; d++) {
                    const int src_lane = (lane + d) & 31;
                    const float va = __shfl_sync(0xffffffffu, a, src_lane);
                    const float vb = __shfl_sync(0xffffffffu, b, src_lane);
                    e[d] = lane + d < 32 ? va : vb;
                }
                const float odd = hermite(e[1], (e[2] - e[0]) / 2, e[2], (e[3] - e[1]) / 2, 0.5f);
                *reinterpret_cast<float2*>(st.HH + r * kStageTile + 2 * lane) = make_float2(e[1], odd);
            }
        }
        __syncthreads();
        return;
    } else {
        for (int r = warp; r < 2 * st.cy_n; r += nwarps) {
            const int p = r >= st.cy_n, rr = r - p * st.cy_n;
            const int gy = min(max(st.cy_lo + rr, 0), ch - 1);
            for (int c = lane; c < st.cx_n; c += 32) {
                const int gx = min(max(st.cx_lo + c, 0), cw - 1);
                st.S[r * kStageMaxSpan + c] = load_norm(im.p[1 + p], im.stride[1 + p], gx, gy, cp, chroma);
            }
        }
    }
    __syncthreads();
    for (int r = warp; r < 2 * st.cy_n; r += nwarps) {
        const float* row = st.S + r * kStageMaxSpan;
        for (int x = lane; x < kStageTile; x += 32) {
            const int j = st.hb[x];
            float v;
            if (cp.subw) {
                const float em1 = row[j], e0 = row[j + 1], e1 = row[j + 2], e2 = row[j + 3];
                v = hermite(e0, (e1 - em1) / 2, e1, (e2 - e0) / 2, st.ht[x]);
            } else {
                v = row[min(j, st.cx_n - 1)];
            }
            st.HH[r * kStageTile + x] = v;
        }
    }
    __syncthreads();
}

// Both chroma values at tile-local luma (x, y) of a tile prepared by chroma_stage.
__device__ __forceinline__ float2 chroma_from_stage(const ChromaStage& st, const ColourParams& cp, int x, int y) {
    const int nh = st.cy_n * kStageTile;
    const int j = st.vb[y];
    if (!cp.subh) return make_float2(st.HH[j * kStageTile + x], st.HH[nh + j * kStageTile + x]);
    const float t = st.vt[y];
    float out[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const float* col = st.HH + p * nh + j * kStageTile + x;
        const float h0 = col[0], h1 = col[kStageTile], h2 = col[2 * kStageTile], h3 = col[3 * kStageTile];
        out[p] = hermite(h1, (h2 - h0) / 2, h2, (h3 - h1) / 2, t);
    }
    return make_float2(out[0], out[1]);
}

// ICtCp (BT.2100) to linear RGB in FP64: I'Ct'Cp' -> L'M'S' (YUVToLinRGB.hpp:47-63), the
// transfer, LMS -> RGB (:28-43), with the reference's sequential substitutions.  Both
// matrices subtract nearly equal terms (S' = 33.03 L' - 32.03 M' - 7.54 Cp, R = 3.44 L -
// 2.51 M + ...), and PQ raises (V^(1/m) - c1) to 1/n ~ 6.3, so FP32 rounding anywhere in
// this chain reaches ~1e-4 of the linear value of dark pixels and moves Butteraugli norms by
// a few 1e-4.  Only ICtCp clips take this path.
static __device__ __noinline__ float3 ictcp_to_linear(float3 in, int trc) {
    const double I = in.x, Ct = in.y, Cp = in.z;
    double v[3];
    v[0] = fma(Ct, 0.0086090370379327566, fma(Cp, 0.11102962500302595655, I));
    v[1] = fma(Ct, -0.01721807407586551, fma(Cp, -0.22205925000605192, v[0]));
    v[2] = fma(v[0], 33.025782688766114, fma(v[1], -32.025782688766114, -Cp * 7.543278084714549));
    if (trc == Vship_TRC_PQ) {
        const double m = 78.843750000000000, n = 0.15930175781250000;
        const double c1 = 0.83593750000000000, c2 = 18.851562500000000, c3 = 18.687500000000000;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double x = pow(fmax(0.0, v[k]), 1.0 / m);
            v[k] = 100.0 * pow(fmax(0.0, x - c1) / (c2 - c3 * x), 1.0 / n);
        }
    } else if (trc == Vship_TRC_HLG) {
        const double a = 0.17883277, b = 1.0 - 4.0 * a, c = 0.5 - a * -0.3350097945111627;
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = v[k] <= 0.5 ? v[k] * v[k] / 3.0 : (exp((v[k] - c) / a) + b) / 12.0;
        const double s = pow(0.2627 * v[0] + 0.6780 * v[1] + 0.0593 * v[2], 1.2 - 1.0);
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] *= s;
    } else {
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = (double)trc_one((float)v[k], trc);
    }
    const double L = v[0], M = v[1], S = v[2];
    const double R = fma(L, 3.4366066943330784267, fma(M, -2.5064521186562698975, S * 0.069845424323191470954));
    const double G = fma(R, -0.23026480071281397, fma(M, 1.4064527541936944, -S * 0.2083538389058436));
    const double B = fma(R, -0.02684381778741865, fma(G, -0.08378524945770065, S * 1.106879231557486));
    return make_float3((float)R, (float)G, (float)B);
}

// Y'CbCr (or R'G'B') -> linear RGB of one pixel in the clip's own primaries (the
// reference's linRGB destination, src/gpuColorToLinear/vshipColor.hpp:111-113).
__device__ __forceinline__ float3 to_linear_native(float3 v, const ColourParams& cp) {
    if (cp.matrix == Vship_MATRIX_BT2100_ICTCP && !cp.skip_yuv) return ictcp_to_linear(v, cp.trc);
    if (!cp.skip_yuv) {
        v = gamma_light(v, cp.matrix);
        v = transfer(v, cp.trc);
        v = linear_light(v, cp.matrix);
    }
    return v;
}

// Y'CbCr (or R'G'B') -> linear BT.709 RGB of one pixel.
__device__ __forceinline__ float3 to_linear_709(float3 v, const ColourParams& cp) {
    return primaries_to_709(to_linear_native(v, cp), cp.primaries);
}

// Linear RGB in primaries `prim` -> CIE XYZ (primariesToPrimaries_device<P, INTERNAL>,
// src/gpuColorToLinear/primaries.hpp:17-112).
__device__ __forceinline__ float3 rgb_to_xyz(float3 v, int prim) {
    switch (prim) {
    case Vship_PRIMARIES_BT709:
        return mat3f(v, 0.4124f, 0.3576f, 0.1805f, 0.2126f, 0.7152f, 0.0722f, 0.0193f, 0.1192f, 0.9505f);
    case Vship_PRIMARIES_BT2020:
        return mat3f(v, 0.6370f, 0.1446f, 0.1689f, 0.2627f, 0.6780f, 0.0593f, 0.f, 0.0281f, 1.0610f);
    case Vship_PRIMARIES_ST170_M:
    case Vship_PRIMARIES_ST240_M:
        return mat3f(v, 0.39349893f, 0.3652766f, 0.19162447f, 0.2123645f, 0.70109542f, 0.08654008f, 0.01873804f, 0.1119396f, 0.95812235f);
    case Vship_PRIMARIES_BT470_BG:
        return mat3f(v, 0.4305f, 0.3416f, 0.1783f, 0.2220f, 0.7067f, 0.07132f, 0.0202f, 0.1296f, 0.9391f);
    case Vship_PRIMARIES_BT470_M:
        return mat3f(v, 0.6068f, 0.1735f, 0.2003f, 0.2989f, 0.5866f, 0.1145f, 0.f, 0.06609f, 1.116f);
    default:
        return v;  // INTERNAL: already XYZ
    }
}

// Linear RGB of luma (X, Y) inside the tile with origin (X0, Y0) prepared by chroma_stage
// (or of any pixel when the clip is not chroma-subsampled): BT.709 primaries, or the clip's
// own primaries when kNative.
template <bool kNative = false>
__device__ __forceinline__ float3 ingest_staged(const RawImage& im, const ColourParams& cp, const ChromaStage& st,
                                               int X, int Y, int X0, int Y0) {
    float3 v;
    v.x = load_norm(im.p[0], im.stride[0], X, Y, cp, false);
    if (cp.subw == 0 && cp.subh == 0) {
        const bool chroma = cp.yuv_chroma != 0;
        v.y = load_norm(im.p[1], im.stride[1], X, Y, cp, chroma);
        v.z = load_norm(im.p[2], im.stride[2], X, Y, cp, chroma);
    } else {
        const float2 c = chroma_from_stage(st, cp, X - X0, Y - Y0);
        v.y = c.x;
        v.z = c.y;
    }
    return kNative ? to_linear_native(v, cp) : to_linear_709(v, cp);
}

// Linear BT.709 RGB of luma position (X, Y) of one raw image.
__device__ __forceinline__ float3 ingest_pixel(const RawImage& im, int64_t X, int64_t Y, const ColourParams& cp) {
    float3 v;
    v.x = load_norm(im.p[0], im.stride[0], X, Y, cp, false);
    v.y = chroma_at(im, 1, X, Y, cp);
    v.z = chroma_at(im, 2, X, Y, cp);
    return to_linear_709(v, cp);
}

// ---------------------------------------------------------------------------------------
// Compile-time specialised pixel paths for the two most common clip formats; every other
// colourspace takes the generic runtime-dispatched path above.  Results are identical to the
// generic path (same operations in the same order), only the dispatch is resolved at compile
// time.
//   kFastYuv420Bt709: 16-bit containers, 4:2:0, Left siting, BT.709 matrix, transfer, primaries
//   kFastRgb8Srgb:    8-bit R'G'B' 4:4:4, sRGB transfer, BT.709 primaries
// (kFastGeneric, kFastYuv420Bt709, kFastRgb8Srgb are declared before chroma_stage.)
// ---------------------------------------------------------------------------------------

__host__ __device__ inline int fast_path_of(const ColourParams& cp) {
    const bool u16 = cp.sample != Vship_SampleUINT8 && cp.sample != Vship_SampleFLOAT && cp.sample != Vship_SampleHALF;
    if (u16 && !cp.misaligned && cp.subw == 1 && cp.subh == 1 && !cp.hcenter && cp.vcenter && cp.yuv_chroma &&
        cp.matrix == Vship_MATRIX_BT709 && cp.trc == Vship_TRC_BT709 && cp.primaries == Vship_PRIMARIES_BT709)
        return kFastYuv420Bt709;
    if (cp.sample == Vship_SampleUINT8 && cp.subw == 0 && cp.subh == 0 && !cp.yuv_chroma && cp.matrix == Vship_MATRIX_RGB &&
        cp.trc == Vship_TRC_sRGB && cp.primaries == Vship_PRIMARIES_BT709)
        return kFastRgb8Srgb;
    return kFastGeneric;
}

__device__ __forceinline__ float srgb_to_linear(float a) {
    if (a < 0) return a < -0.04045f ? -fast_pow((-a + 0.055f) * (1.0f / 1.055f), 2.4f) : a * (1.0f / 12.92f);
    return a > 0.04045f ? fast_pow((a + 0.055f) * (1.0f / 1.055f), 2.4f) : a * (1.0f / 12.92f);
}

__device__ __forceinline__ float range_luma(float v, const ColourParams& cp) {
    if (cp.full_range) return v * cp.full_scale;
    return (v * cp.lim_scale - 16.f) * (1.0f / 219.f);
}

template <int kFast>
__device__ __forceinline__ float3 ingest_fast(const RawImage& im, const ColourParams& cp, const ChromaStage& st, int X, int Y,
                                             int X0, int Y0) {
    if constexpr (kFast == kFastYuv420Bt709) {
        const unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(im.p[0] + (int64_t)Y * im.stride[0]) + X);
        float3 v;
        v.x = range_luma((float)(u & cp.mask), cp);
        const float2 c = chroma_from_stage(st, cp, X - X0, Y - Y0);
        v.y = c.x;
        v.z = c.y;
        v = ncl_to_rgb(v, 0.2126f, 0.0722f);
        v.x = signed_powf(v.x, 2.4f);
        v.y = signed_powf(v.y, 2.4f);
        v.z = signed_powf(v.z, 2.4f);
        return v;
    } else {
        const int64_t o = (int64_t)Y * im.stride[0] + X;
        float3 v;
        v.x = srgb_to_linear(range_luma((float)__ldg(im.p[0] + o), cp));
        v.y = srgb_to_linear(range_luma((float)__ldg(im.p[1] + (int64_t)Y * im.stride[1] + X), cp));
        v.z = srgb_to_linear(range_luma((float)__ldg(im.p[2] + (int64_t)Y * im.stride[2] + X), cp));
        return v;
    }
}

// Linear RGB of the 2x2 luma quad at even (X, Y) of a kFastYuv420Bt709 tile with origin
// (X0, Y0) (also even); `right` / `down` say whether column X + 1 / row Y + 1 exist (the
// entries of missing pixels hold values read from in-bounds shared memory and must be
// ignored).  The values equal four ingest_fast calls: with vertically
// centred 4:2:0 chroma the two luma rows of a quad take chroma rows j .. j + 3 and
// j + 1 .. j + 4 (fractions 0.75 and 0.25), so each plane reads five shared tap rows, each
// as one 8-byte load covering both columns, and interpolates both columns of a luma row with
// one packed spline (hermite2).  Luma pairs are read as one 4-byte load when the row is
// 4-byte aligned.
__device__ __forceinline__ void ingest_quad_yuv420(const RawImage& im, const ColourParams& cp, const ChromaStage& st,
                                                   int X, int Y, int X0, int Y0, bool right, bool down, float3 q[4]) {
    const int x = X - X0, y = Y - Y0;
    float lum[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int r = 0; r < 2; r++) {
        if (r == 1 && !down) break;
        const unsigned short* row = reinterpret_cast<const unsigned short*>(im.p[0] + (int64_t)(Y + r) * im.stride[0]);
        unsigned short u0, u1 = 0;
        if (right && (reinterpret_cast<uintptr_t>(row + X) & 3u) == 0) {
            const ushort2 u = __ldg(reinterpret_cast<const ushort2*>(row + X));
            u0 = u.x;
            u1 = u.y;
        } else {
            u0 = __ldg(row + X);
            if (right) u1 = __ldg(row + X + 1);
        }
        lum[2 * r] = range_luma((float)(u0 & cp.mask), cp);
        lum[2 * r + 1] = range_luma((float)(u1 & cp.mask), cp);
    }
    const int nh = st.cy_n * kStageTile;
    const int j = st.vb[y];
    const float t0 = st.vt[y], t1 = st.vt[y + 1];
    float2 c[4];  // pixel (x, y) (x+1, y) (x, y+1) (x+1, y+1) -> (Cb, Cr)
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const float* col = st.HH + p * nh + j * kStageTile + x;
        float2 h[5];
#pragma unroll
        for (int k = 0; k < 4; k++) h[k] = *reinterpret_cast<const float2*>(col + k * kStageTile);
        h[4] = down ? *reinterpret_cast<const float2*>(col + 4 * kStageTile) : h[3];
        // Both columns at once: lane .x is column x, lane .y column x + 1.
        const float2 g1 = tangent2(h[0], h[2]), g2 = tangent2(h[1], h[3]), g3 = tangent2(h[2], h[4]);
        const float2 av = hermite2(h[1], g1, h[2], g2, t0);
        const float2 bv = hermite2(h[2], g2, h[3], g3, t1);
        const float a0 = av.x, a1 = av.y, b0 = bv.x, b1 = bv.y;
        if (p == 0) { c[0].x = a0; c[1].x = a1; c[2].x = b0; c[3].x = b1; }
        else        { c[0].y = a0; c[1].y = a1; c[2].y = b0; c[3].y = b1; }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float3 v = make_float3(lum[k], c[k].x, c[k].y);
        v = ncl_to_rgb(v, 0.2126f, 0.0722f);
        v.x = signed_powf(v.x, 2.4f);
        v.y = signed_powf(v.y, 2.4f);
        v.z = signed_powf(v.z, 2.4f);
        q[k] = v;
    }
}

}  // namespace vship

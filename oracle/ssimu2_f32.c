/*
 * ssimu2_f32.c -- FP32 restatement of the reference's own SSIMULACRA2 arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY, like oracle.c: the product never links, loads or calls it.
 *
 * oracle.c evaluates Vship's SSIMULACRA2 pipeline in double, which is the exact metric the
 * engine is held to.  The reference library evaluates the same pipeline in float, and its
 * SSIM map subtracts nearly equal float quantities (score.hpp:266-273), so its scores drift
 * from the exact metric by ~1e-3 at 1080p and by up to ~1 on frames of a few pixels.  This
 * file repeats that float arithmetic step for step -- same operand order, same roundings,
 * the same fused multiply-adds where the reference writes fmaf() or where nvcc contracts a
 * product into the following addition, the same zero-padded blur, the same per-block tree
 * sums and 1024-wide reduction passes, the same float feature vector -- so that the
 * reference's scores can be reproduced on the CPU and the drift shown to be rounding, not an
 * algorithm difference.  Transcendentals (powf, cbrtf, expf) go through one array hook:
 * evaluated in double and rounded to float by default, or by CUDA's own float functions on
 * the GPU when the tests install oracle/cuda_math.cu's evaluator (the only way to match the
 * reference bit for bit, since CUDA's results may differ from the correctly rounded ones in
 * the last bit and the tiniest frames amplify one such bit into a visible score change).
 *
 * Each function cites the reference file:line it follows.  Paths are relative to the
 * reference project (src/...).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/VshipColor.h"
#include "../vship_b200/csrc/metric_tables.h"

#define ORACLE_API __attribute__((visibility("default")))

/* Where the reference's source leaves it to the compiler, nvcc fuses a product into the
 * following addition or subtraction (its default -fmad=true).  Which product of a sum of two
 * products it fuses is not visible in the source; the forms below are the ones that reproduce
 * the reference's outputs bit for bit on every golden case: the Hermite spline's Horner steps
 * and its 3*p1 product (resize.hpp:9-22), the Y'CbCr numerators and the G row but not the
 * constant denominators (YUVToLinRGB.hpp:7-18, 66-94), c2 - c3*a of PQ (transferToLinear.hpp:
 * 181), HLG's Ys (:49), and s12 - m1*m2 and the SSIM denominator (score.hpp:262-268). */

static inline int64_t imin(int64_t a, int64_t b) { return a < b ? a : b; }
static inline int64_t imax(int64_t a, int64_t b) { return a > b ? a : b; }

/* The transcendentals the reference calls on the GPU, evaluated over arrays: op 0 is
 * powf(x[i], y), op 1 cbrtf(x[i]), op 2 expf(x[i]).  The default evaluates them in double and
 * rounds to float (the correctly rounded result).  oracle_f32_set_math installs another
 * evaluator; the tests install one that runs CUDA's own powf/cbrtf/expf (oracle/cuda_math.cu)
 * on the GPU, which makes every float of this file equal to the reference's. */
typedef void (*f32_math_fn)(int op, const float* x, float y, float* out, int64_t n);

static void math_cr(int op, const float* x, float y, float* out, int64_t n) {
    for (int64_t i = 0; i < n; i++) {
        if (op == 0) out[i] = (float)pow((double)x[i], (double)y);
        else if (op == 1) out[i] = (float)cbrt((double)x[i]);
        else out[i] = (float)exp((double)x[i]);
    }
}
static f32_math_fn g_math = math_cr;

ORACLE_API void oracle_f32_set_math(f32_math_fn fn) { g_math = fn ? fn : math_cr; }

enum { M_POW = 0, M_CBRT = 1, M_EXP = 2 };

/* ------------------------------------------------------------------------------------ */
/* Sample decode and range (anyDepthToFloat.hpp:24-80, rangeToFull.hpp:24-55)           */
/* ------------------------------------------------------------------------------------ */

static int f_sample_bytes(Vship_Sample_t s) {
    return s == Vship_SampleUINT8 ? 1 : (s == Vship_SampleFLOAT ? 4 : 2);
}

static int f_sample_bits(Vship_Sample_t s) {
    switch (s) {
    case Vship_SampleUINT8: return 8;
    case Vship_SampleUINT9: return 9;
    case Vship_SampleUINT10: return 10;
    case Vship_SampleUINT12: return 12;
    case Vship_SampleUINT14: return 14;
    case Vship_SampleUINT16: return 16;
    default: return 1;
    }
}

static float f_half(uint16_t h) {
    int sign = h >> 15, e = (h >> 10) & 31, m = h & 1023;
    float v;
    if (e == 0) v = ldexpf((float)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexpf((float)(m | 1024), e - 25);
    return sign ? -v : v;
}

static float f_pick(const uint8_t* plane, int64_t stride, int64_t x, int64_t y, Vship_Sample_t s) {
    const uint8_t* p = plane + y * stride + (int64_t)f_sample_bytes(s) * x;
    if (s == Vship_SampleUINT8) return (float)p[0];
    if (s == Vship_SampleFLOAT) { float f; memcpy(&f, p, 4); return f; }
    uint16_t raw = (uint16_t)(p[0] | (p[1] << 8));
    if (s == Vship_SampleHALF) return f_half(raw);
    return (float)(raw & ((1u << f_sample_bits(s)) - 1u));
}

/* FullRange (rangeToFull.hpp:24-55), in float. */
static float f_full_range(float a, Vship_Sample_t s, Vship_Range_t r, int chroma) {
    const int bd = f_sample_bits(s);
    if (r == Vship_RangeFull) {
        const float norm = (float)((1 << bd) - 1);
        a /= norm;
        if (chroma) a -= 0.5f;
        return a;
    }
    if (bd >= 8) a /= (float)(1 << (bd - 8));
    else a *= 256.0f;
    return chroma ? (a - 128.f) / 224.f : (a - 16.f) / 219.f;
}

/* ------------------------------------------------------------------------------------ */
/* Cubic Hermite interpolation (resize.hpp:5-24) and chroma upsampling                   */
/* (chromaUpsample.hpp:28-247)                                                            */
/* ------------------------------------------------------------------------------------ */

typedef struct { float v1, v2, v3, v4; } Herm;

static Herm herm_make(float p0, float m0, float p1, float m1) {
    Herm h;
    /* v1 = 2*p0 + m0 - 2*p1 + m1: the doublings are exact, so contraction cannot change it */
    h.v1 = ((2.f * p0 + m0) - 2.f * p1) + m1;
    /* v2 = -3*p0 + 3*p1 - 2*m0 - m1: nvcc rounds -3*p0 and fuses 3*p1 into the sum */
    const float t = fmaf(p1, 3.f, -3.f * p0);
    h.v2 = (t - 2.f * m0) - m1;
    h.v3 = m0;
    h.v4 = p0;
    return h;
}

/* get (resize.hpp:14-23): res = v1; res *= t; res += v2; ... as three fused steps. */
static float herm_get(Herm h, float t) { return fmaf(fmaf(fmaf(h.v1, t, h.v2), t, h.v3), t, h.v4); }

/* getHorizontalInterpolator_device / getVerticalInterpolator_device (:28-50): the four
 * samples around index i of a sequence of n, read through `at(k)`, edge-replicated. */
static Herm seq_interp(const float* base, int64_t step, int64_t n, int64_t i) {
    i = imin(i, n - 1);
    const float em1 = (i <= 0) ? base[0] : base[(i - 1) * step];
    const float e0 = (i < 0) ? em1 : base[i * step];
    const float e1 = (i >= n - 1) ? e0 : base[(i + 1) * step];
    const float e2 = (i >= n - 2) ? e1 : base[(i + 2) * step];
    return herm_make(e0, (e1 - em1) / 2.f, e1, (e2 - e0) / 2.f);
}

/* Horizontal pass of one row: small (sw samples) -> out (W samples). */
static void h_upsample_row(const float* small, int64_t sw, int64_t W, int sub, int centered, float* out) {
    if (!centered) {
        const int64_t f = (int64_t)1 << sub;
        for (int64_t x = 0; x < sw + 1; x++) {
            Herm h = seq_interp(small, 1, sw, x);
            if (f * x < W) out[f * x] = small[imin(x, sw - 1)];
            if (sub == 1) {
                if (2 * x + 1 < W) out[2 * x + 1] = herm_get(h, 0.5f);
            } else {
                if (4 * x + 1 < W) out[4 * x + 1] = herm_get(h, 0.25f);
                if (4 * x + 2 < W) out[4 * x + 2] = herm_get(h, 0.5f);
                if (4 * x + 3 < W) out[4 * x + 3] = herm_get(h, 0.75f);
            }
        }
    } else {
        for (int64_t x = -1; x < sw + 1; x++) {
            Herm h = seq_interp(small, 1, sw, x);
            if (sub == 1) {
                if (x != -1 && 2 * x + 1 < W) out[2 * x + 1] = herm_get(h, 0.25f);
                if (2 * x + 2 < W) out[2 * x + 2] = herm_get(h, 0.75f);
            } else {
                if (x != -1 && 4 * x + 2 < W) out[4 * x + 2] = herm_get(h, 0.125f);
                if (x != -1 && 4 * x + 3 < W) out[4 * x + 3] = herm_get(h, 0.375f);
                if (4 * x + 4 < W) out[4 * x + 4] = herm_get(h, 0.625f);
                if (4 * x + 5 < W) out[4 * x + 5] = herm_get(h, 0.875f);
            }
        }
    }
}

/* upsample (chromaUpsample.hpp:153-247) of one chroma plane dec (sw x sh) into out (W x H). */
static void f_upsample_plane(const float* dec, int64_t sw, int64_t sh, int64_t W, int64_t H,
                             int subw, int subh, Vship_ChromaLocation_t loc, float* out) {
    const int hcenter = (loc == Vship_ChromaLoc_Center || loc == Vship_ChromaLoc_Top);
    const int vtop = (loc == Vship_ChromaLoc_Top || loc == Vship_ChromaLoc_TopLeft);
    float* tmp = (float*)malloc(sizeof(float) * W * sh);
    for (int64_t y = 0; y < sh; y++) {
        if (subw == 0) memcpy(tmp + y * W, dec + y * sw, sizeof(float) * W);
        else h_upsample_row(dec + y * sw, sw, W, subw, hcenter, tmp + y * W);
    }
    if (subh == 0) {
        memcpy(out, tmp, sizeof(float) * W * H);
        free(tmp);
        return;
    }
    for (int64_t X = 0; X < W; X++) {
        if (vtop) {
            for (int64_t y = 0; y < sh + 1; y++) {
                Herm h = seq_interp(tmp + X, W, sh, y);
                if (2 * y < H) out[(2 * y) * W + X] = tmp[imin(y, sh - 1) * W + X];
                if (2 * y + 1 < H) out[(2 * y + 1) * W + X] = herm_get(h, 0.5f);
            }
        } else {
            for (int64_t y = -1; y < sh + 1; y++) {
                Herm h = seq_interp(tmp + X, W, sh, y);
                if (y != -1 && 2 * y + 1 < H) out[(2 * y + 1) * W + X] = herm_get(h, 0.25f);
                if (2 * y + 2 < H) out[(2 * y + 2) * W + X] = herm_get(h, 0.75f);
            }
        }
    }
    free(tmp);
}

/* ------------------------------------------------------------------------------------ */
/* Y'CbCr -> R'G'B' (YUVToLinRGB.hpp:7-155), transfer (transferToLinear.hpp:19-184),      */
/* primaries (primaries.hpp:9-144)                                                        */
/* ------------------------------------------------------------------------------------ */

/* The constant denominators vscale*Kr + 0.5f are folded at compile time. */
static float fold_den(float s, float k) { return s * k + 0.5f; }

/* ncl_yuv_to_rgb_from_kr_kb (:7-18); v = (Y, Cb, Cr). */
static void f_ncl(float v[3], float Kr, float Kb) {
    const float Kg = (1.f - Kb) - Kr;
    const float us = 0.5f / (1.f - Kb), vs = 0.5f / (1.f - Kr);
    const float r = fmaf(v[0], vs, v[2]) / fold_den(vs, Kr);
    const float b = fmaf(v[0], us, v[1]) / fold_den(us, Kb);
    const float g = fmaf(-Kb, b, fmaf(-Kr, r, v[0])) / Kg;
    v[0] = r; v[1] = g; v[2] = b;
}

static void f_gamma_light(float v[3], Vship_YUVMatrix_t m) {
    switch (m) {
    case Vship_MATRIX_BT709: f_ncl(v, 0.2126f, 0.0722f); break;
    case Vship_MATRIX_BT470_BG:
    case Vship_MATRIX_ST170_M: f_ncl(v, 0.299f, 0.114f); break;
    case Vship_MATRIX_BT2020_NCL: f_ncl(v, 0.2627f, 0.0593f); break;
    case Vship_MATRIX_BT2020_CL: {            /* :77-94 */
        const float Kr = 0.2627f, Kb = 0.0593f;
        const float us = 0.5f / (1.f - Kb), vs = 0.5f / (1.f - Kr);
        const float r = fmaf(v[0], vs, v[2]) / fold_den(vs, Kr);
        const float b = fmaf(v[0], us, v[1]) / fold_den(us, Kb);
        v[1] = v[0]; v[0] = r; v[2] = b;
        break;
    }
    case Vship_MATRIX_BT2100_ICTCP: {         /* :47-63, sequential substitution */
        v[0] = fmaf(v[1], 0.0086090370379327566f, fmaf(v[2], 0.11102962500302595655f, v[0]));
        v[1] = fmaf(v[1], -0.01721807407586551f, fmaf(v[2], -0.22205925000605192f, v[0]));
        v[2] = fmaf(v[0], 33.025782688766114f, fmaf(v[1], -32.025782688766114f, -v[2] * 7.543278084714549f));
        break;
    }
    default: break;
    }
}

static void f_linear_light(float v[3], Vship_YUVMatrix_t m) {
    if (m == Vship_MATRIX_BT2020_CL) {        /* :66-75 */
        const float Kr = 0.2627f, Kb = 0.0593f, Kg = (1.f - Kr) - Kb;
        v[1] = fmaf(-Kb, v[2], fmaf(-Kr, v[0], v[1])) / Kg;
    } else if (m == Vship_MATRIX_BT2100_ICTCP) { /* :28-43 */
        v[0] = fmaf(v[0], 3.4366066943330784267f, fmaf(v[1], -2.5064521186562698975f, v[2] * 0.069845424323191470954f));
        v[1] = fmaf(v[0], -0.23026480071281397f, fmaf(v[1], 1.4064527541936944f, -v[2] * 0.2083538389058436f));
        v[2] = fmaf(v[0], -0.02684381778741865f, fmaf(v[1], -0.08378524945770065f, (float)((double)v[2] * 1.106879231557486)));
    }
}

/* Transfer functions (transferToLinear.hpp:19-184) over the n values of v (all three
 * channels), in three steps: the float/double arithmetic before the transcendental, one
 * array evaluation of it, the arithmetic after.  Per value the steps are those of the
 * reference's transferLinearize<TRC>. */
static void f_trc_array(float* v, int64_t n, Vship_TransferFunction_t t) {
    float* arg = (float*)malloc(sizeof(float) * n);
    float* res = (float*)malloc(sizeof(float) * n);
    switch (t) {
    case Vship_TRC_sRGB:                      /* :73-88, the affine part in double */
        for (int64_t i = 0; i < n; i++) {
            const float a = v[i];
            arg[i] = a < 0 ? (float)(((double)(-a) + 0.055) * (1.0 / 1.055)) : (float)(((double)a + 0.055) * (1.0 / 1.055));
        }
        g_math(M_POW, arg, 2.4f, res, n);
        for (int64_t i = 0; i < n; i++) {
            const float a = v[i];
            if (a < 0) v[i] = a < -0.04045f ? -res[i] : (float)((double)a * (1.0 / 12.92));
            else v[i] = a > 0.04045f ? res[i] : (float)((double)a * (1.0 / 12.92));
        }
        break;
    case Vship_TRC_BT709:                     /* :111-118 (pure gamma), :120-141 */
    case Vship_TRC_BT470_M:
    case Vship_TRC_BT470_BG:
    case Vship_TRC_BT601:
    case Vship_TRC_ST428: {                   /* :161-165 */
        const float g = t == Vship_TRC_BT709 ? 2.4f : t == Vship_TRC_BT470_M ? 2.2f : t == Vship_TRC_ST428 ? 2.6f : 2.8f;
        for (int64_t i = 0; i < n; i++) arg[i] = v[i] < 0 ? -v[i] : v[i];
        g_math(M_POW, arg, g, res, n);
        for (int64_t i = 0; i < n; i++) {
            float a = v[i] < 0 ? -res[i] : res[i];
            if (t == Vship_TRC_ST428) a = (float)((double)a * (52.37 / 48.));
            v[i] = a;
        }
        break;
    }
    case Vship_TRC_ST240_M:                   /* :143-158 */
        for (int64_t i = 0; i < n; i++) arg[i] = v[i] < 0 ? -v[i] : v[i];
        g_math(M_POW, arg, 0.45f, res, n);
        for (int64_t i = 0; i < n; i++) {
            const float a = v[i];
            if (a >= 0) v[i] = (double)a < 0.0228 ? 4.f * a : (float)((double)(1.1115f * res[i]) - 0.1115);
            else v[i] = (double)a > -0.0228 ? 4.f * a : (float)((double)(-1.1115f * res[i]) + 0.1115);
        }
        break;
    case Vship_TRC_PQ: {                      /* :169-184 */
        const float Lmax = 100.f, pn = 0.15930175781250000f, pm = 78.843750000000000f;
        const float c1 = 0.83593750000000000f, c2 = 18.851562500000000f, c3 = 18.687500000000000f;
        for (int64_t i = 0; i < n; i++) arg[i] = v[i] > 0.f ? v[i] : 0.f;
        g_math(M_POW, arg, 1.f / pm, res, n);
        for (int64_t i = 0; i < n; i++) {
            const float a = res[i];
            const float num = (a - c1) > 0.f ? (a - c1) : 0.f;
            const float den = fmaf(-c3, a, c2);
            arg[i] = num / den;
        }
        g_math(M_POW, arg, 1.f / pn, res, n);
        for (int64_t i = 0; i < n; i++) v[i] = Lmax * res[i];
        break;
    }
    default: break;                           /* Linear */
    }
    free(arg);
    free(res);
}

/* transferLinearizeHLG (transferToLinear.hpp:23-51) on planar p (3 x n). */
static void f_hlg_array(float* p, int64_t n) {
    const float a = 0.17883277f, b = 1.f - 4.f * a;
    const float c = 0.5f - a * -0.3350097945111627f;
    const float gamma = 1.2f;
    float* arg = (float*)malloc(sizeof(float) * 3 * n);
    float* res = (float*)malloc(sizeof(float) * 3 * n);
    for (int64_t i = 0; i < 3 * n; i++) arg[i] = (p[i] - c) / a;
    g_math(M_EXP, arg, 0.f, res, 3 * n);
    for (int64_t i = 0; i < 3 * n; i++) p[i] = p[i] <= 0.5f ? p[i] * p[i] / 3.f : (res[i] + b) / 12.f;
    for (int64_t i = 0; i < n; i++) {
        const float x = p[i], y = p[n + i], z = p[2 * n + i];
        const float part = fmaf(0.2627f, x, 0.6780f * y);
        const double ys = fma(0.0593, (double)z, (double)part);
        arg[i] = (float)ys;
    }
    g_math(M_POW, arg, gamma - 1.f, res, n);
    for (int64_t i = 0; i < n; i++) {
        p[i] = p[i] * res[i];
        p[n + i] = p[n + i] * res[i];
        p[2 * n + i] = p[2 * n + i] * res[i];
    }
    free(arg);
    free(res);
}

/* res.k = fmaf(a.x, m0, fmaf(a.y, m1, a.z*m2)) with m2 negated as written where the
 * reference writes -a.z*c (primaries.hpp:17-112). */
static void f_mat(float v[3], const float m[9]) {
    float r = fmaf(v[0], m[0], fmaf(v[1], m[1], v[2] * m[2]));
    float g = fmaf(v[0], m[3], fmaf(v[1], m[4], v[2] * m[5]));
    float b = fmaf(v[0], m[6], fmaf(v[1], m[7], v[2] * m[8]));
    v[0] = r; v[1] = g; v[2] = b;
}

static const float* f_to_xyz(Vship_Primaries_t p) {
    static const float st170[9] = {0.39349893f, 0.3652766f, 0.19162447f, 0.2123645f, 0.70109542f, 0.08654008f, 0.01873804f, 0.1119396f, 0.95812235f};
    static const float bg[9] = {0.4305f, 0.3416f, 0.1783f, 0.2220f, 0.7067f, 0.07132f, 0.0202f, 0.1296f, 0.9391f};
    static const float m470[9] = {0.6068f, 0.1735f, 0.2003f, 0.2989f, 0.5866f, 0.1145f, 0.f, 0.06609f, 1.116f};
    static const float bt709[9] = {0.4124f, 0.3576f, 0.1805f, 0.2126f, 0.7152f, 0.0722f, 0.0193f, 0.1192f, 0.9505f};
    static const float bt2020[9] = {0.6370f, 0.1446f, 0.1689f, 0.2627f, 0.6780f, 0.0593f, 0.f, 0.0281f, 1.0610f};
    switch (p) {
    case Vship_PRIMARIES_ST170_M: case Vship_PRIMARIES_ST240_M: return st170;
    case Vship_PRIMARIES_BT470_BG: return bg;
    case Vship_PRIMARIES_BT470_M: return m470;
    case Vship_PRIMARIES_BT709: return bt709;
    case Vship_PRIMARIES_BT2020: return bt2020;
    default: return NULL;
    }
}

/* primariesToPrimaries_device2<T1, BT709> (primaries.hpp:134-144). */
static void f_primaries_to_709(float v[3], Vship_Primaries_t p) {
    static const float xyz_to_709[9] = {3.2410f, -1.5374f, -0.4986f, -0.9692f, 1.8760f, 0.0416f, 0.0556f, -0.2040f, 1.0570f};
    static const float bt2020_to_709[9] = {1.6605f, -0.5876f, -0.0728f, -0.1246f, 1.1329f, -0.0083f, -0.0182f, -0.1006f, 1.1187f};
    if (p == Vship_PRIMARIES_BT709) return;
    if (p == Vship_PRIMARIES_BT2020) { f_mat(v, bt2020_to_709); return; }
    const float* m = f_to_xyz(p);
    if (m) f_mat(v, m);
    f_mat(v, xyz_to_709);
}

/* horizontalResizeTranspose_Kernel (resize.hpp:26-48). */
static void f_resize_transpose(const float* src, int64_t sw, int64_t sh, int64_t rw, float* dst) {
    for (int64_t y = 0; y < sh; y++) {
        const float* row = src + y * sw;
        for (int64_t x = 0; x < rw; x++) {
            const float approx = (float)x * (float)sw / (float)rw;
            const int64_t b = (int64_t)approx;
            const float v1 = row[b];
            const float v0 = b - 1 >= 0 ? row[b - 1] : v1;
            const float v2 = b + 1 < sw ? row[b + 1] : v1;
            const float v3 = b + 2 < sw ? row[b + 2] : v2;
            Herm h = herm_make(v1, (v2 - v0) / 2.f, v2, (v3 - v1) / 2.f);
            dst[x * sh + y] = herm_get(h, approx - (float)b);
        }
    }
}

/* Converter::convert (vshipColor.hpp:62-146) to linear BT.709 RGB, planar float. */
ORACLE_API int oracle_f32_convert(const uint8_t* const planes[3], const int64_t linesize[3],
                                  const Vship_Colorspace_t* cs, float* out) {
    const int64_t W = cs->width, H = cs->height;
    const int subw = cs->subsampling.subw, subh = cs->subsampling.subh;
    if (subw < 0 || subw > 2 || subh < 0 || subh > 1) return 1;
    const int64_t N = W * H;
    float* full = (float*)malloc(sizeof(float) * 3 * N);
    for (int c = 0; c < 3; c++) {
        const int64_t pw = c ? ((W - 1) >> subw) + 1 : W, ph = c ? ((H - 1) >> subh) + 1 : H;
        const int chroma = c != 0 && cs->colorFamily == Vship_ColorYUV;
        float* dec = (c && (subw || subh)) ? (float*)malloc(sizeof(float) * pw * ph) : full + c * N;
        for (int64_t y = 0; y < ph; y++)
            for (int64_t x = 0; x < pw; x++)
                dec[y * pw + x] = f_full_range(f_pick(planes[c], linesize[c], x, y, cs->sample), cs->sample, cs->range, chroma);
        if (dec != full + c * N) {
            f_upsample_plane(dec, pw, ph, W, H, subw, subh, cs->chromaLocation, full + c * N);
            free(dec);
        }
    }
    /* YUVToLinRGBPipeline_Device (YUVToLinRGB.hpp:157-163), skipped for linear RGB (:219),
     * then the primaries (vshipColor.hpp:119-123) */
    const int skip_yuv = (cs->transferFunction == Vship_TRC_Linear && cs->YUVMatrix == Vship_MATRIX_RGB);
    if (!skip_yuv) {
        for (int64_t i = 0; i < N; i++) {
            float v[3] = {full[i], full[N + i], full[2 * N + i]};
            f_gamma_light(v, cs->YUVMatrix);
            full[i] = v[0]; full[N + i] = v[1]; full[2 * N + i] = v[2];
        }
        if (cs->transferFunction == Vship_TRC_HLG) f_hlg_array(full, N);
        else f_trc_array(full, 3 * N, cs->transferFunction);
    }
    for (int64_t i = 0; i < N; i++) {
        float v[3] = {full[i], full[N + i], full[2 * N + i]};
        if (!skip_yuv) f_linear_light(v, cs->YUVMatrix);
        f_primaries_to_709(v, cs->primaries);
        full[i] = v[0]; full[N + i] = v[1]; full[2 * N + i] = v[2];
    }
    const int64_t TW = cs->target_width == -1 ? W : cs->target_width;
    const int64_t TH = cs->target_height == -1 ? H : cs->target_height;
    const int64_t OW = TW - cs->crop.left - cs->crop.right, OH = TH - cs->crop.top - cs->crop.bottom;
    for (int c = 0; c < 3; c++) {
        const float* src = full + c * N;
        float* rs = NULL;
        if (TW != W || TH != H) {
            float* tmp = (float*)malloc(sizeof(float) * TW * H);
            rs = (float*)malloc(sizeof(float) * TW * TH);
            f_resize_transpose(src, W, H, TW, tmp);
            f_resize_transpose(tmp, H, TW, TH, rs);
            free(tmp);
            src = rs;
        }
        for (int64_t y = 0; y < OH; y++)
            memcpy(out + c * OW * OH + y * OW, src + (y + cs->crop.top) * TW + cs->crop.left, sizeof(float) * OW);
        free(rs);
    }
    free(full);
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Pyramid and XYB (ssimu2/downsample.hpp:3-19, makeXYB.hpp:6-47)                        */
/* ------------------------------------------------------------------------------------ */

static void f_downsample(const float* src, int64_t w, int64_t h, float* dst) {
    const int64_t nw = (w - 1) / 2 + 1, nh = (h - 1) / 2 + 1;
    for (int64_t y = 0; y < nh; y++) {
        const int64_t y0 = imin(2 * y, h - 1), y1 = imin(2 * y + 1, h - 1);
        for (int64_t x = 0; x < nw; x++) {
            const int64_t x0 = imin(2 * x, w - 1), x1 = imin(2 * x + 1, w - 1);
            float d = src[y0 * w + x0];
            d += src[y1 * w + x0];
            d += src[y0 * w + x1];
            d += src[y1 * w + x1];
            dst[y * nw + x] = d * 0.25f;
        }
    }
}

/* rgb_to_positive_xyb_d (makeXYB.hpp:6-47) over n pixels of planar p: the opsin sums are
 * the reference's fmaf chains; make_positive_xyb adds double literals, so those three sums
 * are formed in double. */
static void f_positive_xyb(float* p0, float* p1, float* p2, int64_t n) {
    const float bias = 0.0037930734f, absb = -0.1559542025327239f;
    float* lms = (float*)malloc(sizeof(float) * 3 * n);
    float* cr = (float*)malloc(sizeof(float) * 3 * n);
    for (int64_t i = 0; i < n; i++) {
        const float r = p0[i], g = p1[i], b = p2[i];
        const float l = fmaf(0.30f, r, fmaf(0.622f, g, fmaf(0.078f, b, bias)));
        const float m = fmaf(0.23f, r, fmaf(0.692f, g, fmaf(0.078f, b, bias)));
        const float s = fmaf(0.24342269f, r, fmaf(0.20476745f, g, fmaf(0.55180986f, b, bias)));
        lms[3 * i] = l * (float)(l >= 0);
        lms[3 * i + 1] = m * (float)(m >= 0);
        lms[3 * i + 2] = s * (float)(s >= 0);
    }
    g_math(M_CBRT, lms, 0.f, cr, 3 * n);
    for (int64_t i = 0; i < n; i++) {
        const float l = cr[3 * i] + absb, m = cr[3 * i + 1] + absb, s = cr[3 * i + 2] + absb;
        const float X = 0.5f * (l - m);
        const float Y = X + m;
        p2[i] = (float)((double)(s - Y) + 0.55);
        p0[i] = (float)((double)(X * 14.0f) + 0.42);
        p1[i] = (float)((double)Y + 0.01);
    }
    free(lms);
    free(cr);
}

/* ------------------------------------------------------------------------------------ */
/* Maps and reductions (gaussianblur.hpp:7-77, score.hpp:116-460)                        */
/* ------------------------------------------------------------------------------------ */

static float g_taps[17], g_integral[18];

/* GaussianHandle::init (gaussianblur.hpp:7-18): taps in the reference's float/double steps,
 * and their running sums in float. */
static void f_gauss_init(void) {
    const float sigma = 1.5f;
    const double tau = 6.28318530718;
    g_integral[0] = 0.f;
    for (int i = 0; i < 17; i++) {
        const int d = 8 - i;
        /* -(d*d) is an int; 2*SIGMA*SIGMA is float; the exponent is formed in float */
        const float e = (float)(-(d * d)) / (2.f * sigma * sigma);
        /* std::exp of a float is the host's expf; the quotient by the double root is double */
        g_taps[i] = (float)((double)expf(e) / sqrt(tau * (double)sigma * (double)sigma));
        g_integral[i + 1] = g_integral[i] + g_taps[i];
    }
}

/* GaussianSmart_Device (gaussianblur.hpp:41-77) over a whole plane.  The 32x32 tile is
 * zero outside the image and the tap sum is accumulated from the left (top) tap with a
 * fused multiply-add per tap; zero samples leave the running sum unchanged, so each
 * output is the same chain over its in-image taps.  Each pass divides by the in-image
 * tap sum, a difference of two running sums. */
static void f_blur(const float* src, float* tmp, float* dst, int64_t w, int64_t h) {
    for (int64_t y = 0; y < h; y++) {
        for (int64_t x = 0; x < w; x++) {
            const int64_t beg = imax(0, x - 8) - (x - 8);
            const int64_t end = imin(w, x + 9) - imin(w, x - 8);
            const float tot = g_integral[end] - g_integral[beg];
            float acc = 0.f;
            for (int i = 0; i < 17; i++) {
                const int64_t xx = x - 8 + i;
                if (xx >= 0 && xx < w) acc = fmaf(src[y * w + xx], g_taps[i], acc);
            }
            tmp[y * w + x] = acc / tot;
        }
    }
    for (int64_t y = 0; y < h; y++) {
        const int64_t beg = imax(0, y - 8) - (y - 8);
        const int64_t end = imin(h, y + 9) - imin(h, y - 8);
        const float tot = g_integral[end] - g_integral[beg];
        for (int64_t x = 0; x < w; x++) {
            float acc = 0.f;
            for (int i = 0; i < 17; i++) {
                const int64_t yy = y - 8 + i;
                if (yy >= 0 && yy < h) acc = fmaf(tmp[yy * w + x], g_taps[i], acc);
            }
            dst[y * w + x] = acc / tot;
        }
    }
}

/* Pairwise tree over n (a power of two) values, as the shared-memory loops of
 * planescale_map_Kernel (score.hpp:299-312) and sumreduce (:145-188) add them. */
static float f_tree(float* v, int n) {
    for (int next = 1; next < n; next *= 2)
        for (int i = 0; i + next < n; i += 2 * next) v[i] += v[i + next];
    return v[0];
}

static int f_map_on(int plane, int scale, int map) {
    const float w1 = (float)kSsimu2Weights[plane * 36 + scale * 6 + map];
    const float w4 = (float)kSsimu2Weights[plane * 36 + scale * 6 + 3 + map];
    return !(w1 <= VSHIP_SSIMU2_PRUNE && w4 <= VSHIP_SSIMU2_PRUNE);
}

/* planescale_map (score.hpp:192-378): the six norms of one (plane, scale) as the reference
 * forms them: per 16x16 block a tree sum divided by w*h, then 1024-wide tree passes. */
static void f_planescale(const float* a, const float* b, int64_t w, int64_t h,
                         int do_ssim, int do_art, int do_det, float out[6]) {
    const int64_t n = w * h;
    float* buf = (float*)malloc(sizeof(float) * n * 7);
    float *prod = buf, *sq = buf + n, *m1 = buf + 2 * n, *m2 = buf + 3 * n, *s12 = buf + 4 * n, *ssq = buf + 5 * n;
    float* tmp = buf + 6 * n;
    for (int64_t i = 0; i < n; i++) {
        prod[i] = a[i] * b[i];
        const float t = a[i] + b[i];
        sq[i] = t * t;
    }
    if (do_ssim) { f_blur(prod, tmp, s12, w, h); f_blur(sq, tmp, ssq, w, h); }
    f_blur(a, tmp, m1, w, h);
    f_blur(b, tmp, m2, w, h);

    const int64_t bx = (w - 1) / 16 + 1, by = (h - 1) / 16 + 1, nb = bx * by;
    float* part = (float*)malloc(sizeof(float) * 6 * nb);
    const float area = (float)(w * h);
    float vals[6][256];
    for (int64_t B = 0; B < nb; B++) {
        const int64_t x0 = (B % bx) * 16, y0 = (B / bx) * 16;
        for (int t = 0; t < 256; t++) {
            const int64_t x = x0 + (t & 15), y = y0 + (t >> 4);
            float ssim = 0.f, art = 0.f, det = 0.f;
            if (x < w && y < h) {
                const int64_t i = y * w + x;
                if (do_ssim) {
                    const float M1 = m1[i], M2 = m2[i], S12 = s12[i];
                    const float s1122 = ssq[i] - 2.f * S12;
                    const float md = M1 - M2;
                    const float num_m = fmaf(md, md * -1.0f, 1.0f);
                    const float num_s = fmaf(fmaf(-M1, M2, S12), 2.0f, 0.0009f);
                    const float den_s = fmaf(-M2, M2, fmaf(-M1, M1, s1122)) + 0.0009f;
                    const float q = 1.0f - (num_m * num_s) / den_s;
                    ssim = q > 0.f ? q : 0.f;
                }
                if (do_art || do_det) {
                    const float v1 = (fabsf(b[i] - m2[i]) + 1.0f) / (fabsf(a[i] - m1[i]) + 1.0f) - 1.0f;
                    if (do_art) art = v1 > 0.f ? v1 : 0.f;
                    if (do_det) det = -v1 > 0.f ? -v1 : 0.f;
                }
            }
            float s2 = ssim * ssim, a2 = art * art, d2 = det * det;
            vals[0][t] = ssim; vals[1][t] = art; vals[2][t] = det;
            vals[3][t] = s2 * s2; vals[4][t] = a2 * a2; vals[5][t] = d2 * d2;
        }
        for (int k = 0; k < 6; k++) part[k * nb + B] = f_tree(vals[k], 256) / area;
    }
    /* sumreduce passes (score.hpp:361-378) */
    int64_t cnt = nb;
    float* cur = part;
    float chunk[1024];
    while (cnt != 1) {
        const int64_t groups = (cnt - 1) / 1024 + 1;
        float* nxt = (float*)malloc(sizeof(float) * 6 * groups);
        for (int k = 0; k < 6; k++)
            for (int64_t g = 0; g < groups; g++) {
                for (int t = 0; t < 1024; t++) {
                    const int64_t idx = g * 1024 + t;
                    chunk[t] = idx < cnt ? cur[k * cnt + idx] : 0.f;
                }
                nxt[k * groups + g] = f_tree(chunk, 1024);
            }
        if (cur != part) free(cur);
        cur = nxt;
        cnt = groups;
    }
    for (int k = 0; k < 6; k++) out[k] = cur[k];
    if (cur != part) free(cur);
    free(part);
    free(buf);
}

/* ssimu2GPUProcess (main.hpp:27-78), allscore_map (score.hpp:380-440) and final_score
 * (:442-460) on planar float linear RGB of w x h.  features gets the 108 floats the host
 * receives (4-norms already rooted); the return value is the float score widened. */
ORACLE_API double oracle_f32_ssimu2(const float* rgb1, const float* rgb2, int64_t w, int64_t h, float* features) {
    f_gauss_init();
    int64_t ws[6], hs[6], off[6], total = 0;
    ws[0] = w; hs[0] = h;
    for (int s = 0; s < 6; s++) {
        if (s) { ws[s] = (ws[s - 1] - 1) / 2 + 1; hs[s] = (hs[s - 1] - 1) / 2 + 1; }
        off[s] = total;
        total += ws[s] * hs[s];
    }
    float* pyr[2][3];
    for (int im = 0; im < 2; im++) {
        const float* rgb = im ? rgb2 : rgb1;
        for (int c = 0; c < 3; c++) {
            pyr[im][c] = (float*)malloc(sizeof(float) * total);
            memcpy(pyr[im][c], rgb + c * w * h, sizeof(float) * w * h);
            for (int s = 1; s < 6; s++)
                f_downsample(pyr[im][c] + off[s - 1], ws[s - 1], hs[s - 1], pyr[im][c] + off[s]);
        }
        f_positive_xyb(pyr[im][0], pyr[im][1], pyr[im][2], total);
    }
    float res[108];
    memset(res, 0, sizeof(res));
    for (int s = 0; s < 6; s++)
        for (int p = 0; p < 3; p++) {
            const int ds = f_map_on(p, s, 0), da = f_map_on(p, s, 1), dd = f_map_on(p, s, 2);
            if (!ds && !da && !dd) continue;
            float o[6];
            f_planescale(pyr[0][p] + off[s], pyr[1][p] + off[s], ws[s], hs[s], ds, da, dd, o);
            for (int k = 0; k < 6; k++) res[p * 36 + s * 6 + k] = o[k];
        }
    for (int s = 0; s < 6; s++)
        for (int p = 0; p < 3; p++)
            for (int m = 0; m < 3; m++)
                if (f_map_on(p, s, m)) res[p * 36 + s * 6 + 3 + m] = sqrtf(sqrtf(res[p * 36 + s * 6 + 3 + m]));
    for (int im = 0; im < 2; im++)
        for (int c = 0; c < 3; c++) free(pyr[im][c]);
    if (features) memcpy(features, res, sizeof(res));
    double ssim = 0.0;
    for (int i = 0; i < 108; i++) ssim = fmaf((float)kSsimu2Weights[i], res[i], (float)ssim);
    ssim *= VSHIP_SSIMU2_SCALE;
    ssim = (VSHIP_SSIMU2_C3 * ssim * ssim) * ssim + VSHIP_SSIMU2_C1 * ssim - VSHIP_SSIMU2_C2 * ssim * ssim;
    ssim = ssim > 0.0 ? pow(ssim, VSHIP_SSIMU2_EXP) * -10.0 + 100.0 : 100.0;
    return (double)(float)ssim;
}

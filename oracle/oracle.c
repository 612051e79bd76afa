/*
 * oracle.c -- FP64 CPU restatement of Vship's SSIMULACRA2 and Butteraugli hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA engine is compared against
 * and the CPU baseline that bench.py times; the product (vship_b200/libvship.so) never
 * links, loads or calls it.  Every stage follows the reference file:line cited beside it,
 * including Vship's own quirks (weight pruning, truncated renormalised blurs, pure-gamma
 * "BT.709" transfer, the float accumulation in final_score, the doubled 0.8 factor of the
 * asymmetric L2 term).  All arithmetic is in double; constants are the reference's decimal
 * literals.  Loops over rows are OpenMP-parallel so the CPU baseline uses every host core.
 *
 * Parity pin: tests/golden/ holds scores produced by the reference itself (built from its
 * own sources by oracle/build_ref.sh and run on a B200); tests/test_oracle.py checks this
 * restatement against them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/VshipColor.h"
#include "../vship_b200/csrc/metric_tables.h"

#define ORACLE_API __attribute__((visibility("default")))

static inline int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
static inline int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }
static inline int64_t clampi(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------------------------ */
/* Sample decode and range (src/gpuColorToLinear/anyDepthToFloat.hpp:9-68,             */
/* src/gpuColorToLinear/rangeToFull.hpp:5-55)                                            */
/* ------------------------------------------------------------------------------------ */

static int sample_bytes(Vship_Sample_t s) {
    switch (s) {
    case Vship_SampleUINT8: return 1;
    case Vship_SampleFLOAT: return 4;
    default: return 2;
    }
}

static int sample_bits(Vship_Sample_t s) {
    switch (s) {
    case Vship_SampleUINT8: return 8;
    case Vship_SampleUINT9: return 9;
    case Vship_SampleUINT10: return 10;
    case Vship_SampleUINT12: return 12;
    case Vship_SampleUINT14: return 14;
    case Vship_SampleUINT16: return 16;
    default: return 1; /* float and half */
    }
}

/* IEEE-754 binary16 -> double. */
static double half_to_double(uint16_t h) {
    int sign = h >> 15, e = (h >> 10) & 31, m = h & 1023;
    double v;
    if (e == 0) v = ldexp((double)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexp((double)(m | 1024), e - 25);
    return sign ? -v : v;
}

/* PickValue (anyDepthToFloat.hpp:24-68): integer samples keep only their low bits. */
static double pick_sample(const uint8_t* plane, int64_t stride, int64_t x, int64_t y, Vship_Sample_t s) {
    const uint8_t* p = plane + y * stride + (int64_t)sample_bytes(s) * x;
    if (s == Vship_SampleUINT8) return (double)p[0];
    if (s == Vship_SampleFLOAT) { float f; memcpy(&f, p, 4); return (double)f; }
    uint16_t raw = (uint16_t)(p[0] | (p[1] << 8));
    if (s == Vship_SampleHALF) return half_to_double(raw);
    return (double)(raw & ((1u << sample_bits(s)) - 1u));
}

/* FullRange (rangeToFull.hpp:24-55). */
static double to_full_range(double a, Vship_Sample_t s, Vship_Range_t r, int chroma) {
    int bd = sample_bits(s);
    if (r == Vship_RangeFull) {
        a /= (double)((1 << bd) - 1);
        if (chroma) a -= 0.5;
        return a;
    }
    if (bd >= 8) a /= (double)(1 << (bd - 8));
    else a *= 256.0;
    return chroma ? (a - 128.0) / 224.0 : (a - 16.0) / 219.0;
}

/* ------------------------------------------------------------------------------------ */
/* Chroma upsampling (src/gpuColorToLinear/chromaUpsample.hpp:28-247)                    */
/* ------------------------------------------------------------------------------------ */

/* Cubic Hermite on [p0, p1] with tangents m0, m1 (resize.hpp:5-24). */
static double hermite(double p0, double m0, double p1, double m1, double t) {
    double v1 = 2 * p0 + m0 - 2 * p1 + m1;
    double v2 = -3 * p0 + 3 * p1 - 2 * m0 - m1;
    return ((v1 * t + v2) * t + m0) * t + p0;
}

/* Interpolate a clamped 1-D sequence get(i) between i and i+1 at fraction t
 * (getHorizontalInterpolator_device / getVerticalInterpolator_device, :28-50). */
static double interp_seq(const double* base, int64_t step, int64_t n, int64_t i, double t) {
    double em1 = base[clampi(i - 1, 0, n - 1) * step];
    double e0 = base[clampi(i, 0, n - 1) * step];
    double e1 = base[clampi(i + 1, 0, n - 1) * step];
    double e2 = base[clampi(i + 2, 0, n - 1) * step];
    return hermite(e0, (e1 - em1) / 2, e1, (e2 - e0) / 2, t);
}

/* Position of full-resolution sample X on the decimated axis: interval start i and
 * fraction t.  sub is log2 of the factor; centered selects the Center variants
 * (chroma sample between luma samples) instead of the co-sited Left/Top variants. */
static void upsample_phase(int64_t X, int sub, int centered, int64_t* i, double* t) {
    if (sub == 0) { *i = X; *t = 0.0; return; }
    int64_t f = (int64_t)1 << sub;
    if (!centered) {                       /* bicubic*LeftUpscaleX*, bicubicVerticalTop */
        *i = X / f;
        *t = (double)(X % f) / (double)f;
    } else {                               /* bicubic*CenterUpscaleX* */
        int64_t off = X - f / 2;           /* X = f*i + f/2 + k, k in [0, f) */
        int64_t q = off >= 0 ? off / f : -((-off + f - 1) / f);
        *i = q;
        *t = ((double)(off - q * f) + 0.5) / (double)f;
    }
}

/* Upsamples one chroma plane (sw x sh) to (W x H): horizontal pass over the sh rows,
 * then vertical pass (upsample(), chromaUpsample.hpp:153-247). */
static void upsample_plane(const double* small, int64_t sw, int64_t sh, int64_t W, int64_t H,
                           int subw, int subh, Vship_ChromaLocation_t loc, double* out) {
    int hcenter = (loc == Vship_ChromaLoc_Center || loc == Vship_ChromaLoc_Top);
    int vcenter = (loc == Vship_ChromaLoc_Center || loc == Vship_ChromaLoc_Left);
    double* tmp = (double*)malloc(sizeof(double) * W * sh);
    #pragma omp parallel for
    for (int64_t y = 0; y < sh; y++) {
        for (int64_t X = 0; X < W; X++) {
            int64_t i; double t;
            upsample_phase(X, subw, hcenter, &i, &t);
            tmp[y * W + X] = (subw == 0) ? small[y * sw + X] : interp_seq(small + y * sw, 1, sw, i, t);
        }
    }
    #pragma omp parallel for
    for (int64_t Y = 0; Y < H; Y++) {
        int64_t i; double t;
        upsample_phase(Y, subh, vcenter, &i, &t);
        for (int64_t X = 0; X < W; X++)
            out[Y * W + X] = (subh == 0) ? tmp[Y * W + X] : interp_seq(tmp + X, W, sh, i, t);
    }
    free(tmp);
}

/* ------------------------------------------------------------------------------------ */
/* Y'CbCr -> R'G'B', transfer, primaries (YUVToLinRGB.hpp:7-181,                        */
/* transferToLinear.hpp:19-184, primaries.hpp:9-158)                                     */
/* ------------------------------------------------------------------------------------ */

static void ncl_to_rgb(double v[3], double kr, double kb) {
    double kg = 1.0 - kb - kr, us = 0.5 / (1.0 - kb), vs = 0.5 / (1.0 - kr);
    double r = (v[2] + v[0] * vs) / (vs * kr + 0.5);
    double b = (v[1] + v[0] * us) / (us * kb + 0.5);
    double g = (v[0] - kr * r - kb * b) / kg;
    v[0] = r; v[1] = g; v[2] = b;
}

static void gamma_light(double v[3], Vship_YUVMatrix_t m) {
    switch (m) {
    case Vship_MATRIX_BT709: ncl_to_rgb(v, 0.2126, 0.0722); break;
    case Vship_MATRIX_BT470_BG:
    case Vship_MATRIX_ST170_M: ncl_to_rgb(v, 0.299, 0.114); break;
    case Vship_MATRIX_BT2020_NCL: ncl_to_rgb(v, 0.2627, 0.0593); break;
    case Vship_MATRIX_BT2020_CL: {           /* :78-94, R' and B' only, Y' kept */
        double kr = 0.2627, kb = 0.0593, us = 0.5 / (1.0 - kb), vs = 0.5 / (1.0 - kr);
        double r = (v[2] + v[0] * vs) / (vs * kr + 0.5);
        double b = (v[1] + v[0] * us) / (us * kb + 0.5);
        v[1] = v[0]; v[0] = r; v[2] = b;
        break;
    }
    case Vship_MATRIX_BT2100_ICTCP: {        /* :47-63, sequential substitution */
        v[0] = v[1] * 0.0086090370379327566 + (v[2] * 0.11102962500302595655 + v[0]);
        v[1] = v[1] * -0.01721807407586551 + (v[2] * -0.22205925000605192 + v[0]);
        v[2] = v[0] * 33.025782688766114 + (v[1] * -32.025782688766114 - v[2] * 7.543278084714549);
        break;
    }
    default: break;                          /* RGB */
    }
}

static void linear_light(double v[3], Vship_YUVMatrix_t m) {
    if (m == Vship_MATRIX_BT2020_CL) {       /* :66-75 */
        double kr = 0.2627, kb = 0.0593, kg = 1.0 - kr - kb;
        v[1] = (v[1] - kr * v[0] - kb * v[2]) / kg;
    } else if (m == Vship_MATRIX_BT2100_ICTCP) { /* :28-43, sequential substitution */
        v[0] = v[0] * 3.4366066943330784267 + (v[1] * -2.5064521186562698975 + v[2] * 0.069845424323191470954);
        v[1] = v[0] * -0.23026480071281397 + (v[1] * 1.4064527541936944 - v[2] * 0.2083538389058436);
        v[2] = v[0] * -0.02684381778741865 + (v[1] * -0.08378524945770065 + v[2] * 1.106879231557486);
    }
}

static double signed_pow(double a, double g) { return a < 0 ? -pow(-a, g) : pow(a, g); }

static double trc_one(double a, Vship_TransferFunction_t t) {
    switch (t) {
    case Vship_TRC_sRGB:                     /* :73-88 */
        if (a < 0) return a < -0.04045 ? -pow((-a + 0.055) / 1.055, 2.4) : a / 12.92;
        return a > 0.04045 ? pow((a + 0.055) / 1.055, 2.4) : a / 12.92;
    case Vship_TRC_BT709: return signed_pow(a, 2.4);        /* :110-118, pure gamma */
    case Vship_TRC_BT470_M: return signed_pow(a, 2.2);      /* :128-131 */
    case Vship_TRC_BT470_BG:
    case Vship_TRC_BT601: return signed_pow(a, 2.8);        /* :133-141 */
    case Vship_TRC_ST240_M:                                  /* :143-158 */
        if (a >= 0) return a < 0.0228 ? 4 * a : 1.1115 * pow(a, 0.45) - 0.1115;
        return a > -0.0228 ? 4 * a : -1.1115 * pow(-a, 0.45) + 0.1115;
    case Vship_TRC_ST428: return signed_pow(a, 2.6) * 52.37 / 48.0; /* :161-165 */
    case Vship_TRC_PQ: {                                     /* :169-184, Lmax = 100 */
        const double n = 0.15930175781250000, m = 78.843750000000000;
        const double c1 = 0.83593750000000000, c2 = 18.851562500000000, c3 = 18.687500000000000;
        a = a > 0 ? a : 0;
        a = pow(a, 1.0 / m);
        double num = a - c1 > 0 ? a - c1 : 0;
        return 100.0 * pow(num / (c2 - c3 * a), 1.0 / n);
    }
    default: return a;                                       /* Linear */
    }
}

static void transfer(double v[3], Vship_TransferFunction_t t) {
    if (t == Vship_TRC_HLG) {                /* :23-50 */
        const double a = 0.17883277, b = 1.0 - 4.0 * a, c = 0.5 - a * -0.3350097945111627;
        for (int i = 0; i < 3; i++)
            v[i] = v[i] <= 0.5 ? v[i] * v[i] / 3.0 : (exp((v[i] - c) / a) + b) / 12.0;
        double ys = 0.2627 * v[0] + 0.6780 * v[1] + 0.0593 * v[2];
        double s = pow(ys, 1.2 - 1.0);
        for (int i = 0; i < 3; i++) v[i] *= s;
        return;
    }
    for (int i = 0; i < 3; i++) v[i] = trc_one(v[i], t);
}

static void mat3(double v[3], const double m[9]) {
    double r = v[0] * m[0] + (v[1] * m[1] + v[2] * m[2]);
    double g = v[0] * m[3] + (v[1] * m[4] + v[2] * m[5]);
    double b = v[0] * m[6] + (v[1] * m[7] + v[2] * m[8]);
    v[0] = r; v[1] = g; v[2] = b;
}

/* RGB -> XYZ matrices per primaries (primaries.hpp:17-112). */
static const double* to_xyz(Vship_Primaries_t p) {
    static const double st170[9] = {0.39349893, 0.3652766, 0.19162447, 0.2123645, 0.70109542, 0.08654008, 0.01873804, 0.1119396, 0.95812235};
    static const double bg[9] = {0.4305, 0.3416, 0.1783, 0.2220, 0.7067, 0.07132, 0.0202, 0.1296, 0.9391};
    static const double m470[9] = {0.6068, 0.1735, 0.2003, 0.2989, 0.5866, 0.1145, 0.0, 0.06609, 1.116};
    static const double bt709[9] = {0.4124, 0.3576, 0.1805, 0.2126, 0.7152, 0.0722, 0.0193, 0.1192, 0.9505};
    static const double bt2020[9] = {0.6370, 0.1446, 0.1689, 0.2627, 0.6780, 0.0593, 0.0, 0.0281, 1.0610};
    switch (p) {
    case Vship_PRIMARIES_ST170_M: case Vship_PRIMARIES_ST240_M: return st170;
    case Vship_PRIMARIES_BT470_BG: return bg;
    case Vship_PRIMARIES_BT470_M: return m470;
    case Vship_PRIMARIES_BT709: return bt709;
    case Vship_PRIMARIES_BT2020: return bt2020;
    default: return NULL;                    /* INTERNAL: already XYZ */
    }
}

/* Linear RGB in primaries p -> linear BT.709 (vshipColor.hpp:119-123, primaries.hpp:134-144). */
static void primaries_to_709(double v[3], Vship_Primaries_t p) {
    static const double xyz_to_709[9] = {3.2410, -1.5374, -0.4986, -0.9692, 1.8760, 0.0416, 0.0556, -0.2040, 1.0570};
    static const double bt2020_to_709[9] = {1.6605, -0.5876, -0.0728, -0.1246, 1.1329, -0.0083, -0.0182, -0.1006, 1.1187};
    if (p == Vship_PRIMARIES_BT709) return;
    if (p == Vship_PRIMARIES_BT2020) { mat3(v, bt2020_to_709); return; }
    const double* m = to_xyz(p);
    if (m) mat3(v, m);
    mat3(v, xyz_to_709);
}

/* horizontalResizeTranspose_Kernel (resize.hpp:26-48): cubic Hermite resize of each row
 * to rw samples, written transposed.  The source coordinate x*sw/rw is formed in float as
 * in the reference. */
void oracle_resize_transpose(const double* src, int64_t sw, int64_t sh, int64_t rw, double* dst) {
    #pragma omp parallel for
    for (int64_t y = 0; y < sh; y++) {
        for (int64_t x = 0; x < rw; x++) {
            float approx = (float)x * (float)sw / (float)rw;
            int64_t b = (int64_t)approx;
            const double* row = src + y * sw;
            double v1 = row[b];
            double v0 = b - 1 >= 0 ? row[b - 1] : v1;
            double v2 = b + 1 < sw ? row[b + 1] : v1;
            double v3 = b + 2 < sw ? row[b + 2] : v2;
            dst[x * sh + y] = hermite(v1, (v2 - v0) / 2, v2, (v3 - v1) / 2, (double)(approx - (float)b));
        }
    }
}

/* Converter::convert (vshipColor.hpp:62-146): raw planes -> linear RGB, planar, at the
 * final (resized, cropped) size; in BT.709 primaries (destination linRGBBT709), or in the
 * clip's own primaries when `native` (destination linRGB, used by CVVDP,
 * src/cvvdp/main.hpp:188).  Returns 0, or 1 for an unsupported subsampling. */
static int convert_impl(const uint8_t* const planes[3], const int64_t linesize[3],
                        const Vship_Colorspace_t* cs, int native, double* out) {
    const int64_t W = cs->width, H = cs->height;
    const int subw = cs->subsampling.subw, subh = cs->subsampling.subh;
    if (subw < 0 || subw > 2 || subh < 0 || subh > 1) return 1;
    const int64_t N = W * H;
    double* full = (double*)malloc(sizeof(double) * 3 * N);
    for (int c = 0; c < 3; c++) {
        int64_t pw = c ? ((W - 1) >> subw) + 1 : W, ph = c ? ((H - 1) >> subh) + 1 : H;
        int chroma = c != 0 && cs->colorFamily == Vship_ColorYUV;
        double* dec = (c && (subw || subh)) ? (double*)malloc(sizeof(double) * pw * ph) : full + c * N;
        #pragma omp parallel for
        for (int64_t y = 0; y < ph; y++)
            for (int64_t x = 0; x < pw; x++)
                dec[y * pw + x] = to_full_range(pick_sample(planes[c], linesize[c], x, y, cs->sample), cs->sample, cs->range, chroma);
        if (dec != full + c * N) {
            upsample_plane(dec, pw, ph, W, H, subw, subh, cs->chromaLocation, full + c * N);
            free(dec);
        }
    }
    const int skip_yuv = (cs->transferFunction == Vship_TRC_Linear && cs->YUVMatrix == Vship_MATRIX_RGB);
    #pragma omp parallel for
    for (int64_t i = 0; i < N; i++) {
        double v[3] = {full[i], full[N + i], full[2 * N + i]};
        if (!skip_yuv) {
            gamma_light(v, cs->YUVMatrix);
            transfer(v, cs->transferFunction);
            linear_light(v, cs->YUVMatrix);
        }
        if (!native) primaries_to_709(v, cs->primaries);
        full[i] = v[0]; full[N + i] = v[1]; full[2 * N + i] = v[2];
    }
    const int64_t TW = cs->target_width == -1 ? W : cs->target_width;
    const int64_t TH = cs->target_height == -1 ? H : cs->target_height;
    const int64_t OW = TW - cs->crop.left - cs->crop.right, OH = TH - cs->crop.top - cs->crop.bottom;
    for (int c = 0; c < 3; c++) {
        const double* src = full + c * N;
        double* rs = NULL;
        if (TW != W || TH != H) {
            double* tmp = (double*)malloc(sizeof(double) * TW * H);
            rs = (double*)malloc(sizeof(double) * TW * TH);
            oracle_resize_transpose(src, W, H, TW, tmp);   /* -> TW rows of H */
            oracle_resize_transpose(tmp, H, TW, TH, rs);   /* -> TH rows of TW */
            free(tmp);
            src = rs;
        }
        for (int64_t y = 0; y < OH; y++)
            memcpy(out + c * OW * OH + y * OW, src + (y + cs->crop.top) * TW + cs->crop.left, sizeof(double) * OW);
        free(rs);
    }
    free(full);
    return 0;
}

ORACLE_API int oracle_convert(const uint8_t* const planes[3], const int64_t linesize[3],
                              const Vship_Colorspace_t* cs, double* out) {
    return convert_impl(planes, linesize, cs, 0, out);
}

ORACLE_API int oracle_convert_native(const uint8_t* const planes[3], const int64_t linesize[3],
                                     const Vship_Colorspace_t* cs, double* out) {
    return convert_impl(planes, linesize, cs, 1, out);
}

/* ------------------------------------------------------------------------------------ */
/* Renormalised truncated Gaussian blur (src/ssimu2/gaussianblur.hpp:7-77,                */
/* src/butter/gaussianblur.hpp:3-187): separable; each 1-D pass divides by the sum of   */
/* the taps that fall inside the image.                                                  */
/* ------------------------------------------------------------------------------------ */

static void blur_plane(const double* src, double* dst, int64_t w, int64_t h, double sigma, int r) {
    double g[64];
    for (int i = 0; i <= 2 * r; i++) g[i] = exp(-(double)((r - i) * (r - i)) / (2 * sigma * sigma));
    double* tmp = (double*)malloc(sizeof(double) * w * h);
    #pragma omp parallel for
    for (int64_t y = 0; y < h; y++) {
        for (int64_t x = 0; x < w; x++) {
            double s = 0, n = 0;
            for (int j = -r; j <= r; j++) {
                int64_t xx = x + j;
                if (xx < 0 || xx >= w) continue;
                s += g[j + r] * src[y * w + xx];
                n += g[j + r];
            }
            tmp[y * w + x] = s / n;
        }
    }
    #pragma omp parallel for
    for (int64_t y = 0; y < h; y++) {
        for (int64_t x = 0; x < w; x++) {
            double s = 0, n = 0;
            for (int j = -r; j <= r; j++) {
                int64_t yy = y + j;
                if (yy < 0 || yy >= h) continue;
                s += g[j + r] * tmp[yy * w + x];
                n += g[j + r];
            }
            dst[y * w + x] = s / n;
        }
    }
    free(tmp);
}

/* 2x2 box average with edge clamp, output ((w-1)/2+1) x ((h-1)/2+1)
 * (src/ssimu2/downsample.hpp:3-19, src/butter/downupsample.hpp:4-20). */
static void downsample2(const double* src, int64_t w, int64_t h, double* dst) {
    int64_t nw = (w - 1) / 2 + 1, nh = (h - 1) / 2 + 1;
    #pragma omp parallel for
    for (int64_t y = 0; y < nh; y++) {
        int64_t y0 = imin64(2 * y, h - 1), y1 = imin64(2 * y + 1, h - 1);
        for (int64_t x = 0; x < nw; x++) {
            int64_t x0 = imin64(2 * x, w - 1), x1 = imin64(2 * x + 1, w - 1);
            dst[y * nw + x] = 0.25 * (src[y0 * w + x0] + src[y1 * w + x0] + src[y0 * w + x1] + src[y1 * w + x1]);
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* SSIMULACRA2 (src/ssimu2/main.hpp:16-78, makeXYB.hpp:6-47, score.hpp:116-460)         */
/* ------------------------------------------------------------------------------------ */

/* rgb_to_positive_xyb_d (makeXYB.hpp:6-47). */
static void positive_xyb(double v[3]) {
    const double bias = 0.0037930734, absb = -0.1559542025327239;
    double l = 0.30 * v[0] + 0.622 * v[1] + 0.078 * v[2] + bias;
    double m = 0.23 * v[0] + 0.692 * v[1] + 0.078 * v[2] + bias;
    double s = 0.24342269 * v[0] + 0.20476745 * v[1] + 0.55180986 * v[2] + bias;
    l = cbrt(l >= 0 ? l : 0) + absb;
    m = cbrt(m >= 0 ? m : 0) + absb;
    s = cbrt(s >= 0 ? s : 0) + absb;
    double X = 0.5 * (l - m), Y = X + m, B = s;
    v[2] = (B - Y) + 0.55;
    v[0] = X * 14.0 + 0.42;
    v[1] = Y + 0.01;
}

static int ssimu2_map_on(int plane, int scale, int map) {
    return kSsimu2Weights[plane * 36 + scale * 6 + map] > VSHIP_SSIMU2_PRUNE ||
           kSsimu2Weights[plane * 36 + scale * 6 + 3 + map] > VSHIP_SSIMU2_PRUNE;
}

/* Maps and norms of one (plane, scale) (planescale_map_Kernel, score.hpp:192-322):
 * means of ssim, artifact, detail-loss and of their 4th powers. */
static void ssimu2_planescale(const double* a, const double* b, int64_t w, int64_t h,
                              int do_ssim, int do_art, int do_det, double out[6]) {
    const int64_t n = w * h;
    double* prod = (double*)malloc(sizeof(double) * n * 8);
    double *ab = prod, *sq = prod + n, *m1 = prod + 2 * n, *m2 = prod + 3 * n;
    double *s12 = prod + 4 * n, *ssq = prod + 5 * n;
    for (int64_t i = 0; i < n; i++) { ab[i] = a[i] * b[i]; sq[i] = (a[i] + b[i]) * (a[i] + b[i]); }
    blur_plane(a, m1, w, h, 1.5, 8);
    blur_plane(b, m2, w, h, 1.5, 8);
    if (do_ssim) { blur_plane(ab, s12, w, h, 1.5, 8); blur_plane(sq, ssq, w, h, 1.5, 8); }
    double acc[6] = {0, 0, 0, 0, 0, 0};
    #pragma omp parallel
    {
        double loc[6] = {0, 0, 0, 0, 0, 0};
        #pragma omp for
        for (int64_t i = 0; i < n; i++) {
            double ssim = 0, art = 0, det = 0;
            if (do_ssim) {
                double s11s22 = ssq[i] - 2 * s12[i];
                double num_m = 1.0 - (m1[i] - m2[i]) * (m1[i] - m2[i]);
                double num_s = 2 * (s12[i] - m1[i] * m2[i]) + 0.0009;
                double den_s = s11s22 - m1[i] * m1[i] - m2[i] * m2[i] + 0.0009;
                ssim = 1.0 - num_m * num_s / den_s;
                if (ssim < 0) ssim = 0;
            }
            if (do_art || do_det) {
                double v1 = (fabs(b[i] - m2[i]) + 1.0) / (fabs(a[i] - m1[i]) + 1.0) - 1.0;
                if (do_art) art = v1 > 0 ? v1 : 0;
                if (do_det) det = -v1 > 0 ? -v1 : 0;
            }
            loc[0] += ssim; loc[1] += art; loc[2] += det;
            loc[3] += ssim * ssim * ssim * ssim; loc[4] += art * art * art * art; loc[5] += det * det * det * det;
        }
        #pragma omp critical
        for (int k = 0; k < 6; k++) acc[k] += loc[k];
    }
    for (int k = 0; k < 6; k++) out[k] = acc[k] / (double)n;
    free(prod);
}

/* final_score (score.hpp:442-460).  quirk != 0 reproduces the reference exactly: the
 * weighted sum goes through float fmaf and the result is returned as float. */
static double ssimu2_final(const double f[108], int quirk) {
    double s = 0.0;
    for (int i = 0; i < 108; i++) {
        if (quirk) s = (double)fmaf((float)kSsimu2Weights[i], (float)f[i], (float)s);
        else s += kSsimu2Weights[i] * f[i];
    }
    s *= VSHIP_SSIMU2_SCALE;
    s = (VSHIP_SSIMU2_C3 * s * s) * s + VSHIP_SSIMU2_C1 * s - VSHIP_SSIMU2_C2 * s * s;
    s = s > 0.0 ? pow(s, VSHIP_SSIMU2_EXP) * -10.0 + 100.0 : 100.0;
    return quirk ? (double)(float)s : s;
}

/* ssimu2GPUProcess (main.hpp:27-78) on planar linear RGB inputs of w x h. */
ORACLE_API void oracle_ssimu2(const double* rgb1, const double* rgb2, int64_t w, int64_t h,
                              double* features, double* score_quirk, double* score_double) {
    double* lv[2][6][3];
    int64_t ws[6], hs[6];
    ws[0] = w; hs[0] = h;
    for (int s = 1; s < 6; s++) { ws[s] = (ws[s - 1] - 1) / 2 + 1; hs[s] = (hs[s - 1] - 1) / 2 + 1; }
    for (int im = 0; im < 2; im++) {
        const double* rgb = im ? rgb2 : rgb1;
        for (int s = 0; s < 6; s++)
            for (int c = 0; c < 3; c++) {
                lv[im][s][c] = (double*)malloc(sizeof(double) * ws[s] * hs[s]);
                if (s == 0) memcpy(lv[im][0][c], rgb + c * w * h, sizeof(double) * w * h);
                else downsample2(lv[im][s - 1][c], ws[s - 1], hs[s - 1], lv[im][s][c]);
            }
        for (int s = 0; s < 6; s++) {
            int64_t n = ws[s] * hs[s];
            #pragma omp parallel for
            for (int64_t i = 0; i < n; i++) {
                double v[3] = {lv[im][s][0][i], lv[im][s][1][i], lv[im][s][2][i]};
                positive_xyb(v);
                lv[im][s][0][i] = v[0]; lv[im][s][1][i] = v[1]; lv[im][s][2][i] = v[2];
            }
        }
    }
    double f[108];
    memset(f, 0, sizeof(f));
    for (int s = 0; s < 6; s++) {
        for (int p = 0; p < 3; p++) {
            int on[3] = {ssimu2_map_on(p, s, 0), ssimu2_map_on(p, s, 1), ssimu2_map_on(p, s, 2)};
            if (!on[0] && !on[1] && !on[2]) continue;
            double o[6];
            ssimu2_planescale(lv[0][s][p], lv[1][s][p], ws[s], hs[s], on[0], on[1], on[2], o);
            for (int k = 0; k < 3; k++) {
                f[p * 36 + s * 6 + k] = o[k];
                f[p * 36 + s * 6 + 3 + k] = on[k] ? sqrt(sqrt(o[3 + k])) : o[3 + k];
            }
        }
    }
    for (int im = 0; im < 2; im++)
        for (int s = 0; s < 6; s++)
            for (int c = 0; c < 3; c++) free(lv[im][s][c]);
    if (features) memcpy(features, f, sizeof(f));
    if (score_quirk) *score_quirk = ssimu2_final(f, 1);
    if (score_double) *score_double = ssimu2_final(f, 0);
}

/* Score from an externally supplied feature vector (used to test final_score alone). */
ORACLE_API double oracle_ssimu2_final(const double* features, int quirk) { return ssimu2_final(features, quirk); }

/* ------------------------------------------------------------------------------------ */
/* Butteraugli (src/butter/*.hpp)                                                        */
/* ------------------------------------------------------------------------------------ */

static void butter_opsin_mix(const double in[3], double out[3]) {  /* colors.hpp:33-56 */
    out[0] = 0.29956550340058319 * in[0] + 0.63373087833825936 * in[1] + 0.077705617820981968 * in[2] + 1.7557483643287353;
    out[1] = 0.22158691104574774 * in[0] + 0.69391388044116142 * in[1] + 0.0987313588422 * in[2] + 1.7557483643287353;
    out[2] = 0.02 * in[0] + 0.02 * in[1] + 0.20480129041026129 * in[2] + 12.226454707163354;
}

static double butter_gamma(double v) { return 19.245013259874995 * log(v + 9.9710635769299145) - 23.16046239805755; }

/* opsinDynamicsImage (colors.hpp:57-91): rgb planes -> XYB planes (in place). */
static void butter_opsin(double* rgb, int64_t w, int64_t h, double intensity) {
    const int64_t n = w * h;
    double* bl = (double*)malloc(sizeof(double) * 3 * n);
    for (int c = 0; c < 3; c++) blur_plane(rgb + c * n, bl + c * n, w, h, kButterSigma[0], kButterRadius[0]);
    #pragma omp parallel for
    for (int64_t i = 0; i < n; i++) {
        double src[3] = {rgb[i] * intensity, rgb[n + i] * intensity, rgb[2 * n + i] * intensity};
        double b[3] = {bl[i] * intensity, bl[n + i] * intensity, bl[2 * n + i] * intensity};
        double ob[3], os[3], sens[3];
        butter_opsin_mix(b, ob);
        ob[0] = fmax(ob[0], 1.7557483643287353); ob[1] = fmax(ob[1], 1.7557483643287353); ob[2] = fmax(ob[2], 12.226454707163354);
        for (int k = 0; k < 3; k++) {
            ob[k] = fmax(ob[k], 1e-4);
            sens[k] = fmax(butter_gamma(ob[k]) / ob[k], 1e-4);
        }
        butter_opsin_mix(src, os);
        for (int k = 0; k < 3; k++) os[k] *= sens[k];
        os[0] = fmax(os[0], 1.7557483643287353); os[1] = fmax(os[1], 1.7557483643287353); os[2] = fmax(os[2], 12.226454707163354);
        rgb[i] = os[0] - os[1];
        rgb[n + i] = os[0] + os[1];
        rgb[2 * n + i] = os[2];
    }
    free(bl);
}

static double remove_range(double x, double w) { return x > w ? x - w : (x < -w ? x + w : 0.0); }   /* separatefrequencies.hpp:49-51 */
static double amplify_range(double x, double w) { return x > w ? x + w : (x < -w ? x - w : 2.0 * x); } /* :44-46 */
static double maximum_clamp(double v, double maxval) {                                            /* :24-35 */
    const double k = 0.688059627878;
    if (v >= maxval) return (v - maxval) * k + maxval;
    if (v < -maxval) return (v + maxval) * k - maxval;
    return v;
}

typedef struct { double *lf[3], *mf[3], *hf[2], *uhf[2]; } bands;

/* separateFrequencies (separatefrequencies.hpp:160-203). */
static void butter_separate(const double* xyb, int64_t w, int64_t h, bands* o) {
    const int64_t n = w * h;
    double* d = (double*)malloc(sizeof(double) * n);
    for (int c = 0; c < 3; c++) {
        o->lf[c] = (double*)malloc(sizeof(double) * n);
        o->mf[c] = (double*)malloc(sizeof(double) * n);
        blur_plane(xyb + c * n, o->lf[c], w, h, kButterSigma[4], kButterRadius[4]);
        for (int64_t i = 0; i < n; i++) d[i] = xyb[c * n + i] - o->lf[c][i];
        blur_plane(d, o->mf[c], w, h, kButterSigma[3], kButterRadius[3]);
        if (c == 2) break;
        o->uhf[c] = (double*)malloc(sizeof(double) * n);   /* holds hf before its own blur */
        for (int64_t i = 0; i < n; i++) {
            o->uhf[c][i] = d[i] - o->mf[c][i];
            o->mf[c][i] = c == 0 ? remove_range(o->mf[c][i], 0.29) : amplify_range(o->mf[c][i], 0.1);
        }
    }
    for (int64_t i = 0; i < n; i++) {                      /* supressXbyY, :37-41 */
        const double s = 0.653020556257, yw = 46.0;
        double yv = o->uhf[1][i];
        o->uhf[0][i] *= s + (yw * (1.0 - s)) / (yw + yv * yv);
    }
    for (int c = 0; c < 2; c++) {
        o->hf[c] = (double*)malloc(sizeof(double) * n);
        blur_plane(o->uhf[c], o->hf[c], w, h, kButterSigma[1], kButterRadius[1]);
        for (int64_t i = 0; i < n; i++) {
            double hf = o->hf[c][i], uhf = o->uhf[c][i];
            if (c == 0) {
                uhf -= hf;
                hf = remove_range(hf, 1.5);
                uhf = remove_range(uhf, 0.04);
            } else {                                       /* separateHf_Uhf_Kernel, :117-133 */
                hf = maximum_clamp(hf, 28.4691806922);
                uhf -= hf;
                uhf = maximum_clamp(uhf, 5.19175294647);
                uhf *= 2.69313763794;
                hf *= 2.155;
                hf = amplify_range(hf, 0.132);
            }
            o->hf[c][i] = hf; o->uhf[c][i] = uhf;
        }
    }
    for (int64_t i = 0; i < n; i++) {                      /* XybLowFreqToVals, :3-12 */
        double x = o->lf[0][i], y = o->lf[1][i], b = o->lf[2][i];
        b = (b + -0.362267051518 * y) * 49.87984651440;
        o->lf[0][i] = x * 33.832837186260;
        o->lf[1][i] = y * 14.458268100570;
        o->lf[2][i] = b;
    }
    free(d);
}

static void free_bands(bands* b) {
    for (int c = 0; c < 3; c++) { free(b->lf[c]); free(b->mf[c]); }
    for (int c = 0; c < 2; c++) { free(b->hf[c]); free(b->uhf[c]); }
}

/* MaltaDiffMap / MaltaDiffMapLF (maltaDiff.hpp:514-684), accumulated into acc. */
static void butter_malta(const double* l0, const double* l1, double* acc, int64_t w, int64_t h,
                         double w0gt1, double w0lt1, double norm1, int lf) {
    const double len = 3.75, mulli = lf ? 0.611612573796 : 0.39905817637;
    const double len2 = len * 2.0 + 1.0;
    const double n2gt = mulli * sqrt(0.5 * w0gt1) / len2 * norm1;
    const double n2lt = mulli * sqrt(0.33 * w0lt1) / len2 * norm1;
    const int64_t n = w * h;
    double* d = (double*)malloc(sizeof(double) * n);
    #pragma omp parallel for
    for (int64_t i = 0; i < n; i++) {
        double a = l0[i], b = l1[i];
        double absval = 0.5 * fabs(a) + 0.5 * fabs(b);
        double diff = a - b;
        double v = n2gt / (norm1 + absval) * diff;
        double sc2 = n2lt / (norm1 + absval);
        double ts = 0.55 * fabs(a), tb = 1.05 * fabs(a), impact = 0.0;
        if (a < 0.0) {
            if (b > -ts) impact = b + ts;
            else if (b < -tb) impact = -b - tb;
        } else {
            if (b < ts) impact = -b + ts;
            else if (b > tb) impact = b - tb;
        }
        impact *= sc2;
        d[i] = diff < 0.0 ? v - impact : v + impact;
    }
    #pragma omp parallel for
    for (int64_t y = 0; y < h; y++) {
        for (int64_t x = 0; x < w; x++) {
            double r = 0.0;
            for (int p = 0; p < 16; p++) {
                double s = 0.0;
                int ntaps = lf ? 5 : 9;
                for (int t = 0; t < ntaps; t++) {
                    vship_malta_tap tp = lf ? kMaltaLF[p][t] : kMaltaHF[p][t];
                    if (tp.dx == VSHIP_MALTA_PAD) continue;
                    int64_t xx = x + tp.dx, yy = y + tp.dy;
                    if (xx < 0 || xx >= w || yy < 0 || yy >= h) continue;
                    s += d[yy * w + xx];
                }
                r += s * s;
            }
            acc[y * w + x] += r;
        }
    }
    free(d);
}

static void butter_l2(const double* a, const double* b, double* acc, int64_t n, double wt) {   /* simplerdiff.hpp:44-61 */
    if (wt == 0) return;
    for (int64_t i = 0; i < n; i++) { double d = a[i] - b[i]; acc[i] += wt * d * d; }
}

static void butter_l2asym(const double* a, const double* b, double* acc, int64_t n, double wgt, double wlt) { /* :63-101 */
    if (wgt == 0.0 && wlt == 0.0) return;
    wgt *= 0.8; wlt *= 0.8;
    for (int64_t i = 0; i < n; i++) {
        double d = a[i] - b[i];
        acc[i] += wgt * d * d;
        double f0 = fabs(a[i]), ts = 0.4 * f0, tb = f0;
        if (a[i] < 0) {
            if (b[i] > -ts) { double v = b[i] + ts; acc[i] += wlt * v * v; }
            else if (b[i] < -tb) { double v = -b[i] - tb; acc[i] += wlt * v * v; }
        } else {
            if (b[i] < ts) { double v = ts - b[i]; acc[i] += wlt * v * v; }
            else if (b[i] > tb) { double v = b[i] - tb; acc[i] += wlt * v * v; }
        }
    }
}

static void store_min3(double v, double* m0, double* m1, double* m2) {   /* maskPsycho.hpp:42-55 */
    if (v < *m2) {
        if (v < *m0) { *m2 = *m1; *m1 = *m0; *m0 = v; }
        else if (v < *m1) { *m2 = *m1; *m1 = v; }
        else *m2 = v;
    }
}

/* fuzzyerrosion_Kernel (maskPsycho.hpp:57-104). */
static void fuzzy_erosion(const double* src, double* dst, int64_t w, int64_t h) {
    const int64_t k = 3;
    #pragma omp parallel for
    for (int64_t y = 0; y < h; y++) {
        for (int64_t x = 0; x < w; x++) {
            double m0 = src[y * w + x], m1 = 2.0 * m0, m2 = m1;
            if (x >= k) {
                store_min3(src[y * w + x - k], &m0, &m1, &m2);
                if (y >= k) store_min3(src[(y - k) * w + x - k], &m0, &m1, &m2);
                if (y < h - k) store_min3(src[(y + k) * w + x - k], &m0, &m1, &m2);
            }
            if (x < w - k) {
                store_min3(src[y * w + x + k], &m0, &m1, &m2);
                if (y >= k) store_min3(src[(y - k) * w + x + k], &m0, &m1, &m2);
                if (y < h - k) store_min3(src[(y + k) * w + x + k], &m0, &m1, &m2);
            }
            if (y >= k) store_min3(src[(y - k) * w + x], &m0, &m1, &m2);
            if (y < h - k) store_min3(src[(y + k) * w + x], &m0, &m1, &m2);
            dst[y * w + x] = 0.45 * m0 + 0.3 * m1 + 0.25 * m2;
        }
    }
}

static double mask_y(double delta) {                       /* combineMasks.hpp:3-11 */
    double c = 2.5485944793 / (0.451936922203 * delta + 0.829591754942);
    double r = (1.0 + c) * (1.0 / (0.79079917404 * 17.83));
    return r * r;
}

static double mask_dc_y(double delta) {                    /* combineMasks.hpp:13-20 */
    double c = 0.505054525019 / (3.87449418804 * delta + 0.20025578522);
    double r = (1.0 + c) * (1.0 / (0.79079917404 * 17.83));
    return r * r;
}

/* getdiffmap (butter/main.hpp:25-115): one scale, inputs are linear RGB planes. */
static void butter_diffmap_scale(const double* rgb1, const double* rgb2, int64_t w, int64_t h,
                                 double intensity, double* out) {
    const int64_t n = w * h;
    double* x1 = (double*)malloc(sizeof(double) * 3 * n);
    double* x2 = (double*)malloc(sizeof(double) * 3 * n);
    memcpy(x1, rgb1, sizeof(double) * 3 * n);
    memcpy(x2, rgb2, sizeof(double) * 3 * n);
    butter_opsin(x1, w, h, intensity);
    butter_opsin(x2, w, h, intensity);
    bands b1, b2;
    butter_separate(x1, w, h, &b1);
    butter_separate(x2, w, h, &b2);
    double* ac = (double*)calloc(3 * n, sizeof(double));
    double* dc = (double*)calloc(3 * n, sizeof(double));
    const double asym = 0.8;
    butter_malta(b1.uhf[1], b2.uhf[1], ac + n, w, h, 1.10039032555 * asym, 1.10039032555 / asym, 71.7800275169, 0);
    butter_malta(b1.uhf[0], b2.uhf[0], ac, w, h, 173.5 * asym, 173.5 / asym, 5.0, 0);
    butter_malta(b1.hf[1], b2.hf[1], ac + n, w, h, 18.7237414387 * sqrt(asym), 18.7237414387 / sqrt(asym), 4498534.45232, 1);
    butter_malta(b1.hf[0], b2.hf[0], ac, w, h, 6923.99476109 * sqrt(asym), 6923.99476109 / sqrt(asym), 8051.15833247, 1);
    butter_malta(b1.mf[1], b2.mf[1], ac + n, w, h, 37.0819870399, 37.0819870399, 130262059.556, 1);
    butter_malta(b1.mf[0], b2.mf[0], ac, w, h, 8246.75321353, 8246.75321353, 1009002.70582, 1);
    const double wmul[9] = {400.0, 1.50815703118, 0.0, 2150.0, 10.6195433239, 16.2176043152,
                            29.2353797994, 0.844626970982, 0.703646627719};
    for (int c = 0; c < 3; c++) {
        if (c < 2) butter_l2asym(b1.hf[c], b2.hf[c], ac + c * n, n, wmul[c] * asym, wmul[c] / asym);
        butter_l2(b1.mf[c], b2.mf[c], ac + c * n, n, wmul[3 + c]);
        butter_l2(b1.lf[c], b2.lf[c], dc + c * n, n, wmul[6 + c]);
    }
    /* MaskPsychoImage (maskPsycho.hpp:113-135) */
    double* m0 = (double*)malloc(sizeof(double) * n);
    double* m1 = (double*)malloc(sizeof(double) * n);
    double* bl0 = (double*)malloc(sizeof(double) * n);
    double* bl1 = (double*)malloc(sizeof(double) * n);
    double* mask = (double*)malloc(sizeof(double) * n);
    const double mul = 6.19424080439, bias = 6.19424080439 * 12.61050594197;
    for (int64_t i = 0; i < n; i++) {
        double xd = (b1.uhf[0][i] + b1.hf[0][i]) * 2.5, yd = b1.uhf[1][i] * 0.4 + b1.hf[1][i] * 0.4;
        double mk = sqrt(xd * xd + yd * yd);
        m0[i] = sqrt(mul * fabs(mk) + bias) - sqrt(bias);
        xd = (b2.uhf[0][i] + b2.hf[0][i]) * 2.5; yd = b2.uhf[1][i] * 0.4 + b2.hf[1][i] * 0.4;
        mk = sqrt(xd * xd + yd * yd);
        m1[i] = sqrt(mul * fabs(mk) + bias) - sqrt(bias);
    }
    blur_plane(m0, bl0, w, h, kButterSigma[2], kButterRadius[2]);
    blur_plane(m1, bl1, w, h, kButterSigma[2], kButterRadius[2]);
    fuzzy_erosion(bl0, mask, w, h);
    butter_l2(bl0, bl1, ac + n, n, 10.0);
    for (int64_t i = 0; i < n; i++) {                      /* computeDiffmap_Kernel, combineMasks.hpp:22-33 */
        double sac = ac[i] + ac[n + i] + ac[2 * n + i];
        double sdc = dc[i] + dc[n + i] + dc[2 * n + i];
        out[i] = sqrt(mask_y(mask[i]) * sac + mask_dc_y(mask[i]) * sdc);
    }
    free(m0); free(m1); free(bl0); free(bl1); free(mask);
    free(ac); free(dc);
    free_bands(&b1); free_bands(&b2);
    free(x1); free(x2);
}

/* butterprocess (butter/main.hpp:118-181, diffnorms.hpp:86-130): two scales, supersampled
 * combination, then the Q-norm, 3-norm and max norm of the distortion map. */
ORACLE_API void oracle_butteraugli(const double* rgb1, const double* rgb2, int64_t w, int64_t h,
                                   double intensity, int qnorm, double* distmap, double norms[3]) {
    const int64_t n = w * h, nw = (w - 1) / 2 + 1, nh = (h - 1) / 2 + 1, nn = nw * nh;
    double* s1 = (double*)malloc(sizeof(double) * 3 * nn);
    double* s2 = (double*)malloc(sizeof(double) * 3 * nn);
    for (int c = 0; c < 3; c++) {
        downsample2(rgb1 + c * n, w, h, s1 + c * nn);
        downsample2(rgb2 + c * n, w, h, s2 + c * nn);
    }
    double* d0 = distmap ? distmap : (double*)malloc(sizeof(double) * n);
    double* d1 = (double*)malloc(sizeof(double) * nn);
    butter_diffmap_scale(rgb1, rgb2, w, h, intensity, d0);
    butter_diffmap_scale(s1, s2, nw, nh, intensity, d1);
    for (int64_t y = 0; y < h; y++)                        /* addsupersample2X_kernel, downupsample.hpp:35-55 */
        for (int64_t x = 0; x < w; x++)
            d0[y * w + x] = d0[y * w + x] * (1.0 - 0.3 * 0.5) + 0.5 * d1[(y / 2) * nw + x / 2];
    double sq = 0, s3 = 0, mx = 0;
    for (int64_t i = 0; i < n; i++) {
        double v = fabs(d0[i]);
        sq += pow(v, (double)qnorm);
        s3 += v * v * v;
        if (v > mx) mx = v;
    }
    norms[0] = pow(sq / (double)n, 1.0 / (double)qnorm);
    norms[1] = pow(s3 / (double)n, 1.0 / 3.0);
    norms[2] = mx;
    if (!distmap) free(d0);
    free(d1); free(s1); free(s2);
}

/* Exposed stage helpers for unit tests of the restatement itself. */
ORACLE_API void oracle_blur(const double* src, double* dst, int64_t w, int64_t h, double sigma, int radius) {
    blur_plane(src, dst, w, h, sigma, radius);
}

ORACLE_API void oracle_downsample(const double* src, int64_t w, int64_t h, double* dst) { downsample2(src, w, h, dst); }

/* Planar linear RGB (3 planes of n samples) to positive XYB, in place. */
ORACLE_API void oracle_positive_xyb(double* planes, int64_t n) {
    for (int64_t i = 0; i < n; i++) {
        double v[3] = {planes[i], planes[n + i], planes[2 * n + i]};
        positive_xyb(v);
        planes[i] = v[0];
        planes[n + i] = v[1];
        planes[2 * n + i] = v[2];
    }
}

ORACLE_API int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

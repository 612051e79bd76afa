// CVVDP on the B200: the reference's ColorVideoVDP variant (src/cvvdp/*.hpp) as a handful
// of fused kernels per frame pair.
//
//   cv_ingest     raw planes -> linear RGB (clip primaries) -> display model -> XYZ -> DKL,
//                 both clips in one launch, written into the ring slot of the new frame
//                 (main.hpp:234-347, colors.hpp)
//   cv_temporal   the ring convolved with the four temporal filters: Y sustained, RG, YV,
//                 Y transient at pyramid level 0 (temporalFilter.hpp:150-193)
//   cv_reduce     one Gaussian pyramid step of all eight planes (two clips x four
//                 channels) per launch (lpyr.hpp:7-36)
//   cv_contrast   one Laplacian band of both clips: expansion of the next level, contrast
//                 against the background luminance, CSF weighting; writes the masking input
//                 min(|R|,|T|) and |R-T| per channel (lpyr.hpp:177-236, csf.hpp,
//                 maskingModel.hpp:5-15)
//   cv_mask       the sigma-3 masking blur, cross-channel masking, the saturating D and
//                 per-tile FP64 sums of D^2; one 32x32 tile per CTA (maskingModel.hpp:28-96)
//   cv_pool       pooled norm of every band and channel (pooling.hpp), the last CTA doing the
//                 baseband: mean luminance, contrast, D (lpyr.hpp:219-229,
//                 maskingModel.hpp:106-114)
// The score of the sequence (pooling over bands, channels and frames, JOD) is formed on the
// host from 4 x bands doubles, as the reference does (main.hpp:135-158, 376-388).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "colour.cuh"
#include "frontend.cuh"
#include "engines.h"
#include "cvvdp_csf_table.h"

namespace vship {
namespace cvvdp {
namespace {

// ---- model constants (src/cvvdp/parameters.hpp:5-68) ---------------------------------------
constexpr double kPi = 3.14159265359;  // the reference's PI (src/util/preprocessor.hpp:83)
constexpr float kMaskP = 2.264355182647705f;
constexpr float kMaskC = -0.7954971194267273f;
constexpr float kSensitivityCorrection = -0.2797423303127289f;
constexpr float kJodA = 0.0439569391310215f;
constexpr float kJodExp = 0.9302042722702026f;
__device__ constexpr float kMaskQ[4] = {1.302622675895691f, 2.8885908126831055f, 3.6807713508605957f, 3.588787317276001f};
constexpr float kChTransW = 0.8081134557723999f;  // ch_chrom_w is 1
constexpr float kSigmaTf[4] = {5.79336f, 14.1255f, 6.63661f, 0.12314f};
constexpr float kBetaTf[4] = {1.3314f, 1.1196f, 0.947901f, 0.1898f};
constexpr float kXcmWeights[16] = {
    -0.18950104713439941f, -5.962151050567627f, -4.31834602355957f, -1.9321587085723877f,
    2.5655593872070312f,   0.34406712651252747f, -2.719646453857422f, -0.4970424771308899f,
    3.8118371963500977f,   -1.0051705837249756f, -0.5193376541137695f, -0.5653647780418396f,
    -7.054771423339844f,   -5.527150630950928f, -3.5106418132781982f, -2.08804988861084f};
__device__ constexpr float kBasebandWeight[4] = {0.0036334486212581396f, 1.6627724170684814f, 4.11874532699585f, 25.25969886779785f};
constexpr float kDMax = 2.5642454624176025f;
constexpr float kImageInt = 0.577918291091919f;
constexpr int kMaxLevels = 14;

// Pyramid kernel [0.25 - a/2, 0.25, a, 0.25, 0.25 - a/2] with a = 0.4 (lpyr.hpp:5-6).
__device__ __forceinline__ float pyr_k(int i) {
    constexpr float a = 0.4f;
    constexpr float e = (float)(0.25 - a / 2.);
    return i == 2 ? a : ((i == 1 || i == 3) ? 0.25f : e);
}

// Display parameters applied to every pixel (colors.hpp:98-117).
struct DisplayDev {
    float peak, black, refl, exposure;
    int hdr;
};

__device__ __forceinline__ float display_encode(float a, const DisplayDev& d, int trc) {
    if (d.hdr && trc == Vship_TRC_PQ) {
        a *= 100.f;
        return fmaxf(fmaxf(0.005f, d.black), fminf(d.peak, a * d.exposure)) + d.black + d.refl;
    }
    if (d.hdr && trc == Vship_TRC_Linear) return fmaxf(fmaxf(0.005f, d.black), fminf(d.peak, a * d.exposure)) + d.refl;
    return (d.peak - d.black) * fmaxf(0.f, fminf(1.f, a * d.exposure)) + d.black + d.refl;
}

// XYZ -> LMS (CIE 2006) -> DKL d65 (colors.hpp:30-49).
__device__ __forceinline__ float3 xyz_to_dkl(float3 a) {
    const float l = fmaf(0.187596268556126f, a.x, fmaf(0.585168649077728f, a.y, -0.026384263306304f * a.z));
    const float m = fmaf(-0.133397430663221f, a.x, fmaf(0.405505777260049f, a.y, 0.034502127690364f * a.z));
    const float s = fmaf(0.000244379021663f, a.x, fmaf(-0.000542995890619f, a.y, 0.019406849066323f * a.z));
    const float ach = l + m;
    return make_float3(ach, fmaf(-3.311130179947035f, m, ach), fmaf(50.977571328718781f, s, -ach));
}

__device__ __forceinline__ float3 encode_pixel(float3 lin, const DisplayDev& d, int trc, int prim) {
    lin.x = display_encode(lin.x, d, trc);
    lin.y = display_encode(lin.y, d, trc);
    lin.z = display_encode(lin.z, d, trc);
    return xyz_to_dkl(rgb_to_xyz(lin, prim));
}

// ---- ingest ------------------------------------------------------------------------------

struct IngestParams {
    RawImage im[2];
    ColourParams cp[2];
    float* slot[2];  // ring slot of the new frame: 3 planes of n floats
    int64_t n;
    int trc[2], prim[2];
    DisplayDev disp;
};

// Raw planes straight to the ring (no resize or crop): one 64x64 tile of one clip per CTA,
// chroma staged in shared memory as in the other metrics' fronts.
// kFast selects a compile-time pixel path (colour.cuh) when both clips use it; those paths
// are BT.709-primaries formats, whose native linear RGB is the BT.709 one they produce.
template <int kFast>
__global__ void __launch_bounds__(256, 3) cv_ingest_kernel(const __grid_constant__ IngestParams p) {
    extern __shared__ float stage_mem[];
    const int k = blockIdx.z;
    const ColourParams& cp = p.cp[k];
    const int X0 = blockIdx.x * kStageTile, Y0 = blockIdx.y * kStageTile;
    if (X0 >= cp.W || Y0 >= cp.H) return;
    ChromaStage st{};
    if (cp.subw || cp.subh) chroma_stage<kFast>(p.im[k], cp, X0, Y0, stage_mem, st);
    float* out = p.slot[k];
    if constexpr (kFast == kFastYuv420Bt709) {
        // One 2x2 quad per work item: the quad's chroma rows and luma pairs are read together
        // (ingest_quad_yuv420), the same values as four single-pixel reads.
        for (int q = threadIdx.x; q < kStageTile * kStageTile / 4; q += blockDim.x) {
            const int X = X0 + 2 * (q & (kStageTile / 2 - 1)), Y = Y0 + 2 * (q / (kStageTile / 2));
            if (X >= cp.W || Y >= cp.H) continue;
            const bool right = X + 1 < cp.W, down = Y + 1 < cp.H;
            float3 lin[4];
            ingest_quad_yuv420(p.im[k], cp, st, X, Y, X0, Y0, right, down, lin);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                if (((e & 1) && !right) || ((e & 2) && !down)) continue;
                const float3 v = encode_pixel(lin[e], p.disp, p.trc[k], p.prim[k]);
                const int64_t o = (int64_t)(Y + (e >> 1)) * cp.W + X + (e & 1);
                out[o] = v.x;
                out[p.n + o] = v.y;
                out[2 * p.n + o] = v.z;
            }
        }
        return;
    }
    for (int i = threadIdx.x; i < kStageTile * kStageTile; i += blockDim.x) {
        const int X = X0 + (i & (kStageTile - 1)), Y = Y0 + i / kStageTile;
        if (X >= cp.W || Y >= cp.H) continue;
        float3 lin;
        if constexpr (kFast == kFastGeneric) lin = ingest_staged<true>(p.im[k], cp, st, X, Y, X0, Y0);
        else lin = ingest_fast<kFast>(p.im[k], cp, st, X, Y, X0, Y0);
        const float3 v = encode_pixel(lin, p.disp, p.trc[k], p.prim[k]);
        const int64_t o = (int64_t)Y * cp.W + X;
        out[o] = v.x;
        out[p.n + o] = v.y;
        out[2 * p.n + o] = v.z;
    }
}

struct EncodeParams {
    const float* src[2];  // linear RGB planes (clip primaries)
    int64_t pitch[2], plane[2];
    float* slot[2];
    int64_t w, h;
    int trc[2], prim[2];
    DisplayDev disp;
};

// Linear planes (after resize / crop) to the ring.
__global__ void cv_encode_kernel(const __grid_constant__ EncodeParams p) {
    const int k = blockIdx.y;
    const int64_t n = p.w * p.h;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = i % p.w, y = i / p.w;
        const float* s = p.src[k] + y * p.pitch[k] + x;
        const float3 v = encode_pixel(make_float3(s[0], s[p.plane[k]], s[2 * p.plane[k]]), p.disp, p.trc[k], p.prim[k]);
        p.slot[k][i] = v.x;
        p.slot[k][n + i] = v.y;
        p.slot[k][2 * n + i] = v.z;
    }
}

// Cubic Hermite resize of rows, written transposed (src/cvvdp/resize.hpp:26-49); plane
// blockIdx.y of a stack of planes.
__global__ void cv_resize_kernel(const float* src, int64_t src_pitch, int64_t src_plane, float* dst, int64_t dst_plane,
                                 int64_t sw, int64_t sh, int64_t rw) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rw * sh) return;
    const int64_t x = i % rw, y = i / rw;
    const float approx = (float)x * (float)sw / (float)rw;
    const int64_t b = (int64_t)approx;
    const float* row = src + blockIdx.y * src_plane + y * src_pitch;
    const float v1 = row[b];
    const float v0 = b - 1 >= 0 ? row[b - 1] : v1;
    const float v2 = b + 1 < sw ? row[b + 1] : v1;
    const float v3 = b + 2 < sw ? row[b + 2] : v2;
    dst[blockIdx.y * dst_plane + x * sh + y] = hermite(v1, (v2 - v0) / 2.f, v2, (v3 - v1) / 2.f, approx - (float)b);
}

// ---- temporal filter ---------------------------------------------------------------------

struct TemporalParams {
    const float* ring[2];
    const float* filt;  // 4 x taps: Y sustained, RG, YV, Y transient
    float* out[2][4];
    int64_t n;          // pixels per plane
    int taps, tsize, ind0;
};

__device__ __forceinline__ int ring_slot(const TemporalParams& p, int age) {
    int s = p.ind0 + min(age, p.tsize - 1);
    return s >= p.taps ? s - p.taps : s;
}

// Each thread: 4 consecutive pixels (float4) when kVec, else one.
template <bool kVec>
__global__ void __launch_bounds__(256) cv_temporal_kernel(const __grid_constant__ TemporalParams p) {
    const int k = blockIdx.y;
    const float* ring = p.ring[k];
    const int64_t step = kVec ? 4 : 1;
    const int64_t units = p.n / step;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < units; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = u * step;
        if (kVec) {
            float4 ys = make_float4(0.f, 0.f, 0.f, 0.f), rg = ys, yv = ys, yt = ys;
            if (p.tsize == 1) {
                const float* f = ring + (int64_t)ring_slot(p, 0) * 3 * p.n;
                ys = __ldg(reinterpret_cast<const float4*>(f + i));
                rg = __ldg(reinterpret_cast<const float4*>(f + p.n + i));
                yv = __ldg(reinterpret_cast<const float4*>(f + 2 * p.n + i));
            } else {
#pragma unroll 4
                for (int t = 0; t < p.taps; t++) {
                    const float* f = ring + (int64_t)ring_slot(p, t) * 3 * p.n;
                    const float k0 = __ldg(p.filt + t), k1 = __ldg(p.filt + p.taps + t), k2 = __ldg(p.filt + 2 * p.taps + t),
                                k3 = __ldg(p.filt + 3 * p.taps + t);
                    const float4 a = __ldg(reinterpret_cast<const float4*>(f + i));
                    const float4 b = __ldg(reinterpret_cast<const float4*>(f + p.n + i));
                    const float4 c = __ldg(reinterpret_cast<const float4*>(f + 2 * p.n + i));
                    ys.x = fmaf(a.x, k0, ys.x); ys.y = fmaf(a.y, k0, ys.y); ys.z = fmaf(a.z, k0, ys.z); ys.w = fmaf(a.w, k0, ys.w);
                    yt.x = fmaf(a.x, k3, yt.x); yt.y = fmaf(a.y, k3, yt.y); yt.z = fmaf(a.z, k3, yt.z); yt.w = fmaf(a.w, k3, yt.w);
                    rg.x = fmaf(b.x, k1, rg.x); rg.y = fmaf(b.y, k1, rg.y); rg.z = fmaf(b.z, k1, rg.z); rg.w = fmaf(b.w, k1, rg.w);
                    yv.x = fmaf(c.x, k2, yv.x); yv.y = fmaf(c.y, k2, yv.y); yv.z = fmaf(c.z, k2, yv.z); yv.w = fmaf(c.w, k2, yv.w);
                }
            }
            *reinterpret_cast<float4*>(p.out[k][0] + i) = ys;
            *reinterpret_cast<float4*>(p.out[k][1] + i) = rg;
            *reinterpret_cast<float4*>(p.out[k][2] + i) = yv;
            *reinterpret_cast<float4*>(p.out[k][3] + i) = yt;
        } else {
            float ys = 0.f, rg = 0.f, yv = 0.f, yt = 0.f;
            if (p.tsize == 1) {
                const float* f = ring + (int64_t)ring_slot(p, 0) * 3 * p.n;
                ys = f[i];
                rg = f[p.n + i];
                yv = f[2 * p.n + i];
            } else {
                for (int t = 0; t < p.taps; t++) {
                    const float* f = ring + (int64_t)ring_slot(p, t) * 3 * p.n;
                    const float a = __ldg(f + i);
                    ys = fmaf(a, __ldg(p.filt + t), ys);
                    yt = fmaf(a, __ldg(p.filt + 3 * p.taps + t), yt);
                    rg = fmaf(__ldg(f + p.n + i), __ldg(p.filt + p.taps + t), rg);
                    yv = fmaf(__ldg(f + 2 * p.n + i), __ldg(p.filt + 2 * p.taps + t), yv);
                }
            }
            p.out[k][0][i] = ys;
            p.out[k][1][i] = rg;
            p.out[k][2][i] = yv;
            p.out[k][3][i] = yt;
        }
    }
}

// ---- Gaussian pyramid --------------------------------------------------------------------

struct PlaneSet {
    const float* src[8];
    float* dst[8];
};

// One reduce step of 8 planes (plane blockIdx.y): w x h -> (w+1)/2 x (h+1)/2 with the
// reference's padding (mirror with edge repeat below 0, without it past the end).  A CTA makes
// a 32 x 16 tile of the output: the 68 x 36 input window (mirror resolved while staging) is
// staged in shared memory, then the separable 5-tap kernel runs along rows and columns.
constexpr int kRedW = 32, kRedH = 16;
constexpr int kRedInW = 2 * kRedW + 4, kRedInH = 2 * kRedH + 4;  // 68 x 36
constexpr int kRedThreads = 256;

__device__ __forceinline__ int mirror_index(int i, int n) {
    if (i < 0) i = -i - 1;
    if (i >= n) i = 2 * n - i - 2;
    return min(max(i, 0), n - 1);  // only outputs past the plane edge reach beyond the mirror
}

__global__ void __launch_bounds__(kRedThreads) cv_reduce_kernel(const __grid_constant__ PlaneSet p, int w, int h) {
    // 72-float rows: even, so a thread's pair of input columns is one aligned float2.
    constexpr int kStride = kRedInW + 4;
    __shared__ __align__(16) float in[kRedInH][kStride];
    __shared__ float hs[kRedInH][kRedW + 1];
    const int nw = (w + 1) / 2, nh = (h + 1) / 2;
    const int tiles_x = (nw + kRedW - 1) / kRedW;
    const int ox0 = (blockIdx.x % tiles_x) * kRedW, oy0 = (blockIdx.x / tiles_x) * kRedH;
    const float* src = p.src[blockIdx.y];
    const int ix0 = 2 * ox0 - 2, iy0 = 2 * oy0 - 2;
    // Staging: thread (tx, ty) of 64 x 4 loads columns tx and 64 + tx (when < 68) of rows
    // ty, ty + 4, ...; the mirrored column offsets are formed once.
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    const int ca = mirror_index(ix0 + tx, w);
    const bool has_b = tx < kRedInW - 64;
    const int cb = has_b ? mirror_index(ix0 + 64 + tx, w) : 0;
    constexpr int kRows = kRedInH / 4;  // 9
    static_assert(kRedInH % 4 == 0, "rows split over 4 thread rows");
    float va[kRows], vb[kRows];
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        const float* row = src + (int64_t)mirror_index(iy0 + ty + 4 * k, h) * w;
        va[k] = __ldg(row + ca);
        vb[k] = has_b ? __ldg(row + cb) : 0.f;
    }
#pragma unroll
    for (int k = 0; k < kRows; k++) {
        in[ty + 4 * k][tx] = va[k];
        if (has_b) in[ty + 4 * k][64 + tx] = vb[k];
    }
    __syncthreads();
    const float k0 = pyr_k(0), k1 = pyr_k(1), k2 = pyr_k(2);
    for (int i = threadIdx.x; i < kRedInH * kRedW; i += kRedThreads) {
        const int r = i / kRedW, x = i - r * kRedW;
        const float2 a = *reinterpret_cast<const float2*>(&in[r][2 * x]);
        const float2 b = *reinterpret_cast<const float2*>(&in[r][2 * x + 2]);
        const float c = in[r][2 * x + 4];
        hs[r][x] = fmaf(k0, a.x, fmaf(k1, a.y, fmaf(k2, b.x, fmaf(k1, b.y, k0 * c))));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRedH * kRedW; i += kRedThreads) {
        const int y = i / kRedW, x = i - y * kRedW;
        const int gx = ox0 + x, gy = oy0 + y;
        if (gx >= nw || gy >= nh) continue;
        const float o = fmaf(k0, hs[2 * y][x], fmaf(k1, hs[2 * y + 1][x], fmaf(k2, hs[2 * y + 2][x],
                             fmaf(k1, hs[2 * y + 3][x], k0 * hs[2 * y + 4][x]))));
        p.dst[blockIdx.y][(int64_t)gy * nw + gx] = o;
    }
}

// Value at (x, y) of a coarse plane expanded to w x h (gaussPyrExpand_Kernel, lpyr.hpp:48-90).
__device__ __forceinline__ float pyr_expand(const float* src, int w, int h, int x, int y) {
    const int ow = (w + 1) / 2, oh = (h + 1) / 2;
    float v = 0.f;
    for (int dx = -2 + (x & 1); dx <= 2; dx += 2) {
        int rx = (x + dx) / 2;
        if (rx < 0) rx = -rx - 1;
        if (rx >= ow) rx = 2 * ow - rx - 2;
        const float kx = 2.f * pyr_k(dx + 2);
        for (int dy = -2 + (y & 1); dy <= 2; dy += 2) {
            int ry = (y + dy) / 2;
            if (ry < 0) ry = -ry - 1;
            if (ry >= oh) ry = 2 * oh - ry - 2;
            v = fmaf(kx * (2.f * pyr_k(dy + 2)), __ldg(src + (int64_t)ry * ow + rx), v);
        }
    }
    return v;
}

// CSF sensitivity (computeSensitivityGPU, csf.hpp:60-82) from the band's 32-entry column,
// with the reference's weights (frac on the lower entry); the index is clamped to the table.
__device__ __forceinline__ float sensitivity(const float* col, float lum0, float span, float lbkg) {
    float frac = 31.f * (log10f(lbkg) - lum0) / span;
    int imin = (int)frac;
    imin = min(max(imin, 0), 31);
    const int imax = min(31, imin + 1);
    frac -= (float)imin;
    const float logs = col[imin] * frac + col[imax] * (1.f - frac) + kSensitivityCorrection / 20.f;
    return exp10f(logs);
}

// ---- one Laplacian band: contrast and CSF ------------------------------------------------

// Positive x to the power g through the hardware base-2 exponential and logarithm
// (relative error about 1e-6); 0 for x <= 0.
__device__ __forceinline__ float pow_pos(float x, float g) { return x > 0.f ? ex2_approx(g * __log2f(x)) : 0.f; }

constexpr int kCW = 64;                   // contrast tile: 64 x 16 pixels of the band, one
constexpr int kCHt = 16;                  // 2x2 quad per thread
constexpr int kCoarseW = kCW / 2 + 2;     // 34 coarse columns feed it (expansion taps)
constexpr int kCoarseH = kCHt / 2 + 2;    // 10 coarse rows
constexpr int kContrastThreads = (kCW / 2) * (kCHt / 2);  // 256

struct ContrastBand {
    const float* g[2][4];   // level b planes (w x h)
    const float* gn[2][4];  // level b+1 planes
    float* mn[4];           // out: min(|R|, |T|) per channel (w x h)
    float* df[4];           // out: |R - T| per channel
    const float* csf;       // 4 x 32 log10 sensitivities of this band
    int w, h, tiles_x, tile_start;
    float mult;             // contrast multiplier: 1 at band 0, 2 below
};

// All bands but the baseband in one launch, coarsest first (their few long-running tiles then
// overlap the finest band's many).
struct ContrastParams {
    ContrastBand band[kMaxLevels - 1];
    int nbands;
    float lum0, span;       // log10 of the first luminance sample and the axis span
};

// Laplacian layer of both clips (G_b - expand(G_b+1), the Y channel against the clamped
// background; lpyr.hpp:177-215), contrast against the background luminance, CSF weighting by
// the reference clip's background (preGaussianPreCompute_kernel, maskingModel.hpp:5-15).
// The tile's coarse neighbourhood of all eight next-level planes is staged in shared memory
// with the expansion's mirror padding already applied; each thread expands a 2x2 quad from
// its 3x3 coarse neighbourhood, separably (even pixels take taps 0.1/0.8/0.1 of the
// neighbourhood, odd pixels 0.5/0.5 of its last two samples).
__global__ void __launch_bounds__(kContrastThreads) cv_contrast_kernel(const __grid_constant__ ContrastParams prm) {
    __shared__ float coarse[8][kCoarseH][kCoarseW];
    __shared__ float csf[4][32];
    const int tid = threadIdx.x;
    int bi = 0;
    while (bi + 1 < prm.nbands && (int)blockIdx.x >= prm.band[bi + 1].tile_start) bi++;
    const ContrastBand& p = prm.band[bi];
    const int tile = blockIdx.x - p.tile_start;
    const int X0 = (tile % p.tiles_x) * kCW, Y0 = (tile / p.tiles_x) * kCHt;
    const int ow = (p.w + 1) / 2, oh = (p.h + 1) / 2;
    const int cx0 = X0 / 2 - 1, cy0 = Y0 / 2 - 1;
    if (tid < 128) csf[tid >> 5][tid & 31] = p.csf[tid];
    // Coarse staging: each thread's (up to 11) loads issued before any is stored.
    constexpr int kStage = 8 * kCoarseH * kCoarseW;
    constexpr int kPer = (kStage + kContrastThreads - 1) / kContrastThreads;
    float v[kPer];
#pragma unroll
    for (int it = 0; it < kPer; it++) {
        const int i = tid + it * kContrastThreads;
        v[it] = 0.f;
        if (i < kStage) {
            const int q = i / (kCoarseH * kCoarseW), r = (i / kCoarseW) % kCoarseH, c = i % kCoarseW;
            int rx = cx0 + c, ry = cy0 + r;
            if (rx < 0) rx = -rx - 1;
            if (rx >= ow) rx = 2 * ow - rx - 2;
            if (ry < 0) ry = -ry - 1;
            if (ry >= oh) ry = 2 * oh - ry - 2;
            rx = min(max(rx, 0), ow - 1);  // only pixels past the band edge reach beyond the mirror
            ry = min(max(ry, 0), oh - 1);
            v[it] = __ldg(p.gn[q >> 2][q & 3] + (int64_t)ry * ow + rx);
        }
    }
#pragma unroll
    for (int it = 0; it < kPer; it++) {
        const int i = tid + it * kContrastThreads;
        if (i < kStage) (&coarse[0][0][0])[i] = v[it];
    }
    __syncthreads();
    const int qx = tid % (kCW / 2), qy = tid / (kCW / 2);
    const int x0 = X0 + 2 * qx, y0 = Y0 + 2 * qy;
    if (x0 >= p.w || y0 >= p.h) return;
    const float we = 2.f * pyr_k(0), wc = 2.f * pyr_k(2), wo = 2.f * pyr_k(1);  // 0.1, 0.8, 0.5
    // e[q][v][u]: plane q expanded at pixel (x0 + u, y0 + v)
    float e[8][2][2];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        float he[3], ho[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float c0 = coarse[q][qy + a][qx], c1 = coarse[q][qy + a][qx + 1], c2 = coarse[q][qy + a][qx + 2];
            he[a] = fmaf(we, c0, fmaf(wc, c1, we * c2));
            ho[a] = fmaf(wo, c1, wo * c2);
        }
        e[q][0][0] = fmaf(we, he[0], fmaf(wc, he[1], we * he[2]));
        e[q][0][1] = fmaf(we, ho[0], fmaf(wc, ho[1], we * ho[2]));
        e[q][1][0] = fmaf(wo, he[1], wo * he[2]);
        e[q][1][1] = fmaf(wo, ho[1], wo * ho[2]);
    }
#pragma unroll
    for (int v = 0; v < 2; v++)
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int x = x0 + u, y = y0 + v;
            if (x >= p.w || y >= p.h) continue;
            const int64_t j = (int64_t)y * p.w + x;
            float con[2][4];
            float lref = 0.f;
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const float lb = fmaxf(e[4 * k][v][u], 0.01f);
                if (k == 0) lref = lb;
                const float inv = __frcp_rn(lb);
                con[k][0] = fminf((__ldg(p.g[k][0] + j) - lb) * inv, 1000.f) * p.mult;
#pragma unroll
                for (int c = 1; c < 4; c++)
                    con[k][c] = fminf((__ldg(p.g[k][c] + j) - e[4 * k + c][v][u]) * inv, 1000.f) * p.mult;
            }
            // CSF lookup (computeSensitivityGPU, csf.hpp:60-82) at the reference's background,
            // the reference's weights (frac on the lower entry); index clamped to the table.
            float frac = 31.f * (log10f(lref) - prm.lum0) / prm.span;
            int imin = min(max((int)frac, 0), 31);
            const int imax = min(31, imin + 1);
            frac -= (float)imin;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float logs = csf[c][imin] * frac + csf[c][imax] * (1.f - frac) + kSensitivityCorrection / 20.f;
                const float s = ex2_approx(logs * 3.32192809488736f) * (c == 1 ? 1.45f : 1.f);
                const float r = con[0][c] * s, t = con[1][c] * s;
                p.mn[c][j] = fminf(fabsf(r), fabsf(t));
                p.df[c][j] = fabsf(r - t);
            }
        }
}

// ---- one Laplacian band: masking and D ---------------------------------------------------

constexpr int kBT = 32;               // output tile
constexpr int kBH = 8;                // masking blur radius
constexpr int kBI = kBT + 2 * kBH;    // 48: tile with halo
constexpr int kMaskThreads = 128;
constexpr int kMaskRPT = 8;           // vertical pass: consecutive output rows per thread

struct MaskBand {
    const float* mn[4];
    const float* df[4];
    double* partials;       // 4 sums of D^2 per tile of this band
    float* merged;          // distortion-map plane of this band (nullable)
    int w, h, tiles_x, tile_start;
    float merge_div;
};

struct MaskParams {
    MaskBand band[kMaxLevels - 1];  // coarsest first
    int nbands;
    float blur_w[17];
    float xcm2[16];         // 2^xcm_weights[k * 4 + c]
};

// Channels travel in pairs (0,1) and (2,3) so one 64-bit shared access and one packed FMA
// serve two of them.
struct MaskSmem {
    float2 in[2][kBI][kBI + 1];   // masking input over the tile and its halo (0 outside the plane)
    float2 hb[2][kBI][kBT + 1];   // horizontally blurred
    float invx[kBT], invy[kBT];   // 1 / in-plane tap weight of each output column and row
    double red[kMaskThreads / 32][4];
};

// Sum of the blur taps that fall inside [0, n) for a window centred on pos (pos clamped into
// the plane for the tile's padding; their outputs are never used).
__device__ __forceinline__ float mask_tap_sum(const float* w, int pos, int n) {
    pos = min(pos, n - 1);
    float s = 0.f;
#pragma unroll
    for (int t = 0; t < 17; t++) {
        const int q = pos - 8 + t;
        s += (q >= 0 && q < n) ? w[t] : 0.f;
    }
    return s;
}

// The sigma-3 renormalised blur of min(|R|, |T|) (GaussianSmart_Device, gaussianBlur.hpp:62-119),
// cross-channel masking, the saturating D with the channel weights (computeD_Kernel,
// maskingModel.hpp:28-96), the tile's FP64 sums of D^2 and, for the distortion map, the
// 4-norm over channels (mergeChromaNorm_Kernel, distmap_specifics.hpp:27-33).
__global__ void __launch_bounds__(kMaskThreads) cv_mask_kernel(const __grid_constant__ MaskParams prm) {
    extern __shared__ __align__(16) unsigned char mask_smem_raw[];
    MaskSmem& sm = *reinterpret_cast<MaskSmem*>(mask_smem_raw);
    const int tid = threadIdx.x;
    int bi = 0;
    while (bi + 1 < prm.nbands && (int)blockIdx.x >= prm.band[bi + 1].tile_start) bi++;
    const MaskBand& p = prm.band[bi];
    const int tile = blockIdx.x - p.tile_start;
    const int X0 = (tile % p.tiles_x) * kBT, Y0 = (tile / p.tiles_x) * kBT;
    // Halo loads in two batches of 9 elements per thread, every load of a batch issued before
    // any is stored, so one memory round trip covers nine elements.
    static_assert(kBI * kBI == 18 * kMaskThreads, "halo splits into 18 elements per thread");
#pragma unroll
    for (int half = 0; half < 2; half++) {
        float4 v[9];
#pragma unroll
        for (int it = 0; it < 9; it++) {
            const int i = tid + (half * 9 + it) * kMaskThreads;
            const int r = i / kBI, c = i - r * kBI;
            const int gx = X0 - kBH + c, gy = Y0 - kBH + r;
            v[it] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gx >= 0 && gx < p.w && gy >= 0 && gy < p.h) {
                const int64_t j = (int64_t)gy * p.w + gx;
                v[it] = make_float4(__ldg(p.mn[0] + j), __ldg(p.mn[1] + j), __ldg(p.mn[2] + j), __ldg(p.mn[3] + j));
            }
        }
#pragma unroll
        for (int it = 0; it < 9; it++) {
            const int i = tid + (half * 9 + it) * kMaskThreads;
            const int r = i / kBI, c = i - r * kBI;
            sm.in[0][r][c] = make_float2(v[it].x, v[it].y);
            sm.in[1][r][c] = make_float2(v[it].z, v[it].w);
        }
    }
    if (tid < kBT) sm.invx[tid] = 1.f / mask_tap_sum(prm.blur_w, X0 + tid, p.w);
    else if (tid < 2 * kBT) sm.invy[tid - kBT] = 1.f / mask_tap_sum(prm.blur_w, Y0 + tid - kBT, p.h);
    __syncthreads();
    // Horizontal pass: 48 rows x 32 columns per channel pair; a work item is four adjacent
    // output columns of one row, consecutive threads take consecutive rows.
    for (int u = tid; u < 2 * kBI * (kBT / 4); u += kMaskThreads) {
        const int pr = u / (kBI * (kBT / 4));
        const int rem = u - pr * (kBI * (kBT / 4));
        const int cg = rem / kBI, r = rem - cg * kBI, c0 = cg * 4;
        float2 v[20];
#pragma unroll
        for (int j = 0; j < 20; j++) v[j] = sm.in[pr][r][c0 + j];
        float2 acc[4];
#pragma unroll
        for (int o = 0; o < 4; o++) acc[o] = make_float2(0.f, 0.f);
#pragma unroll
        for (int t = 0; t < 17; t++) {
            const float2 wt = make_float2(prm.blur_w[t], prm.blur_w[t]);
#pragma unroll
            for (int o = 0; o < 4; o++) acc[o] = __ffma2_rn(wt, v[o + t], acc[o]);
        }
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const float inv = sm.invx[c0 + o];
            sm.hb[pr][r][c0 + o] = make_float2(acc[o].x * inv, acc[o].y * inv);
        }
    }
    __syncthreads();
    // Vertical pass: each thread 8 consecutive output rows of one column.
    const int c = tid & (kBT - 1);
    const int r0 = (tid >> 5) * kMaskRPT;
    const int gx = X0 + c;
    // |R - T| of this thread's 8 pixels, loaded now so the loads overlap the blur.
    float dfv[kMaskRPT][4];
#pragma unroll
    for (int o = 0; o < kMaskRPT; o++) {
        const int gy = Y0 + r0 + o;
        const bool ok = gx < p.w && gy < p.h;
        const int64_t j = ok ? (int64_t)gy * p.w + gx : 0;
#pragma unroll
        for (int k = 0; k < 4; k++) dfv[o][k] = ok ? __ldg(p.df[k] + j) : 0.f;
    }
    float2 m[2][kMaskRPT];
#pragma unroll
    for (int pr = 0; pr < 2; pr++) {
        float2 col[kMaskRPT + 16];
#pragma unroll
        for (int j = 0; j < kMaskRPT + 16; j++) col[j] = sm.hb[pr][r0 + j][c];
#pragma unroll
        for (int o = 0; o < kMaskRPT; o++) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int t = 0; t < 17; t++) acc = __ffma2_rn(make_float2(prm.blur_w[t], prm.blur_w[t]), col[o + t], acc);
            const float inv = sm.invy[r0 + o];
            m[pr][o] = make_float2(acc.x * inv, acc.y * inv);
        }
    }
    const float powmaskc = exp10f(kMaskC);
    const float max_v = exp10f(kDMax);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int o = 0; o < kMaskRPT; o++) {
        const int gy = Y0 + r0 + o;
        if (gx >= p.w || gy >= p.h) continue;
        const int64_t j = (int64_t)gy * p.w + gx;
        const float mm[4] = {m[0][o].x, m[0][o].y, m[1][o].x, m[1][o].y};
        float cm[4];
#pragma unroll
        for (int k = 0; k < 4; k++) cm[k] = pow_pos(powmaskc * fabsf(mm[k]), kMaskQ[k]);
        float d[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float cmask = fmaf(cm[0], prm.xcm2[k], fmaf(cm[1], prm.xcm2[4 + k], fmaf(cm[2], prm.xcm2[8 + k], cm[3] * prm.xcm2[12 + k])));
            const float du = __fdividef(pow_pos(dfv[o][k], kMaskP), 1.f + cmask);
            d[k] = __fdividef(max_v * du, max_v + du) * (k == 3 ? kChTransW : 1.f);
            acc[k] += (double)(d[k] * d[k]);
        }
        if (p.merged) {
            const float q = (d[0] * d[0]) * (d[0] * d[0]) + (d[1] * d[1]) * (d[1] * d[1]) + (d[2] * d[2]) * (d[2] * d[2]) +
                            (d[3] * d[3]) * (d[3] * d[3]);
            p.merged[j] = pow_pos(q * 0.25f, 0.25f) / p.merge_div;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        double v = acc[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if ((tid & 31) == 0) sm.red[tid >> 5][k] = v;
    }
    __syncthreads();
    if (tid < 4) {
        double v = 0.0;
        for (int wi = 0; wi < kMaskThreads / 32; wi++) v += sm.red[wi][tid];
        p.partials[(int64_t)tile * 4 + tid] = v;
    }
}

// ---- baseband ----------------------------------------------------------------------------

struct PoolParams {
    // bands 0..L-2: tile sums of D^2
    const double* partials;
    int64_t tile_off[kMaxLevels];
    int64_t tiles[kMaxLevels];
    int64_t pixels[kMaxLevels];
    int nbands;             // L - 1
    // baseband (level L-1)
    const float* g[2][4];
    int64_t n;
    const float* csf;
    float lum0, span;
    float* merged;          // nullable
    double* vals;           // out: 4 pooled norms per band, baseband last
};

constexpr int kPoolThreads = 512;

__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[i];
    return t;
}

// Pooled norm sqrt(mean(D^2)) of every band and channel (computeMean<2>, pooling.hpp:54-85):
// CTA b < L-1 sums band b's tile partials; the last CTA does the baseband: mean background
// luminance of both clips, contrast, D with the baseband weights (lpyr.hpp:219-229,
// maskingModel.hpp:106-114) and its norm.
__global__ void __launch_bounds__(kPoolThreads) cv_pool_kernel(const __grid_constant__ PoolParams p) {
    __shared__ double red[kPoolThreads / 32];
    __shared__ float sens[4];
    const int b = blockIdx.x;
    if (b < p.nbands) {
        const double* part = p.partials + p.tile_off[b] * 4;
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int64_t t = threadIdx.x; t < p.tiles[b]; t += blockDim.x)
#pragma unroll
            for (int c = 0; c < 4; c++) v[c] += part[t * 4 + c];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const double s = block_sum(v[c], red);
            if (threadIdx.x == 0) p.vals[b * 4 + c] = sqrt(s / (double)p.pixels[b]);
        }
        return;
    }
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = threadIdx.x; i < p.n; i += blockDim.x) {
        s0 += p.g[0][0][i];
        s1 += p.g[1][0][i];
    }
    const float mean0 = (float)(block_sum(s0, red) / (double)p.n);
    const float mean1 = (float)(block_sum(s1, red) / (double)p.n);
    if (threadIdx.x < 4)
        sens[threadIdx.x] = sensitivity(p.csf + 32 * threadIdx.x, p.lum0, p.span, mean0) * kBasebandWeight[threadIdx.x];
    __syncthreads();
    const float den0 = fmaxf(0.01f, mean0), den1 = fmaxf(0.01f, mean1);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = threadIdx.x; i < p.n; i += blockDim.x) {
        float d[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float x = fminf(p.g[0][c][i] / den0, 1000.f), y = fminf(p.g[1][c][i] / den1, 1000.f);
            d[c] = fabsf(x - y) * sens[c];
            acc[c] += (double)d[c] * (double)d[c];
        }
        if (p.merged) {
            const float q = (d[0] * d[0]) * (d[0] * d[0]) + (d[1] * d[1]) * (d[1] * d[1]) + (d[2] * d[2]) * (d[2] * d[2]) +
                            (d[3] * d[3]) * (d[3] * d[3]);
            p.merged[i] = powf(q * 0.25f, 0.25f);
        }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const double t = block_sum(acc[c], red);
        if (threadIdx.x == 0) p.vals[p.nbands * 4 + c] = sqrt(t / (double)p.n);
    }
}

// ---- distortion map (distmap_specifics.hpp:47-71) ---------------------------------------

__global__ void cv_expand_add_kernel(float* fine, const float* coarse, int w, int h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    fine[i] += pyr_expand(coarse, w, h, i % w, i / w);
}

__host__ __device__ __forceinline__ float to_jod(float a) {
    if (a > 0.1f) return 10.f - kJodA * powf(a, kJodExp);
    const float jod_a_p = kJodA * powf(0.1f, kJodExp - 1.f);
    return 10.f - jod_a_p * a;
}

__global__ void cv_jod_kernel(const float* m, float* out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = 1.f - to_jod(m[i]) * 0.1f;
}

// ---- host: display models (display_models.hpp) ----------------------------------------------

struct Display {
    std::string name, source;
    int64_t res[2] = {1920, 1080};
    bool hdr = false;
    float distance = 0.6f, diagonal = 24.f, max_lum = 200.f, contrast = 1000.f, e_ambient = 250.f, k_refl = 0.005f,
          exposure = 1.f;
    bool set_res = true, set_cs = true, set_dist = true, set_diag = true, set_lum = true, set_contrast = true,
         set_amb = true;

    float ppd() const {  // get_screen_ppd (display_models.hpp:153-164), same float/double steps
        const float ar = (float)res[0] / (float)res[1];
        const float height_meter = (float)(std::sqrt(((double)diagonal * 25.4) * ((double)diagonal * 25.4) / (double)(1 + ar * ar)) / 1000);
        const float width_meter = ar * height_meter;
        const float pix_deg = (float)(2 * 180 * std::atan(0.5 * width_meter / (double)(float)res[0] / (double)distance) / kPi);
        return 1 / pix_deg;
    }
    float black() const { return max_lum / contrast; }
    float refl() const { return (float)(e_ambient * k_refl / kPi); }
};

bool builtin_display(const std::string& key, Display& d) {
    struct Row { const char* key; const char* name; int64_t w, h; bool hdr; float dist, diag, lum, contrast, amb; };
    static const Row rows[] = {
        {"standard_4k", "30-inch 4K monitor, peak luminance 200 cd/m^2, viewed under office light levels (250 lux), seen from 2 x display height",
         3840, 2160, false, 0.7472f, 30.f, 200.f, 1000.f, 250.f},
        {"standard_hdr_pq", "30-inch 4K HDR monitor, peak luminance 1500 cd/m^2, viewed under low light levels (10 lux), seen from 2 x display height",
         3840, 2160, true, 0.7472f, 30.f, 1500.f, 1000000.f, 10.f},
        {"standard_hdr_hlg", "30-inch 4K HDR monitor, peak luminance 1500 cd/m^2, viewed under low light levels (10 lux), seen from 2 x display height",
         3840, 2160, true, 0.7472f, 30.f, 1500.f, 1000000.f, 10.f},
        {"standard_hdr_linear", "30-inch 4K HDR monitor, peak luminance 1500 cd/m^2, viewed under low light levels (10 lux), seen from 2 x display height",
         3840, 2160, true, 0.7472f, 30.f, 1500.f, 1000000.f, 10.f},
        {"standard_hdr_dark", "30-inch 4K HDR monitor, peak luminance 1500 cd/m^2, viewed in a dark room (0 lux), seen from 2 x display height",
         3840, 2160, true, 0.7472f, 30.f, 1500.f, 1000000.f, 0.f},
        {"standard_hdr_linear_zoom", "30-inch 4K HDR monitor, peak luminance 4000 cd/m^2, viewed under low light levels (10 lux), seen from very close to spot super-resolution artifacts",
         3840, 2160, true, 0.25f, 30.f, 10000.f, 1000000.f, 10.f},
        {"standard_fhd", "24-inch FullHD monitor, peak luminance 200 cd/m^2, viewed under office light levels (250 lux), seen from 2 x display height",
         1920, 1080, false, 0.6f, 24.f, 200.f, 1000.f, 250.f},
    };
    for (const Row& r : rows) {
        if (key != r.key) continue;
        d.name = r.name;
        d.source = "none";
        d.res[0] = r.w;
        d.res[1] = r.h;
        d.hdr = r.hdr;
        d.distance = r.dist;
        d.diagonal = r.diag;
        d.max_lum = r.lum;
        d.contrast = r.contrast;
        d.e_ambient = r.amb;
        return true;
    }
    return false;
}

// Minimal JSON reader for display-model files: objects, arrays, strings, numbers, literals.
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    double num = 0;
    std::string str;
    std::vector<Json> items;
    std::vector<std::string> keys;  // Object: keys[i] names items[i]
};

class JsonReader {
public:
    explicit JsonReader(const std::string& text) : s_(text) {}
    Json document() {
        Json v = value(0);
        skip();
        if (i_ != s_.size()) fail("unexpected text after the top-level value");
        return v;
    }

private:
    [[noreturn]] void fail(const std::string& what) {
        VSHIP_THROW(Vship_BadJson, "Illformed json at byte " + std::to_string(i_) + ": " + what);
    }
    void skip() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) i_++;
    }
    bool eat(char c) {
        skip();
        if (i_ < s_.size() && s_[i_] == c) {
            i_++;
            return true;
        }
        return false;
    }
    std::string string_body() {
        std::string out;
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) break;
                const char e = s_[i_++];
                switch (e) {
                case 'n': c = '\n'; break;
                case 't': c = '\t'; break;
                case 'r': c = '\r'; break;
                case 'b': c = '\b'; break;
                case 'f': c = '\f'; break;
                case 'u':
                    if (i_ + 4 > s_.size()) fail("short \\u escape");
                    i_ += 4;
                    c = '?';
                    break;
                default: c = e; break;
                }
            }
            out.push_back(c);
        }
        if (i_ >= s_.size()) fail("string is not terminated");
        i_++;
        return out;
    }
    Json value(int depth) {
        if (depth > 64) fail("nesting too deep");
        skip();
        if (i_ >= s_.size()) fail("missing value");
        Json v;
        const char c = s_[i_];
        if (c == '{') {
            i_++;
            v.kind = Json::Object;
            if (eat('}')) return v;
            do {
                skip();
                if (i_ >= s_.size() || s_[i_] != '"') fail("expected a key");
                i_++;
                v.keys.push_back(string_body());
                if (!eat(':')) fail("expected ':'");
                v.items.push_back(value(depth + 1));
            } while (eat(','));
            if (!eat('}')) fail("expected ',' or '}'");
        } else if (c == '[') {
            i_++;
            v.kind = Json::Array;
            if (eat(']')) return v;
            do v.items.push_back(value(depth + 1));
            while (eat(','));
            if (!eat(']')) fail("expected ',' or ']'");
        } else if (c == '"') {
            i_++;
            v.kind = Json::String;
            v.str = string_body();
        } else if (s_.compare(i_, 4, "true") == 0 || s_.compare(i_, 5, "false") == 0) {
            v.kind = Json::Bool;
            v.num = s_[i_] == 't';
            i_ += s_[i_] == 't' ? 4 : 5;
        } else if (s_.compare(i_, 4, "null") == 0) {
            i_ += 4;
        } else {
            const char* b = s_.c_str() + i_;
            char* e = nullptr;
            v.num = std::strtod(b, &e);
            if (e == b) fail(std::string("unexpected character '") + c + "'");
            v.kind = Json::Number;
            i_ += (size_t)(e - b);
        }
        return v;
    }
    const std::string& s_;
    size_t i_ = 0;
};

float json_number(const Json& v, const std::string& key) {
    if (v.kind != Json::Number) VSHIP_THROW(Vship_BadJson, "field " + key + " must be a number");
    return (float)v.num;
}

// Applies the JSON file's entry `key` (display_models.hpp:174-262); returns false when the
// file has no such entry.
bool apply_json(const std::string& path, const std::string& key, Display& d) {
    std::ifstream f(path, std::ios::binary);
    if (!f) VSHIP_THROW(Vship_BadPath, "Path: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    const Json doc = JsonReader(text).document();
    if (doc.kind != Json::Object) VSHIP_THROW(Vship_BadJson, "the display file must hold one object of displays");
    for (size_t i = 0; i < doc.keys.size(); i++) {
        if (doc.keys[i] != key) continue;
        const Json& m = doc.items[i];
        if (m.kind != Json::Object) VSHIP_THROW(Vship_BadJson, "display " + key + " must be an object");
        for (size_t k = 0; k < m.keys.size(); k++) {
            const std::string& f = m.keys[k];
            const Json& v = m.items[k];
            if (f == "name" || f == "source") {
                if (v.kind != Json::String) VSHIP_THROW(Vship_BadJson, "field " + f + " must be a string");
                (f == "name" ? d.name : d.source) = v.str;
            } else if (f == "colorspace") {
                if (v.kind != Json::String) VSHIP_THROW(Vship_BadJson, "field colorspace must be a string");
                if (v.str == "HDR" || v.str == "BT.2020-PQ" || v.str == "BT.2020-HLG") d.hdr = true;
                else if (v.str == "BT.709-linear" || v.str == "sRGB" || v.str == "SDR") d.hdr = false;
                else VSHIP_THROW(Vship_BadJson, "colospace can either be BT.2020-PQ, BT.2020-HLG, BT.709-linear, HDR, sRGB or SDR");
                d.set_cs = true;
            } else if (f == "resolution") {
                if (v.kind != Json::Array || v.items.size() != 2) VSHIP_THROW(Vship_BadJson, "resolution must be [width, height]");
                for (int a = 0; a < 2; a++) d.res[a] = (int64_t)json_number(v.items[a], "resolution");
                if (d.res[0] <= 0 || d.res[1] <= 0) VSHIP_THROW(Vship_BadJson, "resolution must be positive");
                d.set_res = true;
            } else if (f == "viewing_distance_meters") {
                d.distance = json_number(v, f);
                d.set_dist = true;
            } else if (f == "diagonal_size_inches") {
                d.diagonal = json_number(v, f);
                d.set_diag = true;
            } else if (f == "max_luminance") {
                d.max_lum = json_number(v, f);
                d.set_lum = true;
            } else if (f == "contrast") {
                d.contrast = json_number(v, f);
                d.set_contrast = true;
            } else if (f == "E_ambient") {
                d.e_ambient = json_number(v, f);
                d.set_amb = true;
            } else if (f == "k_refl") {
                d.k_refl = json_number(v, f);
            } else if (f == "exposure") {
                d.exposure = json_number(v, f);
            } else {
                VSHIP_THROW(Vship_BadJson, "Unsupported field " + f + " in selected display");
            }
        }
        return true;
    }
    return false;
}

// DisplayModel::DisplayModel (display_models.hpp:38-152).
Display resolve_display(const std::string& key, const std::string& json) {
    Display d;
    const bool builtin = builtin_display(key, d);
    if (!builtin) d.set_res = d.set_cs = d.set_dist = d.set_diag = d.set_lum = d.set_contrast = d.set_amb = false;
    const bool in_json = !json.empty() && apply_json(json, key, d);
    std::string detail;
    if (!in_json && !builtin) detail = "Display Unset, wrong display name?";
    else if (!d.set_res) detail = "Display Missing resolution";
    else if (!d.set_cs) detail = "Display Missing colorspace";
    else if (!d.set_dist) detail = "Display Missing viewing_distance_meters";
    else if (!d.set_diag) detail = "Display Missing diagonal_size_inches";
    else if (!d.set_lum) detail = "Display Missing max_luminance";
    else if (!d.set_contrast) detail = "Display Missing contrast";
    else if (!d.set_amb) detail = "Display Missing E_ambiant";
    if (!detail.empty()) VSHIP_THROW(Vship_BadDisplayModel, detail);
    return d;
}

// ---- host: pyramid geometry, temporal filters, CSF columns ---------------------------------

// get_frequencies (lpyr.hpp:148-161), same float/double steps; returns the band count.
int band_frequencies(int64_t w, int64_t h, float ppd, float* bf) {
    const float min_freq = 0.2f;
    const int for_res = (int)(std::log2((double)std::min(w, h)) - 1);
    const int for_ppd = (int)(std::ceil(-std::log2(2 * min_freq / 0.3228 / (double)ppd)) + 1);
    const int levels = std::min(for_ppd, std::min(for_res, 14));
    if (levels < 1) return levels;
    bf[0] = (float)(0.5 * ppd);
    for (int i = 0; i < levels - 1; i++) bf[i + 1] = (float)(0.3228 * 0.5 * ppd / (double)(float)(1 << i));
    return levels;
}

// TemporalFilter::init and inverseRealFourrierTransform (temporalFilter.hpp:5-73), same
// float/double steps, including the halved last spectral sample.
std::vector<float> temporal_filters(float fps, int& taps) {
    int size = (int)(std::ceil(0.25 * fps / 2) * 2) + 1;
    size = std::max(size, 1);
    taps = size;
    const int nf = size / 2 + 1;
    std::vector<float> freq(nf);
    for (int i = 0; i < nf; i++) freq[i] = fps * i / 2;
    std::vector<float> spec[4];
    for (int j = 0; j < 3; j++) {
        spec[j].resize(nf);
        for (int i = 0; i < nf; i++) spec[j][i] = std::exp(-std::pow(freq[i], kBetaTf[j]) / kSigmaTf[j]);
    }
    spec[3].resize(nf);
    for (int i = 0; i < nf; i++) {
        float t = (float)((double)std::pow(freq[i], kBetaTf[3]) - std::pow(5.0, (double)kBetaTf[3]));
        t *= t;
        spec[3][i] = std::exp(-t / kSigmaTf[3]);
    }
    std::vector<float> out((size_t)4 * size, 0.f);
    for (int j = 0; j < 4; j++) {
        std::vector<float> inp = spec[j];
        if (nf > size / 2) inp[size / 2] /= 2;
        inp[0] /= 2;
        float* res = out.data() + (size_t)j * size;
        for (int i = 0; i < size; i++)
            for (int k = 0; k < nf; k++) {
                float& r = res[(i + nf - 1) % size];
                r = (float)((double)r + 2 * inp[k] * std::cos(2 * kPi * k * i / size) / size);
            }
    }
    return out;
}

// CSF_Handler::init (csf.hpp:23-54): per band and channel, the 32 log10 sensitivities at the
// band's frequency, interpolated linearly between table columns in log frequency.
std::vector<float> csf_columns(const float* bf, int levels, float& lum0, float& span) {
    using namespace cvvdp_tables;
    float logrho[32], loglum[32];
    for (int i = 0; i < 32; i++) {
        logrho[i] = std::log10(kCsfRho[i]);
        loglum[i] = std::log10(kCsfLum[i]);
    }
    lum0 = loglum[0];
    span = loglum[31] - loglum[0];
    std::vector<float> out((size_t)levels * 128);
    for (int b = 0; b < levels; b++) {
        const float lr = std::log10(bf[b]);
        int x0 = 31;
        for (int i = 1; i < 32; i++)
            if (logrho[i] > lr) {
                x0 = i - 1;
                break;
            }
        x0 = std::min(30, x0);
        const float slope = (lr - logrho[x0]) / (logrho[x0 + 1] - logrho[x0]);
        for (int c = 0; c < 4; c++)
            for (int i = 0; i < 32; i++) {
                const float y0 = kCsfLogS[c][i][x0], y1 = kCsfLogS[c][i][x0 + 1];
                out[(size_t)b * 128 + c * 32 + i] = y0 + (y1 - y0) * slope;
            }
    }
    return out;
}

// ---- engine ------------------------------------------------------------------------------

class Engine final : public CvvdpApi {
public:
    ~Engine() override { release(); }

    void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, float fps, bool resize_to_display,
              const std::string& model_key, const std::string& model_config_json, int device) override {
        device_ = device;
        disp_ = resolve_display(model_key, model_config_json);
        cs_[0] = src;
        cs_[1] = dis;
        for (int k = 0; k < 2; k++) {
            geo_[k] = make_geometry(cs_[k]);
            cp_[k] = make_colour_params(cs_[k], geo_[k], false);
        }
        if (geo_[0].OW != geo_[1].OW || geo_[0].OH != geo_[1].OH) VSHIP_THROW(Vship_DifferingInputType, "");
        sw_ = geo_[0].OW;
        sh_ = geo_[0].OH;
        if (resize_to_display) {  // main.hpp:201-214
            const int64_t rx = disp_.res[0], ry = disp_.res[1];
            if (sw_ * ry >= sh_ * rx) {
                rw_ = rx;
                rh_ = sh_ * rx / sw_;
            } else {
                rh_ = ry;
                rw_ = sw_ * ry / sh_;
            }
        } else {
            rw_ = sw_;
            rh_ = sh_;
        }
        if (rw_ <= 0 || rh_ <= 0) VSHIP_THROW(Vship_BadErrorType, "display resize leaves no pixels");
        mw_ = std::min(rw_, sw_);
        mh_ = std::min(rh_, sh_);
        down_ = (sw_ != rw_ || sh_ != rh_) && sw_ > rw_;
        generic_ = down_ || geo_[0].generic() || geo_[1].generic();
        const float ppd = disp_.ppd();
        levels_ = band_frequencies(rw_, rh_, ppd, band_freq_);
        if (levels_ < 1)
            VSHIP_THROW(Vship_BadErrorType, "frame too small for CVVDP: both dimensions must be at least 4 pixels after the display resize");
        int64_t w = rw_, h = rh_, off = 0, toff = 0;
        for (int i = 0; i < levels_; i++) {
            lw_[i] = w;
            lh_[i] = h;
            level_off_[i] = off;
            off += w * h;
            tile_off_[i] = toff;
            tiles_x_[i] = ceil_div(w, kBT);
            tiles_[i] = tiles_x_[i] * ceil_div(h, kBT);
            if (i < levels_ - 1) toff += tiles_[i];
            w = (w + 1) / 2;
            h = (h + 1) / 2;
        }
        chan_stride_ = round_up(off, 64);
        const std::vector<float> filt = temporal_filters(fps, taps_);
        const std::vector<float> csf = csf_columns(band_freq_, levels_, lum0_, span_);
        dd_.peak = disp_.max_lum;
        dd_.black = disp_.black();
        dd_.refl = disp_.refl();
        dd_.exposure = disp_.exposure;
        dd_.hdr = disp_.hdr ? 1 : 0;
        for (int k = 0; k < 2; k++) {
            trc_[k] = cs_[k].transferFunction;
            prim_[k] = cs_[k].primaries;
        }
        // Masking blur (GaussianHandle::init, gaussianBlur.hpp:9-21): sigma = pu_dilate = 3.
        const float sigma = 3.f;
        blur_prefix_[0] = 0.f;
        for (int i = 0; i < 17; i++) {
            blur_w_[i] = (float)(std::exp(-(float)((8 - i) * (8 - i)) / (2 * sigma * sigma)) / std::sqrt(6.28318530718 * sigma * sigma));
            blur_prefix_[i + 1] = blur_prefix_[i] + blur_w_[i];
        }
        for (int k = 0; k < 4; k++)
            for (int c = 0; c < 4; c++) xcm2_[k * 4 + c] = std::exp2(kXcmWeights[k * 4 + c]);

        CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        CUDA_CHECK(cudaEventCreateWithFlags(&last_done_, cudaEventDisableTiming));
        // per device: the caller has selected this handler's device
        CUDA_CHECK(cudaFuncSetAttribute(cv_mask_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MaskSmem)));
        for (int k = 0; k < 2; k++) {
            int64_t po[3];
            staging_[k].ensure((size_t)dense_image_bytes(geo_[k], po), stream_);
            if (generic_) lin_[k].alloc(geo_[k]);
        }
        if (down_) down_buf_ = device_alloc<float>((size_t)(3 * rw_ * rh_ + rw_ * sh_), "display resize planes");
        const int64_t mn = mw_ * mh_;
        ring_ = device_alloc<float>((size_t)(2 * (int64_t)taps_ * 3 * mn), "temporal ring");
        pyr_ = device_alloc<float>((size_t)(2 * 4 * chan_stride_), "contrast pyramid");
        if (levels_ > 1) mask_buf_ = device_alloc<float>((size_t)(8 * level_off_[levels_ - 1]), "band masking planes");
        if (mw_ < rw_) up_buf_ = device_alloc<float>((size_t)(2 * 4 * mn + rw_ * mh_), "upscale planes");
        filt_d_ = device_alloc<float>(filt.size(), "temporal filters");
        CUDA_CHECK(cudaMemcpy(filt_d_, filt.data(), filt.size() * sizeof(float), cudaMemcpyHostToDevice));
        csf_d_ = device_alloc<float>(csf.size(), "csf columns");
        CUDA_CHECK(cudaMemcpy(csf_d_, csf.data(), csf.size() * sizeof(float), cudaMemcpyHostToDevice));
        partials_ = device_alloc<double>((size_t)std::max<int64_t>(tile_off_[levels_ - 1], 1) * 4, "band partials");
        vals_d_ = device_alloc<double>((size_t)4 * levels_, "pooled norms");
        vals_h_ = pinned_alloc<double>((size_t)4 * levels_, "pooled norms");
        tsize_ = 0;
        ind0_ = 0;
        reset(false);
    }

    double compute(uint8_t* dstp, int64_t dststride, const uint8_t* const s1[3], const uint8_t* const s2[3],
                   const int64_t ls1[3], const int64_t ls2[3]) override {
        if (dstp && dststride < rw_ * 4) VSHIP_THROW(Vship_BadPointer, "dststride smaller than the distortion map width * 4");
        CUDA_CHECK(cudaStreamWaitEvent(stream_, last_done_, 0));
        load(s1, s2, ls1, ls2);
        if (dstp && !merged_) {
            merged_ = device_alloc<float>((size_t)chan_stride_, "distortion map bands");
            dmap_ = device_alloc<float>((size_t)(rw_ * rh_), "distortion map");
        }
        process(dstp != nullptr);
        CUDA_CHECK(cudaMemcpyAsync(vals_h_, vals_d_, sizeof(double) * 4 * levels_, cudaMemcpyDeviceToHost, stream_));
        if (dstp)
            CUDA_CHECK(cudaMemcpy2DAsync(dstp, (size_t)dststride, dmap_, (size_t)rw_ * 4, (size_t)rw_ * 4, (size_t)rh_,
                                         cudaMemcpyDeviceToHost, stream_));
        CUDA_CHECK(cudaEventRecord(last_done_, stream_));
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        // Pooling over bands and channels, then over frames (main.hpp:146-155, 376-388).
        double q = 0.0;
        for (int i = 0; i < 4 * levels_; i++) q += std::pow(vals_h_[i], 4);
        q = std::pow(q, 1. / 4.);
        sq_sum_ += std::pow(q, 2);
        const double resq = num_frame_ == 0 ? q * kImageInt : std::pow(sq_sum_ / (double)num_frame_, 1. / 2);
        num_frame_++;
        return to_jod((float)resq);
    }

    void load_temporal(const uint8_t* const s1[3], const uint8_t* const s2[3], const int64_t ls1[3],
                       const int64_t ls2[3]) override {
        CUDA_CHECK(cudaStreamWaitEvent(stream_, last_done_, 0));
        load(s1, s2, ls1, ls2);
        CUDA_CHECK(cudaEventRecord(last_done_, stream_));
        CUDA_CHECK(cudaStreamSynchronize(stream_));
    }

    void reset(bool only_score) override {
        num_frame_ = 0;
        sq_sum_ = 0.0;
        if (!only_score) tsize_ = 0;
    }

    int64_t distmap_width() const override { return rw_; }
    int64_t distmap_height() const override { return rh_; }
    int bands() const override { return levels_; }
    int ring_frames() const override { return taps_; }
    KernelTimer& timer() override { return timer_; }

private:
    float* plane(int k, int c, int level) const { return pyr_ + (int64_t)(k * 4 + c) * chan_stride_ + level_off_[level]; }

    // loadImageToRing (main.hpp:234-347): rotate the ring, write the new frame of both clips.
    void load(const uint8_t* const s1[3], const uint8_t* const s2[3], const int64_t ls1[3], const int64_t ls2[3]) {
        RawImage raw[2];
        ColourParams cp[2] = {cp_[0], cp_[1]};
        for (int k = 0; k < 2; k++) {
            raw[k] = stage_host_image(staging_[k], geo_[k], k ? s2 : s1, k ? ls2 : ls1, stream_);
            cp[k].misaligned = misaligned_view(raw[k], geo_[k]) ? 1 : 0;
        }
        tsize_ = std::min(taps_, tsize_ + 1);
        ind0_ = (ind0_ + taps_ - 1) % taps_;
        const int64_t mn = mw_ * mh_;
        float* slot[2];
        for (int k = 0; k < 2; k++) slot[k] = ring_ + ((int64_t)k * taps_ + ind0_) * 3 * mn;
        const int t = timer_.begin(0, "cvvdp_ingest", stream_);
        if (!generic_) {
            IngestParams p{};
            for (int k = 0; k < 2; k++) {
                p.im[k] = raw[k];
                p.cp[k] = cp[k];
                p.slot[k] = slot[k];
                p.trc[k] = trc_[k];
                p.prim[k] = prim_[k];
            }
            p.n = mn;
            p.disp = dd_;
            const size_t smem = sizeof(float) * std::max(chroma_stage_floats(cp[0].subw, cp[0].subh),
                                                         chroma_stage_floats(cp[1].subw, cp[1].subh));
            const int f0 = fast_path_of(cp[0]);
            const int fast = f0 == fast_path_of(cp[1]) ? f0 : kFastGeneric;
            auto kernel = fast == kFastYuv420Bt709 ? cv_ingest_kernel<kFastYuv420Bt709>
                        : fast == kFastRgb8Srgb    ? cv_ingest_kernel<kFastRgb8Srgb>
                                                   : cv_ingest_kernel<kFastGeneric>;
            if (smem > 48 * 1024) CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const dim3 grid((unsigned)ceil_div(std::max(cp[0].W, cp[1].W), kStageTile),
                            (unsigned)ceil_div(std::max(cp[0].H, cp[1].H), kStageTile), 2);
            kernel<<<grid, 256, smem, stream_>>>(p);
            CUDA_CHECK(cudaGetLastError());
        } else {
            EncodeParams p{};
            for (int k = 0; k < 2; k++) {
                lin_[k].run(raw[k], cp[k], geo_[k], stream_, true);
                const float* win = lin_[k].planes + (int64_t)geo_[k].crop_top * geo_[k].TW + geo_[k].crop_left;
                if (down_) {  // display resize before the ring (main.hpp:299-305)
                    float* dst = down_buf_;
                    float* mid = down_buf_ + 3 * rw_ * rh_;
                    for (int c = 0; c < 3; c++) {
                        cv_resize_kernel<<<dim3((unsigned)ceil_div(rw_ * sh_, 256), 1), 256, 0, stream_>>>(
                            win + c * lin_[k].plane_floats, geo_[k].TW, 0, mid, 0, sw_, sh_, rw_);
                        CUDA_CHECK(cudaGetLastError());
                        cv_resize_kernel<<<dim3((unsigned)ceil_div(rh_ * rw_, 256), 1), 256, 0, stream_>>>(
                            mid, sh_, 0, dst + c * rw_ * rh_, 0, sh_, rw_, rh_);
                        CUDA_CHECK(cudaGetLastError());
                    }
                    // encode this clip now: the resize buffer is shared by both clips
                    EncodeParams q{};
                    q.src[0] = dst;
                    q.pitch[0] = rw_;
                    q.plane[0] = rw_ * rh_;
                    q.slot[0] = slot[k];
                    q.w = mw_;
                    q.h = mh_;
                    q.trc[0] = trc_[k];
                    q.prim[0] = prim_[k];
                    q.disp = dd_;
                    cv_encode_kernel<<<dim3((unsigned)std::min<int64_t>(ceil_div(mn, 256), 148 * 8), 1), 256, 0, stream_>>>(q);
                    CUDA_CHECK(cudaGetLastError());
                } else {
                    p.src[k] = win;
                    p.pitch[k] = geo_[k].TW;
                    p.plane[k] = lin_[k].plane_floats;
                    p.slot[k] = slot[k];
                    p.trc[k] = trc_[k];
                    p.prim[k] = prim_[k];
                }
            }
            if (!down_) {
                p.w = mw_;
                p.h = mh_;
                p.disp = dd_;
                cv_encode_kernel<<<dim3((unsigned)std::min<int64_t>(ceil_div(mn, 256), 148 * 8), 2), 256, 0, stream_>>>(p);
                CUDA_CHECK(cudaGetLastError());
            }
        }
        timer_.end(t, stream_);
    }

    // CVVDPprocess (main.hpp:24-158) up to the pooled norms in vals_d_.
    void process(bool distmap) {
        const int64_t mn = mw_ * mh_;
        int t = timer_.begin(1, "cvvdp_temporal", stream_);
        TemporalParams tp{};
        for (int k = 0; k < 2; k++) {
            tp.ring[k] = ring_ + (int64_t)k * taps_ * 3 * mn;
            for (int c = 0; c < 4; c++) tp.out[k][c] = mw_ < rw_ ? up_buf_ + (int64_t)(k * 4 + c) * mn : plane(k, c, 0);
        }
        tp.filt = filt_d_;
        tp.n = mn;
        tp.taps = taps_;
        tp.tsize = tsize_;
        tp.ind0 = ind0_;
        const bool vec = mn % 4 == 0;
        const int64_t units = vec ? mn / 4 : mn;
        const dim3 tgrid((unsigned)std::min<int64_t>(ceil_div(units, 256), 148 * 16), 2);
        if (vec) cv_temporal_kernel<true><<<tgrid, 256, 0, stream_>>>(tp);
        else cv_temporal_kernel<false><<<tgrid, 256, 0, stream_>>>(tp);
        CUDA_CHECK(cudaGetLastError());
        if (mw_ < rw_) {  // upscale of the temporal channels to the display size (main.hpp:71-82)
            float* mid = up_buf_ + 8 * mn;
            for (int q = 0; q < 8; q++) {
                cv_resize_kernel<<<dim3((unsigned)ceil_div(rw_ * mh_, 256), 1), 256, 0, stream_>>>(
                    up_buf_ + q * mn, mw_, 0, mid, 0, mw_, mh_, rw_);
                CUDA_CHECK(cudaGetLastError());
                cv_resize_kernel<<<dim3((unsigned)ceil_div(rh_ * rw_, 256), 1), 256, 0, stream_>>>(
                    mid, mh_, 0, plane(q / 4, q % 4, 0), 0, mh_, rw_, rh_);
                CUDA_CHECK(cudaGetLastError());
            }
        }
        timer_.end(t, stream_);

        t = timer_.begin(2, "cvvdp_reduce", stream_);
        for (int i = 0; i + 1 < levels_; i++) {
            PlaneSet ps{};
            for (int q = 0; q < 8; q++) {
                ps.src[q] = plane(q / 4, q % 4, i);
                ps.dst[q] = plane(q / 4, q % 4, i + 1);
            }
            const unsigned rtiles = (unsigned)(ceil_div(lw_[i + 1], kRedW) * ceil_div(lh_[i + 1], kRedH));
            cv_reduce_kernel<<<dim3(rtiles, 8), kRedThreads, 0, stream_>>>(ps, (int)lw_[i], (int)lh_[i]);
            CUDA_CHECK(cudaGetLastError());
        }
        timer_.end(t, stream_);

        if (levels_ > 1) {
            ContrastParams cp{};
            MaskParams mp{};
            int ctiles = 0, mtiles = 0;
            cp.nbands = mp.nbands = levels_ - 1;
            for (int i = 0; i < levels_ - 1; i++) {
                const int b = levels_ - 2 - i;  // coarsest first
                ContrastBand& cb = cp.band[i];
                MaskBand& mb = mp.band[i];
                const int64_t nb = lw_[b] * lh_[b];
                for (int k = 0; k < 2; k++)
                    for (int c = 0; c < 4; c++) {
                        cb.g[k][c] = plane(k, c, b);
                        cb.gn[k][c] = plane(k, c, b + 1);
                    }
                float* mbuf = mask_buf_ + 8 * level_off_[b];
                for (int c = 0; c < 4; c++) {
                    cb.mn[c] = mbuf + c * nb;
                    cb.df[c] = mbuf + (4 + c) * nb;
                    mb.mn[c] = cb.mn[c];
                    mb.df[c] = cb.df[c];
                }
                cb.csf = csf_d_ + (int64_t)b * 128;
                cb.w = mb.w = (int)lw_[b];
                cb.h = mb.h = (int)lh_[b];
                cb.tiles_x = (int)ceil_div(lw_[b], kCW);
                cb.tile_start = ctiles;
                ctiles += cb.tiles_x * (int)ceil_div(lh_[b], kCHt);
                cb.mult = b == 0 ? 1.f : 2.f;
                mb.tiles_x = (int)tiles_x_[b];
                mb.tile_start = mtiles;
                mtiles += (int)tiles_[b];
                mb.partials = partials_ + tile_off_[b] * 4;
                mb.merged = distmap ? merged_ + level_off_[b] : nullptr;
                mb.merge_div = b == 0 ? 1.f : 2.f;
            }
            cp.lum0 = lum0_;
            cp.span = span_;
            std::memcpy(mp.blur_w, blur_w_, sizeof(blur_w_));
            std::memcpy(mp.xcm2, xcm2_, sizeof(xcm2_));
            t = timer_.begin(6, "cvvdp_contrast", stream_);
            cv_contrast_kernel<<<(unsigned)ctiles, kContrastThreads, 0, stream_>>>(cp);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, stream_);
            t = timer_.begin(7, "cvvdp_mask", stream_);
            cv_mask_kernel<<<(unsigned)mtiles, kMaskThreads, sizeof(MaskSmem), stream_>>>(mp);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, stream_);
        }

        t = timer_.begin(4, "cvvdp_pool", stream_);
        const int L = levels_ - 1;
        PoolParams pp{};
        pp.partials = partials_;
        pp.nbands = L;
        for (int b = 0; b < L; b++) {
            pp.tile_off[b] = tile_off_[b];
            pp.tiles[b] = tiles_[b];
            pp.pixels[b] = lw_[b] * lh_[b];
        }
        for (int k = 0; k < 2; k++)
            for (int c = 0; c < 4; c++) pp.g[k][c] = plane(k, c, L);
        pp.n = lw_[L] * lh_[L];
        pp.csf = csf_d_ + (int64_t)L * 128;
        pp.lum0 = lum0_;
        pp.span = span_;
        pp.merged = distmap ? merged_ + level_off_[L] : nullptr;
        pp.vals = vals_d_;
        cv_pool_kernel<<<L + 1, kPoolThreads, 0, stream_>>>(pp);
        CUDA_CHECK(cudaGetLastError());
        timer_.end(t, stream_);

        if (distmap) {
            t = timer_.begin(5, "cvvdp_distmap", stream_);
            for (int b = levels_ - 2; b >= 0; b--) {
                const int64_t nn = lw_[b] * lh_[b];
                cv_expand_add_kernel<<<(unsigned)ceil_div(nn, 256), 256, 0, stream_>>>(merged_ + level_off_[b],
                                                                                       merged_ + level_off_[b + 1],
                                                                                       (int)lw_[b], (int)lh_[b]);
                CUDA_CHECK(cudaGetLastError());
            }
            cv_jod_kernel<<<(unsigned)ceil_div(rw_ * rh_, 256), 256, 0, stream_>>>(merged_, dmap_, rw_ * rh_);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, stream_);
        }
    }

    void release() {
        if (stream_) (void)cudaStreamSynchronize(stream_);
        timer_.destroy();
        for (int k = 0; k < 2; k++) {
            staging_[k].free();
            lin_[k].free();
        }
        device_free(down_buf_);
        device_free(up_buf_);
        device_free(ring_);
        device_free(pyr_);
        device_free(mask_buf_);
        device_free(filt_d_);
        device_free(csf_d_);
        device_free(partials_);
        device_free(vals_d_);
        device_free(merged_);
        device_free(dmap_);
        pinned_free(vals_h_);
        down_buf_ = up_buf_ = ring_ = pyr_ = mask_buf_ = filt_d_ = csf_d_ = merged_ = dmap_ = nullptr;
        partials_ = vals_d_ = vals_h_ = nullptr;
        if (last_done_) {
            (void)cudaEventDestroy(last_done_);
            last_done_ = nullptr;
        }
        if (stream_) {
            (void)cudaStreamDestroy(stream_);
            stream_ = nullptr;
        }
    }

    int device_ = 0;
    Display disp_;
    DisplayDev dd_{};
    Vship_Colorspace_t cs_[2]{};
    ClipGeometry geo_[2];
    ColourParams cp_[2]{};
    int trc_[2] = {0, 0}, prim_[2] = {0, 0};
    int64_t sw_ = 0, sh_ = 0, rw_ = 0, rh_ = 0, mw_ = 0, mh_ = 0;
    bool down_ = false, generic_ = false;
    int levels_ = 0, taps_ = 1, tsize_ = 0, ind0_ = 0;
    float band_freq_[kMaxLevels] = {};
    int64_t lw_[kMaxLevels] = {}, lh_[kMaxLevels] = {}, level_off_[kMaxLevels] = {};
    int64_t tile_off_[kMaxLevels] = {}, tiles_[kMaxLevels] = {}, tiles_x_[kMaxLevels] = {};
    int64_t chan_stride_ = 0;
    float lum0_ = 0.f, span_ = 1.f;
    float blur_w_[17] = {}, blur_prefix_[18] = {}, xcm2_[16] = {};
    int num_frame_ = 0;
    double sq_sum_ = 0.0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t last_done_ = nullptr;
    StagingBuffer staging_[2];
    GenericLinear lin_[2];
    float* down_buf_ = nullptr;
    float* up_buf_ = nullptr;
    float* ring_ = nullptr;
    float* pyr_ = nullptr;
    float* mask_buf_ = nullptr;  // per band: min(|R|,|T|) and |R-T| of each channel (8 planes)
    float* filt_d_ = nullptr;
    float* csf_d_ = nullptr;
    double* partials_ = nullptr;
    double* vals_d_ = nullptr;
    double* vals_h_ = nullptr;
    float* merged_ = nullptr;
    float* dmap_ = nullptr;
    KernelTimer timer_;
};

}  // namespace
}  // namespace cvvdp

CvvdpApi* make_cvvdp_engine() { return new cvvdp::Engine(); }

void cvvdp_display_model(const std::string& model_key, const std::string& model_config_json, VshipExt_CVVDPDisplay* out) {
    const cvvdp::Display d = cvvdp::resolve_display(model_key, model_config_json);
    out->width = d.res[0];
    out->height = d.res[1];
    out->hdr = d.hdr ? 1 : 0;
    out->viewing_distance_meters = d.distance;
    out->diagonal_size_inches = d.diagonal;
    out->max_luminance = d.max_lum;
    out->contrast = d.contrast;
    out->E_ambient = d.e_ambient;
    out->k_refl = d.k_refl;
    out->exposure = d.exposure;
    out->ppd = d.ppd();
    out->black_level = d.black();
    out->reflected_level = d.refl();
}

}  // namespace vship

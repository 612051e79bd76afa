// Butteraugli engine for B200 (sm_100a).
//
// The reference (src/butter/main.hpp:25-231) runs about 60 kernels per scale and image
// pair, each a full-plane pass: separable blurs as separate horizontal and vertical kernels
// and every band/diff/mask step as its own pointwise kernel.  This engine fuses the path into
// eight kernels per scale:
//
//   per image:  opsin    blur(sigma 1.2) of linear RGB + opsin dynamics          -> XYB
//               lf       blur(sigma 7.16, radius 21) of XYB in a row and a column pass,
//                        + low-frequency vals                                     -> lf, XYB-lf
//               mf       blur(sigma 3.22, radius 9) + mf range shaping + X-by-Y suppression
//               hf       blur(sigma 1.56) + hf/uhf split + psycho-mask precompute
//               mask     blur(sigma 2.7) of the mask precompute
//   per pair:   diffmap  6 Malta line filters, asymmetric L2 terms, mask L2, fuzzy erosion,
//                        MaskY / MaskDcY combination -> distortion map of the scale
//   final:      norms    2x supersampled combination of both scales, optional distmap
//                        output, FP64 partial sums of d^Q, |d|^3 and max|d|
//
// Every blur but lf's is a tiled separable renormalised truncated Gaussian: a (32+2R)^2 input
// tile in shared memory (zero outside the image), the horizontal pass into a second shared
// tile, the vertical pass into registers, each pass divided by the sum of its in-bounds taps
// (src/butter/gaussianblur.hpp:59-187).  All storage and arithmetic is FP32, as in the
// reference; only the norm sums are FP64.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>

#include "common.cuh"
#include "colour.cuh"
#include "frontend.cuh"
#include "metric_tables.h"
#include "engines.h"

namespace vship {
namespace butter {

constexpr int kTile = 32;
constexpr int kMaxTaps = 43;  // 2 * 21 + 1

// Gaussian taps and prefix sums of the five sigmas (src/butter/gaussianblur.hpp:3-43).
__constant__ float c_taps[5][kMaxTaps];
__constant__ float c_prefix[5][kMaxTaps + 1];

// Malta field parameters: [field] = {norm1, norm2 (primary), norm2 (half-open)}.
// Fields: 0 uhf Y, 1 uhf X (9-tap); 2 hf Y, 3 hf X, 4 mf Y, 5 mf X (5-tap).
__constant__ float c_malta[6][3];

// Weights of the L2 terms (src/butter/main.hpp:83-95 with the second 0.8 factor of
// L2AsymDiff, src/butter/simplerdiff.hpp:295-298): asym hf X/Y (gt, lt), mf X/Y/B, lf X/Y/B.
__constant__ float c_l2[12];

static void upload_constants() {
    float taps[5][kMaxTaps] = {};
    float prefix[5][kMaxTaps + 1] = {};
    const double tau = 6.283185307179586;
    for (int k = 0; k < 5; k++) {
        const int r = kButterRadius[k];
        const double sigma = kButterSigma[k];
        float acc = 0.f;
        prefix[k][0] = 0.f;
        for (int i = 0; i <= 2 * r; i++) {
            // Same expression and precision as loadGaussianKernel (gaussianblur.hpp:6-12).
            const float v = (float)((double)expf((float)(-(double)((r - i) * (r - i)) / (2 * sigma * sigma))) /
                                    std::sqrt(tau * sigma * sigma));
            taps[k][i] = v;
            acc += v;
            prefix[k][i + 1] = acc;
        }
    }
    CUDA_CHECK(cudaMemcpyToSymbol(c_taps, taps, sizeof(taps)));
    CUDA_CHECK(cudaMemcpyToSymbol(c_prefix, prefix, sizeof(prefix)));

    // MaltaDiffMap / MaltaDiffMapLF host parameters (main.hpp:57-81, maltaDiff.hpp:662-684)
    // and the per-kernel prologue (maltaDiff.hpp:519-526), in float as there.
    const float asym = 0.8f;
    struct F { float w_gt, w_lt, norm1; bool lf; };
    const F fields[6] = {
        {1.10039032555f * asym, 1.10039032555f / asym, 71.7800275169f, false},
        {173.5f * asym, 173.5f / asym, 5.0f, false},
        {18.7237414387f * std::sqrt(asym), 18.7237414387f / std::sqrt(asym), 4498534.45232f, true},
        {6923.99476109f * std::sqrt(asym), 6923.99476109f / std::sqrt(asym), 8051.15833247f, true},
        {37.0819870399f, 37.0819870399f, 130262059.556f, true},
        {8246.75321353f, 8246.75321353f, 1009002.70582f, true},
    };
    float malta[6][3];
    for (int f = 0; f < 6; f++) {
        const float len = 3.75f;
        const float mulli = fields[f].lf ? 0.611612573796f : 0.39905817637f;
        const float len2 = len * 2.0f + 1.0f;
        const float pre_gt = mulli * std::sqrt(0.5f * fields[f].w_gt) / len2;
        const float pre_lt = mulli * std::sqrt(0.33f * fields[f].w_lt) / len2;
        malta[f][0] = fields[f].norm1;
        malta[f][1] = pre_gt * fields[f].norm1;
        malta[f][2] = pre_lt * fields[f].norm1;
    }
    CUDA_CHECK(cudaMemcpyToSymbol(c_malta, malta, sizeof(malta)));

    const float wmul[9] = {400.0f, 1.50815703118f, 0.0f, 2150.0f, 10.6195433239f, 16.2176043152f,
                           29.2353797994f, 0.844626970982f, 0.703646627719f};
    float l2[12];
    for (int c = 0; c < 2; c++) {
        float gt = wmul[c] * asym, lt = wmul[c] / asym;
        gt = (float)((double)gt * 0.8);
        lt = (float)((double)lt * 0.8);
        l2[2 * c] = gt;
        l2[2 * c + 1] = lt;
    }
    for (int c = 0; c < 3; c++) l2[4 + c] = wmul[3 + c];
    for (int c = 0; c < 3; c++) l2[7 + c] = wmul[6 + c];
    l2[10] = 10.0f;
    l2[11] = 0.f;
    CUDA_CHECK(cudaMemcpyToSymbol(c_l2, l2, sizeof(l2)));
}

// ------------------------------------------------------------------------------------------
// Tiled separable blur helper
// ------------------------------------------------------------------------------------------

// One or two planes per blur: two planes travel as float2 through shared memory so that one
// packed FP32x2 FMA (sm_100) serves both, halving the tap arithmetic.
template <int NP> struct BlurVec;
template <> struct BlurVec<1> {
    using T = float;
    __device__ static float zero() { return 0.f; }
    __device__ static float fma(float g, float x, float acc) { return fmaf(x, g, acc); }
    __device__ static float scale(float x, float s) { return x * s; }
};
template <> struct BlurVec<2> {
    using T = float2;
    __device__ static float2 zero() { return make_float2(0.f, 0.f); }
    __device__ static float2 fma(float g, float2 x, float2 acc) { return __ffma2_rn(x, make_float2(g, g), acc); }
    __device__ static float2 scale(float2 x, float s) { return make_float2(x.x * s, x.y * s); }
};

template <int R, int NP>
struct BlurSmem {
    using V = typename BlurVec<NP>::T;
    static constexpr int IN = kTile + 2 * R;
    V in[IN][IN + 1];
    V h[IN][kTile + 1];
    float invx[kTile];   // 1 / in-image tap weight of each output column
    float invy[kTile];   // ... and row
};

__device__ __forceinline__ float tap_sum(int k, int R, int pos, int n) {
    const int beg = max(0, R - pos);
    const int end = min(2 * R + 1, n + R - pos);
    return c_prefix[k][end] - c_prefix[k][beg];
}

// Blurs NP planes over the CTA's 32x32 tile (origin X0, Y0): `src(x, y)` returns the input
// (a float, or a float2 of the two planes) at an in-image position.  Thread t gets column
// t&31, rows 4*(t>>5) .. +3 in out[0..3].  The per-position renormalisation (divide by the
// in-image tap weight, src/butter/gaussianblur.hpp) is applied as a tabulated reciprocal.
template <int R, int K, int NP, typename Src>
__device__ __forceinline__ void blur_tile(BlurSmem<R, NP>& sm, Src src, int X0, int Y0, int w, int h,
                                          typename BlurVec<NP>::T out[4]) {
    using B = BlurVec<NP>;
    using V = typename B::T;
    constexpr int IN = BlurSmem<R, NP>::IN;
    constexpr int NT = 2 * R + 1;
    const int tid = threadIdx.x;
    // Staging: warp k takes halo rows k, k + 8, ...; lane l columns l, l + 32, l + 64 of a
    // row, so each row's bounds test and base address are computed once and a warp's stores
    // fall in one row (no bank conflicts).  Two rows per step, all loads before the stores.
    {
        constexpr int kCols = (IN + 31) / 32;
        const int lane = tid & 31, warp = tid >> 5;
        for (int r0 = warp; r0 < IN; r0 += 16) {
            V v[2][kCols];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int r = r0 + 8 * s;
                const int gy = Y0 - R + r;
                const bool rowin = r < IN && (unsigned)gy < (unsigned)h;
#pragma unroll
                for (int k = 0; k < kCols; k++) {
                    const int c = lane + 32 * k, gx = X0 - R + c;
                    v[s][k] = (rowin && c < IN && (unsigned)gx < (unsigned)w) ? src(gx, gy) : B::zero();
                }
            }
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int r = r0 + 8 * s;
                if (r >= IN) break;
#pragma unroll
                for (int k = 0; k < kCols; k++)
                    if (lane + 32 * k < IN) sm.in[r][lane + 32 * k] = v[s][k];
            }
        }
    }
    if (tid < kTile)
        sm.invx[tid] = 1.0f / tap_sum(K, R, min(X0 + tid, w - 1), w);
    else if (tid < 2 * kTile)
        sm.invy[tid - kTile] = 1.0f / tap_sum(K, R, min(Y0 + tid - kTile, h - 1), h);
    __syncthreads();
    // Horizontal pass: a work item is four adjacent outputs of one row, each input sample
    // loaded once and applied to every output whose window holds it (taps in the same order
    // per output as one output at a time).
    for (int u = tid; u < IN * (kTile / 4); u += 256) {
        const int r = u >> 3, c0 = (u & 7) * 4;
        V a[4] = {B::zero(), B::zero(), B::zero(), B::zero()};
#pragma unroll
        for (int j = 0; j < NT + 3; j++) {
            const V v = sm.in[r][c0 + j];
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const int t = j - o;
                if (t >= 0 && t < NT) a[o] = B::fma(c_taps[K][t], v, a[o]);
            }
        }
#pragma unroll
        for (int o = 0; o < 4; o++) sm.h[r][c0 + o] = B::scale(a[o], sm.invx[c0 + o]);
    }
    __syncthreads();
    const int c = tid & 31, r0 = (tid >> 5) * 4;
    V acc[4] = {B::zero(), B::zero(), B::zero(), B::zero()};
#pragma unroll
    for (int j = 0; j < NT + 3; j++) {
        const V v = sm.h[r0 + j][c];
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const int t = j - o;
            if (t >= 0 && t < NT) acc[o] = B::fma(c_taps[K][t], v, acc[o]);
        }
    }
#pragma unroll
    for (int o = 0; o < 4; o++) {
        const int gy = Y0 + r0 + o;
        out[o] = gy < h ? B::scale(acc[o], sm.invy[r0 + o]) : B::zero();
    }
    __syncthreads();
}

// Two-plane and one-plane blurs of the same radius sharing one shared-memory block.
template <int R>
union BlurSmemPair {
    BlurSmem<R, 2> two;
    BlurSmem<R, 1> one;
};

// Blurs three planes (two packed, one alone) with the same kernel; bl[c][o] as blur_tile.
template <int R, int K, typename Src>
__device__ __forceinline__ void blur_three(BlurSmemPair<R>& sm, Src src, int X0, int Y0, int w, int h,
                                           float bl[3][4]) {
    float2 b01[4];
    blur_tile<R, K, 2>(sm.two, [&](int x, int y) { return make_float2(src(0, x, y), src(1, x, y)); }, X0, Y0, w, h, b01);
    blur_tile<R, K, 1>(sm.one, [&](int x, int y) { return src(2, x, y); }, X0, Y0, w, h, bl[2]);
#pragma unroll
    for (int o = 0; o < 4; o++) {
        bl[0][o] = b01[o].x;
        bl[1][o] = b01[o].y;
    }
}

// ------------------------------------------------------------------------------------------
// Per-image stage kernels
// ------------------------------------------------------------------------------------------

struct Planes {
    int w, h;
    const float* lin[3];
    float* xyb[3];
    float* lf[3];
    float* d[3];
    float* mf[3];
    float* hfpre[2];
    float* hf[2];
    float* uhf[2];
    float* p;
    float* pb;
    float intensity;
};

__device__ __forceinline__ float3 opsin_mix(float3 a, bool clamp) {  // colors.hpp:33-56
    float3 o;
    o.x = fmaf(0.29956550340058319f, a.x, fmaf(0.63373087833825936f, a.y, fmaf(0.077705617820981968f, a.z, 1.7557483643287353f)));
    o.y = fmaf(0.22158691104574774f, a.x, fmaf(0.69391388044116142f, a.y, fmaf(0.0987313588422f, a.z, 1.7557483643287353f)));
    o.z = fmaf(0.02f, a.x, fmaf(0.02f, a.y, fmaf(0.20480129041026129f, a.z, 12.226454707163354f)));
    if (clamp) {
        o.x = fmaxf(o.x, 1.7557483643287353f);
        o.y = fmaxf(o.y, 1.7557483643287353f);
        o.z = fmaxf(o.z, 12.226454707163354f);
    }
    return o;
}

__device__ __forceinline__ float butter_gamma(float v) {  // colors.hpp:3-5
    return fmaf(19.245013259874995f, logf((float)((double)v + 9.9710635769299145)), -23.16046239805755f);
}

// opsinDynamicsImage (colors.hpp:57-91).
__global__ void __launch_bounds__(256) opsin_kernel(Planes P) {
    __shared__ BlurSmemPair<8> sm;
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kTile;
    float bl[3][4];
    const int w = P.w;
    blur_three<8, 0>(sm, [&](int c, int x, int y) { return P.lin[c][(int64_t)y * w + x]; }, X0, Y0, P.w, P.h, bl);
    const int c = threadIdx.x & 31, r0 = (threadIdx.x >> 5) * 4;
    const int x = X0 + c;
    if (x >= P.w) return;
#pragma unroll
    for (int o = 0; o < 4; o++) {
        const int y = Y0 + r0 + o;
        if (y >= P.h) break;
        const int64_t i = (int64_t)y * P.w + x;
        const float m = P.intensity;
        float3 src = make_float3(P.lin[0][i] * m, P.lin[1][i] * m, P.lin[2][i] * m);
        float3 b = make_float3(bl[0][o] * m, bl[1][o] * m, bl[2][o] * m);
        b = opsin_mix(b, true);
        b.x = fmaxf(b.x, 1e-4f); b.y = fmaxf(b.y, 1e-4f); b.z = fmaxf(b.z, 1e-4f);
        float3 sens;
        sens.x = fmaxf(butter_gamma(b.x) / b.x, 1e-4f);
        sens.y = fmaxf(butter_gamma(b.y) / b.y, 1e-4f);
        sens.z = fmaxf(butter_gamma(b.z) / b.z, 1e-4f);
        src = opsin_mix(src, false);
        src.x *= sens.x; src.y *= sens.y; src.z *= sens.z;
        src.x = fmaxf(src.x, 1.7557483643287353f);
        src.y = fmaxf(src.y, 1.7557483643287353f);
        src.z = fmaxf(src.z, 12.226454707163354f);
        P.xyb[0][i] = src.x - src.y;
        P.xyb[1][i] = src.x + src.y;
        P.xyb[2][i] = src.z;
    }
}

// Low-frequency split (separatefrequencies.hpp:160-176, XybLowFreqToVals :3-12) as two
// passes of the radius-21 blur through an intermediate plane, as the reference runs it
// (separate horizontal and vertical kernels for radii above 8, gaussianblur.hpp:60-250): a
// 32x32 tile of the fused form blurs 74 halo rows horizontally for 32 output rows and stages
// 74^2 samples for 1,024 outputs, while the row pass blurs each row once and the column pass
// stages 106 rows for 64.  Measured per 4K pair: 0.64 ms against 0.68 for the tiled form (the
// pass is latency-bound; five column-pass CTAs per SM, 48 registers, beat fewer CTAs with
// more rows per thread).  The intermediate lives in the mf planes, which the mf kernel
// writes only afterwards.  Per output, the taps and the renormalisation are applied in the
// same order as in blur_tile, so the values are those of the tiled blur.
constexpr int kLfR = 21;
constexpr int kLfNT = 2 * kLfR + 1;
constexpr int kLfK = 4;                 // tap set of sigma 7.16
constexpr int kLfHW = 128;              // row pass: 32 rows x 128 columns per CTA
constexpr int kLfVRows = 64;            // column pass: 64 rows x 32 columns per CTA
constexpr int kLfRPT = kLfVRows / 8;    // rows per thread
constexpr int kLfVIn = kLfVRows + 2 * kLfR;

// Row pass of plane blockIdx.z: xyb -> mf (horizontal blur, renormalised per column).  The
// CTA stages a dense box of 32 rows x kLfHBox columns starting kLfHPad columns left of its
// first output (the halo rounded out to a multiple of 4, so that every 4-column group of the
// box is a 16-byte word); warp k blurs rows k, k + 8, k + 16, k + 24 and lane l the outputs
// 4l .. 4l + 3 of a row, reading its 52-column window as 13 float4 (a warp reads 512
// consecutive bytes: no bank conflicts) and writing its four outputs as one float4 when the
// plane row allows.  Per output, the taps are applied in the same order as in blur_tile.
constexpr int kLfHPad = (kLfR + 3) / 4 * 4;        // 24
constexpr int kLfHBox = kLfHW + 2 * kLfHPad;       // 176
constexpr int kLfHWin = (3 + kLfNT + 3 + 3) / 4;   // float4 per lane window: 13

__global__ void __launch_bounds__(256) lf_row_kernel(Planes P) {
    __shared__ alignas(16) float in[32][kLfHBox];
    __shared__ float invx[kLfHW];
    const int c = blockIdx.z;
    const int X0 = blockIdx.x * kLfHW, Y0 = blockIdx.y * 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int w = P.w, h = P.h;
    const float* src = P.xyb[c];
    // Staging: warp k takes rows k, k + 8, k + 16, k + 24; lanes the columns.
    constexpr int kCols = (kLfHBox + 31) / 32;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const int r = warp + 8 * s, gy = Y0 + r;
        const bool rowin = gy < h;
        const float* row = src + (int64_t)(rowin ? gy : 0) * w;
        float v[kCols];
#pragma unroll
        for (int k = 0; k < kCols; k++) {
            const int cc = lane + 32 * k, gx = X0 - kLfHPad + cc;
            v[k] = (rowin && cc < kLfHBox && (unsigned)gx < (unsigned)w) ? row[gx] : 0.f;
        }
#pragma unroll
        for (int k = 0; k < kCols; k++)
            if (lane + 32 * k < kLfHBox) in[r][lane + 32 * k] = v[k];
    }
    if (tid < kLfHW) invx[tid] = 1.0f / tap_sum(kLfK, kLfR, min(X0 + tid, w - 1), w);
    __syncthreads();
    float* dst = P.mf[c];
    const int c0 = 4 * lane;  // first output of the lane; its taps start at box column c0 + 3
    const int gx0 = X0 + c0;
#pragma unroll 1
    for (int s = 0; s < 4; s++) {
        const int r = warp + 8 * s, gy = Y0 + r;
        if (gy >= h) break;  // uniform over the warp
        float win[4 * kLfHWin];
#pragma unroll
        for (int m = 0; m < kLfHWin; m++) {
            const float4 q = *reinterpret_cast<const float4*>(&in[r][c0 + 4 * m]);
            win[4 * m] = q.x; win[4 * m + 1] = q.y; win[4 * m + 2] = q.z; win[4 * m + 3] = q.w;
        }
        float a[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int j = 0; j < kLfNT + 3; j++) {
            const float v = win[kLfHPad - kLfR + j];
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const int t = j - o;
                if (t >= 0 && t < kLfNT) a[o] = fmaf(v, c_taps[kLfK][t], a[o]);
            }
        }
#pragma unroll
        for (int o = 0; o < 4; o++) a[o] = a[o] * invx[c0 + o];
        if (gx0 >= w) continue;
        float* out = dst + (int64_t)gy * w + gx0;
        if (gx0 + 4 <= w && (reinterpret_cast<uintptr_t>(out) & 15) == 0) {
            *reinterpret_cast<float4*>(out) = make_float4(a[0], a[1], a[2], a[3]);
        } else {
#pragma unroll
            for (int o = 0; o < 4; o++)
                if (gx0 + o < w) out[o] = a[o];
        }
    }
}

// Vertical pass of plane c over a staged box (kLfVIn rows of 32 columns, row pitch PITCH
// floats) and the low-frequency epilogue: lf and xyb - blur.  Thread t: column t & 31, rows
// kLfRPT (t >> 5) .. + kLfRPT - 1 of the CTA's kLfVRows.  Plane 2's value needs plane 1's blur,
// which the caller keeps in by[] between the calls.
template <int PITCH>
__device__ __forceinline__ void lf_col_plane(const Planes& P, const float* box, const float* invy, int c, int X0,
                                             int Y0, float (&by)[kLfRPT]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int w = P.w, h = P.h;
    const int x = X0 + lane, r0 = warp * kLfRPT;
    float acc[kLfRPT];
#pragma unroll
    for (int o = 0; o < kLfRPT; o++) acc[o] = 0.f;
#pragma unroll
    for (int j = 0; j < kLfNT + kLfRPT - 1; j++) {
        const float v = box[(r0 + j) * PITCH + lane];
#pragma unroll
        for (int o = 0; o < kLfRPT; o++) {
            const int t = j - o;
            if (t >= 0 && t < kLfNT) acc[o] = fmaf(v, c_taps[kLfK][t], acc[o]);
        }
    }
    if (x >= w) return;
#pragma unroll
    for (int o = 0; o < kLfRPT; o++) {
        const int y = Y0 + r0 + o;
        if (y >= h) break;
        const int64_t i = (int64_t)y * w + x;
        const float bl = acc[o] * invy[r0 + o];
        P.d[c][i] = P.xyb[c][i] - bl;
        if (c == 0) {
            float vx = bl;
            vx = vx * 33.832837186260f;
            P.lf[0][i] = vx;
        } else if (c == 1) {
            by[o] = bl;
            float vy = bl;
            vy = vy * 14.458268100570f;
            P.lf[1][i] = vy;
        } else {
            float vb = bl;
            vb = vb + -0.362267051518f * by[o];
            vb = vb * 49.87984651440f;
            P.lf[2][i] = vb;
        }
    }
}

// Column pass: mf (row-blurred) -> lf and xyb - blur for the three planes in turn, each box
// staged with plain loads into a padded shared tile (any plane width).
__global__ void __launch_bounds__(256, 5) lf_col_kernel(Planes P) {
    __shared__ float hs[kLfVIn][kTile + 1];
    __shared__ float invy[kLfVRows];
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kLfVRows;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int w = P.w, h = P.h;
    const int x = X0 + lane;
    if (tid < kLfVRows) invy[tid] = 1.0f / tap_sum(kLfK, kLfR, min(Y0 + tid, h - 1), h);
    float by[kLfRPT];
#pragma unroll 1
    for (int c = 0; c < 3; c++) {
        if (c) __syncthreads();  // the previous plane's pass has read hs
        const float* src = P.mf[c];
        for (int rb = warp; rb < kLfVIn; rb += 32) {
            float v[4];
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const int r = rb + 8 * s, gy = Y0 - kLfR + r;
                v[s] = (r < kLfVIn && (unsigned)gy < (unsigned)h && x < w) ? src[(int64_t)gy * w + x] : 0.f;
            }
#pragma unroll
            for (int s = 0; s < 4; s++)
                if (rb + 8 * s < kLfVIn) hs[rb + 8 * s][lane] = v[s];
        }
        __syncthreads();
        lf_col_plane<kTile + 1>(P, &hs[0][0], invy, c, X0, Y0, by);
    }
}

// The same column pass with each plane's box brought into shared memory by the tensor-memory
// accelerator (a tiled cp.async.bulk.tensor load of this GPU's own mf plane, no multicast),
// double-buffered across the three planes: plane c + 2's box loads while plane c + 1 is
// blurred.  The box is dense (32 floats per row), which suits this pass: a warp reads one row
// of it at a time, so no padding is needed against bank conflicts.  The box origin's x is a
// multiple of 32 floats (128 bytes); rows above and below the plane read as zero (the tensor
// map's out-of-bounds fill), as do columns past its width.  Used when the plane's row pitch
// (its width in bytes) is a multiple of 16, which a tensor map requires.
struct LfColMaps {
    CUtensorMap m[3];  // the three mf planes of one image at one scale, box 32 x kLfVIn
};

constexpr unsigned kLfBoxBytes = kLfVIn * kTile * sizeof(float);
constexpr long long kTmaWaitLimit = 1ll << 24;  // polls of a box's barrier before giving up
constexpr long long kTmaTestWaitLimit = 1ll << 12;  // the same under the test hook

__device__ __forceinline__ void lf_box_load(const CUtensorMap* map, float* dst, uint64_t* bar, int x, int y) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kLfBoxBytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(b)
        : "memory");
}

// Polls the barrier's phase `parity` at most `limit` times; false if it did not complete.
__device__ __forceinline__ bool lf_box_wait(uint64_t* bar, unsigned parity, long long limit) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    for (long long i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done) : "r"(b), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// `test_skip`: the test hook's launch; plane 0's barrier is armed but its box is never
// loaded, so its wait runs out (after kTmaTestWaitLimit polls) and the error path runs.
__global__ void __launch_bounds__(256, 5) lf_col_tma_kernel(Planes P, const __grid_constant__ LfColMaps maps,
                                                            int* __restrict__ err, int test_skip) {
    __shared__ alignas(128) float box[2][kLfVIn * kTile];
    __shared__ float invy[kLfVRows];
    __shared__ alignas(8) uint64_t bar[2];
    __shared__ int ok[3];
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kLfVRows;
    const int tid = threadIdx.x, h = P.h;
    if (tid == 0) {
        for (int b = 0; b < 2; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&bar[b])) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (test_skip)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         ::"r"((uint32_t)__cvta_generic_to_shared(&bar[0])), "r"(kLfBoxBytes) : "memory");
        else
            lf_box_load(&maps.m[0], box[0], &bar[0], X0, Y0 - kLfR);
        lf_box_load(&maps.m[1], box[1], &bar[1], X0, Y0 - kLfR);
    }
    const long long limit = test_skip ? kTmaTestWaitLimit : kTmaWaitLimit;
    if (tid < kLfVRows) invy[tid] = 1.0f / tap_sum(kLfK, kLfR, min(Y0 + tid, h - 1), h);
    float by[kLfRPT];
#pragma unroll 1
    for (int c = 0; c < 3; c++) {
        const int b = c & 1;
        // One thread waits for the box; the barrier then hands its data to the whole CTA.
        if (tid == 0) {
            ok[c] = lf_box_wait(&bar[b], (unsigned)(c >> 1), limit);
            if (!ok[c]) {
                *(volatile int*)err = 1;  // mapped host memory: a plain store (every writer stores 1)
                // Before the CTA leaves, the other box still loading must land: plane 1's
                // (issued at the start) while plane 0 is awaited, plane 2's while plane 1 is.
                if (c == 0) (void)lf_box_wait(&bar[1], 0u, kTmaWaitLimit);
                if (c == 1) (void)lf_box_wait(&bar[0], 1u, kTmaWaitLimit);
            }
        }
        __syncthreads();
        if (!ok[c]) return;  // uniform: every thread reads the same flag
        lf_col_plane<kTile>(P, box[b], invy, c, X0, Y0, by);
        if (c == 0) {
            __syncthreads();  // every thread has read box 0
            if (tid == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                lf_box_load(&maps.m[2], box[0], &bar[0], X0, Y0 - kLfR);
            }
        }
    }
}

__device__ __forceinline__ float remove_range(float x, float w) { return x > w ? x - w : x < -w ? x + w : 0.0f; }
__device__ __forceinline__ float amplify_range(float x, float w) { return x > w ? x + w : x < -w ? x - w : 2.0f * x; }
__device__ __forceinline__ float maximum_clamp(float v, float maxval) {
    const float k = 0.688059627878f;
    if (v >= maxval) { v -= maxval; v *= k; v += maxval; }
    else if (v < -maxval) { v += maxval; v *= k; v -= maxval; }
    return v;
}

// Medium-frequency split and X-by-Y suppression (separatefrequencies.hpp:161-187).
__global__ void __launch_bounds__(256) mf_kernel(Planes P) {
    __shared__ BlurSmemPair<9> sm;
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kTile;
    float bl[3][4];
    const int w = P.w;
    blur_three<9, 3>(sm, [&](int c, int x, int y) { return P.d[c][(int64_t)y * w + x]; }, X0, Y0, P.w, P.h, bl);
    const int c = threadIdx.x & 31, r0 = (threadIdx.x >> 5) * 4;
    const int x = X0 + c;
    if (x >= P.w) return;
#pragma unroll
    for (int o = 0; o < 4; o++) {
        const int y = Y0 + r0 + o;
        if (y >= P.h) break;
        const int64_t i = (int64_t)y * P.w + x;
        float hx = P.d[0][i] - bl[0][o];
        const float hy = P.d[1][i] - bl[1][o];
        P.mf[0][i] = remove_range(bl[0][o], 0.29f);
        P.mf[1][i] = amplify_range(bl[1][o], 0.1f);
        P.mf[2][i] = bl[2][o];
        const float s = 0.653020556257f, yw = 46.0f;
        hx *= s + (yw * (1.0f - s)) / (yw + hy * hy);
        P.hfpre[0][i] = hx;
        P.hfpre[1][i] = hy;
    }
}

// High / ultra-high split (separatefrequencies.hpp:189-200, :117-133) and the psycho-mask
// precompute of this image (maskPsycho.hpp:4-40, 120-128).
__global__ void __launch_bounds__(256) hf_kernel(Planes P) {
    __shared__ BlurSmem<8, 2> sm;
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kTile;
    float bl[2][4];
    const int w = P.w;
    {
        float2 b01[4];
        blur_tile<8, 1, 2>(sm, [&](int x, int y) {
            const int64_t i = (int64_t)y * w + x;
            return make_float2(P.hfpre[0][i], P.hfpre[1][i]);
        }, X0, Y0, P.w, P.h, b01);
#pragma unroll
        for (int o = 0; o < 4; o++) {
            bl[0][o] = b01[o].x;
            bl[1][o] = b01[o].y;
        }
    }
    const int c = threadIdx.x & 31, r0 = (threadIdx.x >> 5) * 4;
    const int x = X0 + c;
    if (x >= P.w) return;
#pragma unroll
    for (int o = 0; o < 4; o++) {
        const int y = Y0 + r0 + o;
        if (y >= P.h) break;
        const int64_t i = (int64_t)y * P.w + x;
        float hf0 = bl[0][o];
        float uhf0 = P.hfpre[0][i] - hf0;
        hf0 = remove_range(hf0, 1.5f);
        uhf0 = remove_range(uhf0, 0.04f);
        float hf1 = maximum_clamp(bl[1][o], 28.4691806922f);
        float uhf1 = P.hfpre[1][i] - hf1;
        uhf1 = maximum_clamp(uhf1, 5.19175294647f);
        uhf1 *= 2.69313763794f;
        hf1 *= 2.155f;
        hf1 = amplify_range(hf1, 0.132f);
        P.hf[0][i] = hf0;
        P.hf[1][i] = hf1;
        P.uhf[0][i] = uhf0;
        P.uhf[1][i] = uhf1;
        const float xd = (uhf0 + hf0) * 2.5f;
        const float yd = uhf1 * 0.4f + hf1 * 0.4f;
        const float mk = sqrtf(xd * xd + yd * yd);
        const float mul = 6.19424080439f, bias = mul * 12.61050594197f;
        P.p[i] = sqrtf(mul * fabsf(mk) + bias) - sqrtf(bias);
    }
}

// Blur of the mask precompute (maskPsycho.hpp:129-132).
__global__ void __launch_bounds__(256) mask_kernel(Planes P) {
    __shared__ BlurSmem<8, 1> sm;
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kTile;
    float bl[4];
    const float* src = P.p;
    const int w = P.w;
    blur_tile<8, 2, 1>(sm, [&](int x, int y) { return src[(int64_t)y * w + x]; }, X0, Y0, P.w, P.h, bl);
    const int c = threadIdx.x & 31, r0 = (threadIdx.x >> 5) * 4;
    const int x = X0 + c;
    if (x >= P.w) return;
#pragma unroll
    for (int o = 0; o < 4; o++) {
        const int y = Y0 + r0 + o;
        if (y >= P.h) break;
        P.pb[(int64_t)y * P.w + x] = bl[o];
    }
}

// ------------------------------------------------------------------------------------------
// Per-pair distortion map of one scale
// ------------------------------------------------------------------------------------------

struct DiffArgs {
    int w, h;
    const float* f0[6];   // Malta fields, reference image: uhf Y, uhf X, hf Y, hf X, mf Y, mf X
    const float* f1[6];   // same, distorted image
    const float* hf[2][2];
    const float* mf[2][3];
    const float* lf[2][3];
    const float* pb[2];
    float* out;
};

// Malta difference field of one pixel (maltaDiff.hpp:542-577).
__device__ __forceinline__ float malta_field(float l0, float l1, int f) {
    const float norm1 = c_malta[f][0];
    const float absval = 0.5f * fabsf(l0) + 0.5f * fabsf(l1);
    const float diff = l0 - l1;
    const float scaler = c_malta[f][1] / (norm1 + absval);
    float d = scaler * diff;
    const float scaler2 = c_malta[f][2] / (norm1 + absval);
    const float fabs0 = fabsf(l0);
    const float too_small = 0.55f * fabs0, too_big = 1.05f * fabs0;
    float impact = 0.0f;
    if (l0 < 0.0f) {
        if (l1 > -too_small) impact = l1 + too_small;
        else if (l1 < -too_big) impact = -l1 - too_big;
    } else {
        if (l1 < too_small) impact = -l1 + too_small;
        else if (l1 > too_big) impact = l1 - too_big;
    }
    impact *= scaler2;
    return diff < 0.0f ? d - impact : d + impact;
}

constexpr int kMH = 4;                 // Malta halo
constexpr int kMIn = kTile + 2 * kMH;  // 40
constexpr int kEH = 3;                 // erosion halo
constexpr int kEIn = kTile + 2 * kEH;  // 38

// Malta line filter of one pixel: sum over the 16 patterns of the squared sum of the field
// along the pattern (MaltaUnit / MaltaUnitLF, maltaDiff.hpp:4-512).  The offset tables are
// compile-time constants, so after unrolling every tap is an immediate shared-memory offset.
template <bool HF>
__device__ __forceinline__ float malta_sum(const float (*fd)[kMIn + 1], int cy, int cx) {
    constexpr int NT = HF ? 9 : 5;
    constexpr vship_malta_tap hf[16][9] = VSHIP_MALTA_HF_TAPS;
    constexpr vship_malta_tap lf[16][5] = VSHIP_MALTA_LF_TAPS;
    float r = 0.f;
#pragma unroll
    for (int p = 0; p < 16; p++) {
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < NT; t++) {
            const int dx = HF ? hf[p][t].dx : lf[p][t % 5].dx;
            const int dy = HF ? hf[p][t].dy : lf[p][t % 5].dy;
            if (dx == VSHIP_MALTA_PAD) continue;
            s += fd[cy + dy][cx + dx];
        }
        r += s * s;
    }
    return r;
}

__device__ __forceinline__ void store_min3(float v, float& m0, float& m1, float& m2) {  // maskPsycho.hpp:42-55
    if (v < m2) {
        if (v < m0) { m2 = m1; m1 = m0; m0 = v; }
        else if (v < m1) { m2 = m1; m1 = v; }
        else m2 = v;
    }
}

__device__ __forceinline__ float mask_y(float delta) {  // combineMasks.hpp:3-11
    const float c = 2.5485944793f / ((0.451936922203f * delta) + 0.829591754942f);
    const float r = (float)((1.0 + (double)c) * (1.0 / (double)(0.79079917404f * 17.83f)));
    return r * r;
}

__device__ __forceinline__ float mask_dc_y(float delta) {  // combineMasks.hpp:13-20
    const float c = 0.505054525019f / ((3.87449418804f * delta) + 0.20025578522f);
    const float r = (float)((1.0 + (double)c) * (1.0 / (double)(0.79079917404f * 17.83f)));
    return r * r;
}


__global__ void __launch_bounds__(256) diffmap_kernel(DiffArgs a) {
    __shared__ float fd[6][kMIn][kMIn + 1];
    __shared__ float spb[kEIn][kEIn + 1];
    const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kTile;
    const int tid = threadIdx.x;
    for (int i = tid; i < kMIn * kMIn; i += 256) {
        const int r = i / kMIn, c = i % kMIn;
        const int gx = X0 - kMH + c, gy = Y0 - kMH + r;
        const bool in = gx >= 0 && gx < a.w && gy >= 0 && gy < a.h;
        const int64_t o = (int64_t)gy * a.w + gx;
#pragma unroll
        for (int f = 0; f < 6; f++) fd[f][r][c] = in ? malta_field(a.f0[f][o], a.f1[f][o], f) : 0.f;
    }
    for (int i = tid; i < kEIn * kEIn; i += 256) {
        const int r = i / kEIn, c = i % kEIn;
        const int gx = X0 - kEH + c, gy = Y0 - kEH + r;
        spb[r][c] = (gx >= 0 && gx < a.w && gy >= 0 && gy < a.h) ? a.pb[0][(int64_t)gy * a.w + gx] : 0.f;
    }
    __syncthreads();
    const int c = tid & 31, r0 = (tid >> 5) * 4;
    const int x = X0 + c;
    if (x >= a.w) return;
    for (int o = 0; o < 4; o++) {
        const int y = Y0 + r0 + o;
        if (y >= a.h) break;
        const int64_t i = (int64_t)y * a.w + x;
        const int cy = r0 + o + kMH, cx = c + kMH;
        // Accumulation order of each channel follows getdiffmap (main.hpp:61-102).
        float ac0 = 0.f, ac1 = 0.f, ac2 = 0.f;
        ac1 += malta_sum<true>(fd[0], cy, cx);
        ac0 += malta_sum<true>(fd[1], cy, cx);
        ac1 += malta_sum<false>(fd[2], cy, cx);
        ac0 += malta_sum<false>(fd[3], cy, cx);
        ac1 += malta_sum<false>(fd[4], cy, cx);
        ac0 += malta_sum<false>(fd[5], cy, cx);
        // Asymmetric L2 of hf (simplerdiff.hpp:263-293) and L2 of mf / lf (:244-253).
#pragma unroll
        for (int ch = 0; ch < 2; ch++) {
            const float s1 = a.hf[0][ch][i], s2 = a.hf[1][ch][i];
            const float wgt = c_l2[2 * ch], wlt = c_l2[2 * ch + 1];
            float& acc = ch == 0 ? ac0 : ac1;
            const float diff = s1 - s2;
            acc += wgt * diff * diff;
            const float fabs0 = fabsf(s1);
            const float too_small = (float)(0.4 * (double)fabs0), too_big = fabs0;
            if (s1 < 0) {
                if (s2 > -too_small) { const float v = s2 + too_small; acc += wlt * v * v; }
                else if (s2 < -too_big) { const float v = -s2 - too_big; acc += wlt * v * v; }
            } else {
                if (s2 < too_small) { const float v = too_small - s2; acc += wlt * v * v; }
                else if (s2 > too_big) { const float v = s2 - too_big; acc += wlt * v * v; }
            }
        }
        float dc0, dc1, dc2;
        {
            float dm;
            dm = a.mf[0][0][i] - a.mf[1][0][i]; ac0 += c_l2[4] * dm * dm;
            dm = a.mf[0][1][i] - a.mf[1][1][i]; ac1 += c_l2[5] * dm * dm;
            dm = a.mf[0][2][i] - a.mf[1][2][i]; ac2 += c_l2[6] * dm * dm;
            dm = a.lf[0][0][i] - a.lf[1][0][i]; dc0 = c_l2[7] * dm * dm;
            dm = a.lf[0][1][i] - a.lf[1][1][i]; dc1 = c_l2[8] * dm * dm;
            dm = a.lf[0][2][i] - a.lf[1][2][i]; dc2 = c_l2[9] * dm * dm;
        }
        const float b0 = spb[r0 + o + kEH][c + kEH];
        {
            const float dm = b0 - a.pb[1][i];
            ac1 += c_l2[10] * dm * dm;
        }
        // Fuzzy erosion of the reference image's blurred mask (maskPsycho.hpp:57-104).
        float m0 = b0, m1 = 2.0f * m0, m2 = m1;
        const int ey = r0 + o + kEH, ex = c + kEH;
        if (x >= 3) {
            store_min3(spb[ey][ex - 3], m0, m1, m2);
            if (y >= 3) store_min3(spb[ey - 3][ex - 3], m0, m1, m2);
            if (y < a.h - 3) store_min3(spb[ey + 3][ex - 3], m0, m1, m2);
        }
        if (x < a.w - 3) {
            store_min3(spb[ey][ex + 3], m0, m1, m2);
            if (y >= 3) store_min3(spb[ey - 3][ex + 3], m0, m1, m2);
            if (y < a.h - 3) store_min3(spb[ey + 3][ex + 3], m0, m1, m2);
        }
        if (y >= 3) store_min3(spb[ey - 3][ex], m0, m1, m2);
        if (y < a.h - 3) store_min3(spb[ey + 3][ex], m0, m1, m2);
        const float mask = 0.45f * m0 + 0.3f * m1 + 0.25f * m2;
        a.out[i] = sqrtf(mask_y(mask) * (ac0 + ac1 + ac2) + mask_dc_y(mask) * (dc0 + dc1 + dc2));
    }
}

// ------------------------------------------------------------------------------------------
// Two-scale combination and norms (downupsample.hpp:294-308, diffnorms.hpp:86-130)
// ------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) combine_norms_kernel(float* d0, const float* d1, int w, int h, int w1, int qnorm,
                                                            float* distmap, int64_t dst_pitch, double* partials) {
    __shared__ double red[8][3];
    const int64_t n = (int64_t)w * h;
    double sq = 0.0, s3 = 0.0, mx = 0.0;
    const float fq = (float)qnorm;
    for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
        const int y = (int)(i / w), x = (int)(i % w);
        float v = d0[i];
        v = (float)((double)v * (1.0 - 0.3 * 0.5));
        v += 0.5f * d1[(int64_t)(y / 2) * w1 + x / 2];
        if (distmap) distmap[(int64_t)y * dst_pitch + x] = v;
        sq += (double)powf(v, fq);
        s3 += (double)(fabsf(v) * v * v);
        mx = fmax(mx, (double)fabsf(v));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sq += __shfl_xor_sync(0xffffffffu, sq, off);
        s3 += __shfl_xor_sync(0xffffffffu, s3, off);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[warp][0] = sq; red[warp][1] = s3; red[warp][2] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, m = 0;
        for (int k = 0; k < 8; k++) { a += red[k][0]; b += red[k][1]; m = fmax(m, red[k][2]); }
        partials[blockIdx.x * 3 + 0] = a;
        partials[blockIdx.x * 3 + 1] = b;
        partials[blockIdx.x * 3 + 2] = m;
    }
}

__global__ void norms_final_kernel(const double* partials, int nblocks, int64_t n, int qnorm, double* norms) {
    __shared__ double red[8][3];
    double a = 0, b = 0, m = 0;
    for (int i = threadIdx.x; i < nblocks; i += 256) {
        a += partials[i * 3];
        b += partials[i * 3 + 1];
        m = fmax(m, partials[i * 3 + 2]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    }
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5][0] = a; red[threadIdx.x >> 5][1] = b; red[threadIdx.x >> 5][2] = m; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0, sb = 0, sm = 0;
        for (int k = 0; k < 8; k++) { sa += red[k][0]; sb += red[k][1]; sm = fmax(sm, red[k][2]); }
        norms[0] = pow(sa / (double)n, 1.0 / (double)qnorm);
        norms[1] = pow(sb / (double)n, 1.0 / 3.0);
        norms[2] = sm;
    }
}

__global__ void downsample_kernel(const float* src, float* dst, int w, int h) {  // downupsample.hpp:4-20
    const int nw = (w - 1) / 2 + 1, nh = (h - 1) / 2 + 1;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nw || y >= nh) return;
    const int x0 = min(2 * x, w - 1), x1 = min(2 * x + 1, w - 1), y0 = min(2 * y, h - 1), y1 = min(2 * y + 1, h - 1);
    float v = 0.0f;
    v += src[(int64_t)y0 * w + x0];
    v += src[(int64_t)y1 * w + x0];
    v += src[(int64_t)y0 * w + x1];
    v += src[(int64_t)y1 * w + x1];
    dst[(int64_t)y * nw + x] = v * 0.25f;
}

__global__ void copy_window_kernel(const float* src, int64_t src_pitch, int64_t src_plane, float* dst, int64_t dst_plane,
                                   int w, int h) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)w * h;
    if (i >= n) return;
    const int64_t y = i / w, x = i % w;
    for (int c = 0; c < 3; c++) dst[c * dst_plane + i] = src[c * src_plane + y * src_pitch + x];
}

// ------------------------------------------------------------------------------------------
// Engine
// ------------------------------------------------------------------------------------------


// cuTensorMapEncodeTiled through the runtime's driver entry point (the library links only the
// CUDA runtime); null if the driver does not provide it.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// Tensor map of a dense w x h float plane read in boxes of 32 x kLfVIn, zero outside the
// plane.  False when a tensor map cannot describe the plane (row pitch not a multiple of 16
// bytes, base not 16-byte aligned) or the driver refuses it: the caller then uses the
// plain-load column pass.
static bool encode_plane_map(CUtensorMap* m, const float* base, int w, int h) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn || w % 4 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    const cuuint64_t dim[2] = {(cuuint64_t)w, (cuuint64_t)h};
    const cuuint64_t stride[1] = {(cuuint64_t)w * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kTile, (cuuint32_t)kLfVIn};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dim, stride, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

class Engine final : public ButterApi {
public:
    ~Engine() override { release(); }

    void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, int qnorm, float intensity, int device) override {
        device_ = device;
        cs_[0] = src;
        cs_[1] = dis;
        geo_[0] = make_geometry(src);
        geo_[1] = make_geometry(dis);
        if (geo_[0].OW != geo_[1].OW || geo_[0].OH != geo_[1].OH) VSHIP_THROW(Vship_DifferingInputType, "");
        w_ = (int)geo_[0].OW;
        h_ = (int)geo_[0].OH;
        qnorm_ = qnorm;
        intensity_ = intensity;
        for (int c = 0; c < 2; c++) cp_[c] = make_colour_params(cs_[c], geo_[c], false);
        generic_ = geo_[0].generic() || geo_[1].generic();
        CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        CUDA_CHECK(cudaEventCreateWithFlags(&last_done_, cudaEventDisableTiming));
        CUDA_CHECK(cudaStreamCreateWithFlags(&aux_, cudaStreamNonBlocking));
        CUDA_CHECK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
        CUDA_CHECK(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
        upload_constants();
        for (int c = 0; c < 2; c++) {
            int64_t off[3];
            staging_[c].ensure((size_t)dense_image_bytes(geo_[c], off), stream_);
            if (generic_) lin_generic_[c].alloc(geo_[c]);
        }
        const int64_t n0 = (int64_t)w_ * h_;
        // Per image: lin 3, half lin 3, xyb 3, lf 3, d 3, mf 3, hfpre 2, hf 2, uhf 2, p 1, pb 1.
        const int per_image = 26;
        plane_floats_ = round_up(n0, 64);
        pool_ = device_alloc<float>((size_t)(2 * per_image + 2) * plane_floats_, "butteraugli planes");
        nblocks_ = 148 * 8;
        partials_ = device_alloc<double>((size_t)nblocks_ * 3, "norm partials");
        norms_d_ = device_alloc<double>(3, "norms");
        norms_host_ = pinned_alloc<double>(3, "norms");
        // Error word of the tensor-map column pass, in mapped pinned memory so that a call can
        // read what an earlier asynchronous call reported without synchronising.
        CUDA_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&tma_err_host_), sizeof(int), cudaHostAllocMapped));
        *tma_err_host_ = 0;
        CUDA_CHECK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&tma_err_dev_), tma_err_host_, 0));
        const int w1 = (w_ - 1) / 2 + 1, h1 = (h_ - 1) / 2 + 1;
        for (int sc = 0; sc < 2; sc++) {
            const int w = sc ? w1 : w_, h = sc ? h1 : h_;
            bool ok = true;
            for (int im = 0; im < 2; im++) {
                const Planes P = planes_of(im, w, h, sc == 1);
                for (int c = 0; c < 3; c++) ok = ok && encode_plane_map(&lf_maps_[im][sc].m[c], P.mf[c], w, h);
            }
            lf_tma_[sc] = ok;
        }
    }

    // Reports (once) a tensor-map load that an earlier call gave up waiting for.
    void check_tma_error() {
        if (tma_err_host_ && *(volatile int*)tma_err_host_) {
            *(volatile int*)tma_err_host_ = 0;
            VSHIP_THROW(Vship_HIPError, "a tensor-memory load of the low-frequency blur did not complete in time");
        }
    }

    void compute(double norms[3], uint8_t* dstp, int64_t dststride, const uint8_t* const s1[3], const uint8_t* const s2[3],
                 const int64_t ls1[3], const int64_t ls2[3]) override {
        check_tma_error();
        CUDA_CHECK(cudaStreamWaitEvent(stream_, last_done_, 0));
        RawImage raw[2];
        ColourParams cp[2] = {cp_[0], cp_[1]};
        for (int c = 0; c < 2; c++) {
            raw[c] = stage_host_image(staging_[c], geo_[c], c ? s2 : s1, c ? ls2 : ls1, stream_);
            cp[c].misaligned = misaligned_view(raw[c], geo_[c]) ? 1 : 0;
        }
        float* dmap = nullptr;
        if (dstp) {
            if (dststride < (int64_t)w_ * 4) VSHIP_THROW(Vship_BadPointer, "dststride smaller than width * 4");
            ensure_distmap();
            dmap = distmap_d_;
        }
        run(raw, cp, stream_, norms_d_, dmap, w_);
        CUDA_CHECK(cudaMemcpyAsync(norms_host_, norms_d_, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        if (dstp)
            CUDA_CHECK(cudaMemcpy2DAsync(dstp, (size_t)dststride, distmap_d_, (size_t)w_ * 4, (size_t)w_ * 4, (size_t)h_,
                                         cudaMemcpyDeviceToHost, stream_));
        CUDA_CHECK(cudaEventRecord(last_done_, stream_));
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        for (int k = 0; k < 3; k++) norms[k] = norms_host_[k];
        check_tma_error();
    }

    void compute_device(double* d_norms, float* d_distmap, int64_t dststride, const uint8_t* const d1[3],
                        const uint8_t* const d2[3], const int64_t ls1[3], const int64_t ls2[3], cudaStream_t stream) override {
        check_tma_error();
        ColourParams cp[2] = {cp_[0], cp_[1]};
        RawImage raw[2];
        for (int c = 0; c < 2; c++) {
            const uint8_t* const* src = c ? d2 : d1;
            const int64_t* ls = c ? ls2 : ls1;
            for (int p = 0; p < 3; p++) {
                if (src[p] == nullptr) VSHIP_THROW(Vship_BadPointer, "null plane pointer");
                if (ls[p] < geo_[c].pw[p] * geo_[c].bytes) VSHIP_THROW(Vship_BadPointer, "lineSize smaller than one row of samples");
                raw[c].p[p] = src[p];
                raw[c].stride[p] = ls[p];
            }
            if (misaligned_view(raw[c], geo_[c])) cp[c].misaligned = 1;
        }
        if (d_distmap && (dststride % 4 || dststride < (int64_t)w_ * 4))
            VSHIP_THROW(Vship_BadPointer, "distmap stride must be a multiple of 4 bytes and at least width * 4");
        CUDA_CHECK(cudaStreamWaitEvent(stream, last_done_, 0));
        run(raw, cp, stream, d_norms, d_distmap, dststride / 4);  // NULL stream: legacy default stream
        CUDA_CHECK(cudaEventRecord(last_done_, stream));
    }

    bool test_tma_timeout() override {
        if (!lf_tma_[0]) return false;
        tma_test_ = true;
        return true;
    }

    KernelTimer& timer() override { return timer_; }
    int width() const override { return w_; }
    int height() const override { return h_; }

private:
    float* plane(int image, int k) const { return pool_ + ((int64_t)image * 26 + k) * plane_floats_; }

    Planes planes_of(int image, int w, int h, bool half) const {
        Planes P{};
        P.w = w;
        P.h = h;
        for (int c = 0; c < 3; c++) {
            P.lin[c] = plane(image, half ? 3 + c : c);
            P.xyb[c] = plane(image, 6 + c);
            P.lf[c] = plane(image, 9 + c);
            P.d[c] = plane(image, 12 + c);
            P.mf[c] = plane(image, 15 + c);
        }
        for (int c = 0; c < 2; c++) {
            P.hfpre[c] = plane(image, 18 + c);
            P.hf[c] = plane(image, 20 + c);
            P.uhf[c] = plane(image, 22 + c);
        }
        P.p = plane(image, 24);
        P.pb = plane(image, 25);
        P.intensity = intensity_;
        return P;
    }

    float* diffmap(int scale) const { return pool_ + ((int64_t)2 * 26 + scale) * plane_floats_; }

    void ensure_distmap() {
        if (!distmap_d_) distmap_d_ = device_alloc<float>((size_t)w_ * h_, "distortion map");
    }

    // Orders `to` after the work enqueued so far on `from`.
    void after(cudaStream_t to, cudaStream_t from, cudaEvent_t ev) {
        CUDA_CHECK(cudaEventRecord(ev, from));
        CUDA_CHECK(cudaStreamWaitEvent(to, ev, 0));
    }

    // One scale: the per-image kernels of the reference image on `st` and of the distorted
    // image on `aux`, concurrently (they share no planes), then the diff map on `st` once both
    // are done.  The caller has ordered `aux` after the inputs of this scale.
    void scale_pass(int w, int h, bool half, float* out, cudaStream_t st, cudaStream_t aux) {
        const dim3 grid((unsigned)ceil_div(w, kTile), (unsigned)ceil_div(h, kTile));
        Planes P[2] = {planes_of(0, w, h, half), planes_of(1, w, h, half)};
        for (int im = 0; im < 2; im++) {
            const cudaStream_t si = im ? aux : st;
            int t = timer_.begin(0, "butter_opsin", si);
            opsin_kernel<<<grid, 256, 0, si>>>(P[im]);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, si);
            t = timer_.begin(1, "butter_lf", si);
            lf_row_kernel<<<dim3((unsigned)ceil_div(w, kLfHW), (unsigned)ceil_div(h, 32), 3u), 256, 0, si>>>(P[im]);
            CUDA_CHECK(cudaGetLastError());
            const dim3 cgrid((unsigned)ceil_div(w, kTile), (unsigned)ceil_div(h, kLfVRows));
            if (lf_tma_[half ? 1 : 0])
                lf_col_tma_kernel<<<cgrid, 256, 0, si>>>(P[im], lf_maps_[im][half ? 1 : 0], tma_err_dev_,
                                                         tma_test_ && im == 0 && !half);
            else
                lf_col_kernel<<<cgrid, 256, 0, si>>>(P[im]);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, si);
            t = timer_.begin(2, "butter_mf", si);
            mf_kernel<<<grid, 256, 0, si>>>(P[im]);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, si);
            t = timer_.begin(3, "butter_hf", si);
            hf_kernel<<<grid, 256, 0, si>>>(P[im]);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, si);
            t = timer_.begin(4, "butter_mask", si);
            mask_kernel<<<grid, 256, 0, si>>>(P[im]);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, si);
        }
        after(st, aux, join_);
        DiffArgs d{};
        d.w = w;
        d.h = h;
        for (int im = 0; im < 2; im++) {
            const float** f = im ? d.f1 : d.f0;
            f[0] = P[im].uhf[1]; f[1] = P[im].uhf[0];
            f[2] = P[im].hf[1]; f[3] = P[im].hf[0];
            f[4] = P[im].mf[1]; f[5] = P[im].mf[0];
            for (int c = 0; c < 2; c++) d.hf[im][c] = P[im].hf[c];
            for (int c = 0; c < 3; c++) { d.mf[im][c] = P[im].mf[c]; d.lf[im][c] = P[im].lf[c]; }
            d.pb[im] = P[im].pb;
        }
        d.out = out;
        const int t = timer_.begin(5, "butter_diffmap", st);
        diffmap_kernel<<<grid, 256, 0, st>>>(d);
        CUDA_CHECK(cudaGetLastError());
        timer_.end(t, st);
    }

    void run(const RawImage raw[2], const ColourParams cp[2], cudaStream_t st, double* norms_d, float* distmap, int64_t dst_pitch) {
        const int64_t n0 = (int64_t)w_ * h_;
        // The two images' colour conversion, downsampling and per-image kernels run on two
        // streams (image 0 on st, image 1 on the second stream) and meet before each diff
        // map.  With per-kernel timing on, both run on st, so each timed stage runs alone.
        const cudaStream_t aux = timer_.enabled ? st : aux_;
        after(aux, st, fork_);
        for (int c = 0; c < 2; c++) {
            const cudaStream_t si = c ? aux : st;
            float* lin = plane(c, 0);
            if (!generic_) {
                launch_ingest_linear(raw[c], cp[c], lin, plane_floats_, si);
            } else {
                lin_generic_[c].run(raw[c], cp[c], geo_[c], si);
                const float* win = lin_generic_[c].planes + (int64_t)geo_[c].crop_top * geo_[c].TW + geo_[c].crop_left;
                copy_window_kernel<<<(unsigned)ceil_div(n0, 256), 256, 0, si>>>(win, geo_[c].TW, geo_[c].TW * geo_[c].TH,
                                                                                 lin, plane_floats_, w_, h_);
                CUDA_CHECK(cudaGetLastError());
            }
        }
        const int w1 = (w_ - 1) / 2 + 1, h1 = (h_ - 1) / 2 + 1;
        for (int c = 0; c < 2; c++)
            for (int k = 0; k < 3; k++) {
                const dim3 g((unsigned)ceil_div(w1, 16), (unsigned)ceil_div(h1, 16));
                downsample_kernel<<<g, dim3(16, 16), 0, c ? aux : st>>>(plane(c, k), plane(c, 3 + k), w_, h_);
                CUDA_CHECK(cudaGetLastError());
            }
        scale_pass(w_, h_, false, diffmap(0), st, aux);
        // The half scale reuses the full scale's band planes, which the full-scale diff map reads.
        after(aux, st, fork_);
        scale_pass(w1, h1, true, diffmap(1), st, aux);
        tma_test_ = false;  // the test hook covers one call
        const int t = timer_.begin(6, "butter_norms", st);
        combine_norms_kernel<<<nblocks_, 256, 0, st>>>(diffmap(0), diffmap(1), w_, h_, w1, qnorm_, distmap, dst_pitch, partials_);
        CUDA_CHECK(cudaGetLastError());
        norms_final_kernel<<<1, 256, 0, st>>>(partials_, nblocks_, n0, qnorm_, norms_d);
        CUDA_CHECK(cudaGetLastError());
        timer_.end(t, st);
    }

    void release() {
        if (stream_) (void)cudaStreamSynchronize(stream_);
        timer_.destroy();
        for (int c = 0; c < 2; c++) {
            staging_[c].free();
            lin_generic_[c].free();
        }
        device_free(pool_);
        device_free(partials_);
        device_free(norms_d_);
        device_free(distmap_d_);
        pinned_free(norms_host_);
        if (tma_err_host_) (void)cudaFreeHost(tma_err_host_);
        tma_err_host_ = tma_err_dev_ = nullptr;
        pool_ = nullptr; partials_ = nullptr; norms_d_ = nullptr; distmap_d_ = nullptr; norms_host_ = nullptr;
        if (last_done_) {
            (void)cudaEventDestroy(last_done_);
            last_done_ = nullptr;
        }
        if (fork_) (void)cudaEventDestroy(fork_);
        if (join_) (void)cudaEventDestroy(join_);
        fork_ = join_ = nullptr;
        if (aux_) {
            (void)cudaStreamSynchronize(aux_);
            (void)cudaStreamDestroy(aux_);
            aux_ = nullptr;
        }
        if (stream_) {
            (void)cudaStreamDestroy(stream_);
            stream_ = nullptr;
        }
    }

    int device_ = 0;
    Vship_Colorspace_t cs_[2];
    ClipGeometry geo_[2];
    ColourParams cp_[2];
    bool generic_ = false;
    int w_ = 0, h_ = 0, qnorm_ = 2;
    float intensity_ = 203.f;
    cudaStream_t stream_ = nullptr;
    StagingBuffer staging_[2];
    GenericLinear lin_generic_[2];
    int64_t plane_floats_ = 0;
    float* pool_ = nullptr;
    int nblocks_ = 0;
    double* partials_ = nullptr;
    double* norms_d_ = nullptr;
    double* norms_host_ = nullptr;
    float* distmap_d_ = nullptr;
    cudaEvent_t last_done_ = nullptr;  // completion of the previous call, on whichever stream it ran
    cudaStream_t aux_ = nullptr;       // second stream: the distorted image's per-image kernels
    LfColMaps lf_maps_[2][2] = {};     // [image][scale]: tensor maps of the mf planes
    bool lf_tma_[2] = {false, false};  // [scale]: the tensor-map column pass applies
    int* tma_err_host_ = nullptr;      // mapped pinned error word of that pass
    int* tma_err_dev_ = nullptr;
    bool tma_test_ = false;            // the test hook's next call
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    KernelTimer timer_;
};

}  // namespace butter

ButterApi* make_butter_engine() { return new butter::Engine(); }

}  // namespace vship

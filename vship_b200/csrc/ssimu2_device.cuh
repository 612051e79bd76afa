// Device code shared by the SSIMULACRA2 engines (per-handler launches in ssimu2.cu, uneven
// batches in ssimu2_batch.cu): pyramid geometry, the front tile (raw planes -> linear RGB ->
// 6-level pyramid -> positive XYB) and the map tile (blur, maps, per-tile sums).
// Included by exactly those translation units; constants are per translation unit.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cmath>

#include "common.cuh"
#include "colour.cuh"
#include "metric_tables.h"

namespace vship {
namespace ssimu2 {

constexpr int kScales = 6;

// Pyramid of one image: level sizes and the float offset of each stored XYB plane.
struct Pyramid {
    int w[kScales], h[kScales], pitch[kScales];
    int64_t off[kScales][3];  // -1 when no map reads the plane
    int64_t image_floats;
};

inline bool map_on(int plane, int scale, int map) {
    return kSsimu2Weights[plane * 36 + scale * 6 + map] > VSHIP_SSIMU2_PRUNE ||
           kSsimu2Weights[plane * 36 + scale * 6 + 3 + map] > VSHIP_SSIMU2_PRUNE;
}

inline bool plane_needed(int plane, int scale) {
    return map_on(plane, scale, 0) || map_on(plane, scale, 1) || map_on(plane, scale, 2);
}

// 17-tap Gaussian, sigma 1.5, and its prefix sums (src/ssimu2/gaussianblur.hpp:7-18).
// The normalisation constant cancels in the per-pixel renormalisation.
static __constant__ float c_gauss[17];
static __constant__ float c_gauss_prefix[18];
static __constant__ double c_weights[108] = {VSHIP_SSIMU2_WEIGHT_LIST};

// Cube root of max(x, 0) without a division: the inverse cube root r = exp2(-log2(x) / 3)
// on the special-function unit, one Newton step for it, r <- r (4 - x r^3) / 3, then
// x r^2.  Two special-function operations instead of three (the reciprocal of a Newton step
// on the cube root itself); ~2 ulp of error.
__device__ __forceinline__ float fast_cbrt(float x) {
    if (!(x > 0.f)) return 0.f;
    float r = ex2_approx(__log2f(x) * (-1.0f / 3.0f));
    const float r3x = x * r * r * r;
    r = r * (4.0f - r3x) * (1.0f / 3.0f);
    return x * r * r;
}

// fast_cbrt(x) + add for two values, with the multiplies and adds in packed FP32x2 (one issue
// slot per pair).  4 - x r^3 and x r^2 + add are single fused operations, as the compiler
// contracts them in the scalar form (fast_cbrt inlined into positive_xyb).
__device__ __forceinline__ float2 fast_cbrt2_add(float2 x, float add) {
    const float2 e = __fmul2_rn(make_float2(__log2f(x.x), __log2f(x.y)), make_float2(-1.0f / 3.0f, -1.0f / 3.0f));
    float2 r = make_float2(ex2_approx(e.x), ex2_approx(e.y));
    const float2 xrr = __fmul2_rn(__fmul2_rn(x, r), r);
    const float2 t = __ffma2_rn(make_float2(-xrr.x, -xrr.y), r, make_float2(4.0f, 4.0f));
    r = __fmul2_rn(__fmul2_rn(r, t), make_float2(1.0f / 3.0f, 1.0f / 3.0f));
    const float2 y = __ffma2_rn(__fmul2_rn(x, r), r, make_float2(add, add));
    return make_float2(x.x > 0.f ? y.x : add, x.y > 0.f ? y.y : add);
}

// positive XYB of a linear RGB triple (src/ssimu2/makeXYB.hpp:6-47).
__device__ __forceinline__ float3 positive_xyb(float3 a) {
    const float bias = 0.0037930734f;
    float l = fmaf(0.30f, a.x, fmaf(0.622f, a.y, fmaf(0.078f, a.z, bias)));
    float m = fmaf(0.23f, a.x, fmaf(0.692f, a.y, fmaf(0.078f, a.z, bias)));
    float s = fmaf(0.24342269f, a.x, fmaf(0.20476745f, a.y, fmaf(0.55180986f, a.z, bias)));
    const float absb = -0.1559542025327239f;
    const float2 lm = fast_cbrt2_add(make_float2(l, m), absb);
    l = lm.x;
    m = lm.y;
    s = fast_cbrt(s) + absb;
    const float X = 0.5f * (l - m);
    const float Y = X + m;
    // make_positive_xyb (makeXYB.hpp:32-36); the reference adds the offsets in double,
    // here in float (the stored value differs by at most one rounding).
    float3 r;
    r.z = (s - Y) + 0.55f;
    r.x = fmaf(X, 14.0f, 0.42f);
    r.y = Y + 0.01f;
    return r;
}

// Shared-memory tile of one pyramid level: 3 channels of T x T (+1 pad column).
template <int T>
struct LevelTile {
    float v[3][T][T + 1];
};

// Builds level L (tile size T) of tile (tx, ty) from level L-1 held in `src` (tile size 2T),
// writes its XYB planes, keeps its linear RGB in `dst`.  Downsample order and clamps follow
// src/ssimu2/downsample.hpp:3-19.
template <int T, bool kXyb = true>
__device__ __forceinline__ void build_level(const LevelTile<2 * T>& src, LevelTile<T>& dst, int L,
                                            const Pyramid& pyr, float* img_out, int tx, int ty) {
    const int W = pyr.w[L], H = pyr.h[L], Wp = pyr.w[L - 1], Hp = pyr.h[L - 1];
    const int ox = tx * T, oy = ty * T;
    for (int i = threadIdx.x; i < T * T; i += blockDim.x) {
        const int lx = i % T, ly = i / T;
        const int gx = ox + lx, gy = oy + ly;
        if (gx >= W || gy >= H) continue;
        const int x0 = 2 * gx - 2 * ox, y0 = 2 * gy - 2 * oy;
        const int x1 = min(2 * gx + 1, Wp - 1) - 2 * ox, y1 = min(2 * gy + 1, Hp - 1) - 2 * oy;
        float3 d;
        float* dp = &d.x;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float t = src.v[c][y0][x0];
            t += src.v[c][y1][x0];
            t += src.v[c][y0][x1];
            t += src.v[c][y1][x1];
            t *= 0.25f;
            dp[c] = t;
            dst.v[c][ly][lx] = t;
        }
        if (kXyb) {
            const float3 q = positive_xyb(d);
            const float qv[3] = {q.x, q.y, q.z};
#pragma unroll
            for (int p = 0; p < 3; p++)
                if (pyr.off[L][p] >= 0) img_out[pyr.off[L][p] + (int64_t)gy * pyr.pitch[L] + gx] = qv[p];
        }
    }
}

// Shared memory of one front tile: linear RGB of levels 1-5.
struct FrontSmem {
    LevelTile<32> t1;
    LevelTile<16> t2;
    LevelTile<8> t3;
    LevelTile<4> t4;
    LevelTile<2> t5;
};

// Linear planar input of the resize/crop path.
struct LinearIn {
    const float* p;       // first plane at the crop origin
    int64_t plane;        // floats between planes
    int64_t pitch;        // row pitch
};

// One front tile: level-0 pixels [64 tx, 64 tx + 64) x [64 ty, 64 ty + 64) of one image to
// linear RGB, levels 1-5 of the tile in shared memory, and every stored XYB plane of the
// tile written to `out` (the image's pyramid).  `stage_mem` holds the chroma stage when the
// clip is subsampled.  kCoarse computes XYB at levels 3 and 4 only (the inputs of the
// learned surrogate).  Ends after the last level is written (no trailing barrier).
template <bool FromLinear, int kFast, bool kCoarse = false>
__device__ __forceinline__ void front_tile(FrontSmem& fs, float* stage_mem, const ColourParams& cp,
                                           const RawImage& im, const LinearIn& lin, const Pyramid& pyr,
                                           float* out, int tx, int ty) {
    const int W0 = pyr.w[0], H0 = pyr.h[0], W1 = pyr.w[1], H1 = pyr.h[1];
    const int pitch0 = pyr.pitch[0];
    float* y0plane = out + pyr.off[0][1];
    const int X0t = tx * kStageTile, Y0t = ty * kStageTile;
    ChromaStage st{};
    if (!FromLinear && kFast != kFastRgb8Srgb && (cp.subw || cp.subh))
        chroma_stage<kFast>(im, cp, X0t, Y0t, stage_mem, st);

    auto pixel = [&](int X, int Y) -> float3 {
        if (FromLinear) {
            const float* base = lin.p + (int64_t)Y * lin.pitch + X;
            return make_float3(base[0], base[lin.plane], base[2 * lin.plane]);
        } else if (kFast == kFastGeneric) {
            return ingest_staged(im, cp, st, X, Y, X0t, Y0t);
        } else {
            return ingest_fast<kFast>(im, cp, st, X, Y, X0t, Y0t);
        }
    };

    // Level 0 -> level 1: one 2x2 quad of level 0 per work item.
    for (int q = threadIdx.x; q < 32 * 32; q += blockDim.x) {
        const int qx = q & 31, qy = q >> 5;
        const int gx = tx * 32 + qx, gy = ty * 32 + qy;
        if (gx >= W1 || gy >= H1) continue;
        const int X0 = 2 * gx, Y0 = 2 * gy;
        const int X1 = min(X0 + 1, W0 - 1), Y1 = min(Y0 + 1, H0 - 1);
        float3 p00, p01, p10, p11;
        if constexpr (!FromLinear && kFast == kFastYuv420Bt709) {
            float3 q4[4];
            ingest_quad_yuv420(im, cp, st, X0, Y0, X0t, Y0t, X1 != X0, Y1 != Y0, q4);
            p00 = q4[0];
            p01 = (X1 != X0) ? q4[1] : p00;
            p10 = (Y1 != Y0) ? q4[2] : p00;
            p11 = (Y1 != Y0) ? ((X1 != X0) ? q4[3] : p10) : p01;
        } else {
            p00 = pixel(X0, Y0);
            p01 = (X1 != X0) ? pixel(X1, Y0) : p00;
            p10 = (Y1 != Y0) ? pixel(X0, Y1) : p00;
            p11 = (Y1 != Y0) ? ((X1 != X0) ? pixel(X1, Y1) : p10) : p01;
        }
        // Level-0 XYB: only the Y plane has unpruned maps at full resolution.
        if (!kCoarse) {
        const float y00 = positive_xyb(p00).y;
        if (X1 != X0) {
            *reinterpret_cast<float2*>(y0plane + (int64_t)Y0 * pitch0 + X0) = make_float2(y00, positive_xyb(p01).y);
            if (Y1 != Y0)
                *reinterpret_cast<float2*>(y0plane + (int64_t)Y1 * pitch0 + X0) =
                    make_float2(positive_xyb(p10).y, positive_xyb(p11).y);
        } else {
            y0plane[(int64_t)Y0 * pitch0 + X0] = y00;
            if (Y1 != Y0) y0plane[(int64_t)Y1 * pitch0 + X0] = positive_xyb(p10).y;
        }
        }
        float3 d;
        d.x = p00.x; d.x += p10.x; d.x += p01.x; d.x += p11.x; d.x *= 0.25f;
        d.y = p00.y; d.y += p10.y; d.y += p01.y; d.y += p11.y; d.y *= 0.25f;
        d.z = p00.z; d.z += p10.z; d.z += p01.z; d.z += p11.z; d.z *= 0.25f;
        fs.t1.v[0][qy][qx] = d.x;
        fs.t1.v[1][qy][qx] = d.y;
        fs.t1.v[2][qy][qx] = d.z;
        if (!kCoarse) {
            const float3 x1 = positive_xyb(d);
            const float xv[3] = {x1.x, x1.y, x1.z};
#pragma unroll
            for (int p = 0; p < 3; p++)
                if (pyr.off[1][p] >= 0) out[pyr.off[1][p] + (int64_t)gy * pyr.pitch[1] + gx] = xv[p];
        }
    }
    __syncthreads();
    build_level<16, !kCoarse>(fs.t1, fs.t2, 2, pyr, out, tx, ty);
    __syncthreads();
    build_level<8>(fs.t2, fs.t3, 3, pyr, out, tx, ty);
    __syncthreads();
    build_level<4>(fs.t3, fs.t4, 4, pyr, out, tx, ty);
    if (!kCoarse) {
        __syncthreads();
        build_level<2>(fs.t4, fs.t5, 5, pyr, out, tx, ty);
    }
}

constexpr int kTile = 32;
constexpr int kHalo = 8;
constexpr int kIn = kTile + 2 * kHalo;  // 48

__device__ __forceinline__ float blur_norm(int pos, int n) {
    // Sum of the taps of a 17-tap window centred on pos that fall inside [0, n).
    const int beg = max(0, kHalo - pos);
    const int end = min(17, n + kHalo - pos);
    return c_gauss_prefix[end] - c_gauss_prefix[beg];
}

constexpr int kMapThreads = 128;

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

// Packed FP32x2 multiply-add of sm_100: one issue slot for two independent FMAs.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

struct TileRef {
    const float* a;
    const float* b;
    int w, h, pitch, X0, Y0;
};

// Geometry of a map tile of 32 columns x TH rows scored by 128 threads: the halo is
// (TH + 16) x 48, the vertical pass gives each thread RPT consecutive rows of one column in
// each of SUB sub-passes.
template <int TH>
struct MapTile {
    static_assert(TH == 16 || TH == 32 || TH == 64, "tile heights 16, 32, 64");
    static constexpr int kRows = TH + 2 * kHalo;
    static constexpr int kHaloPerThread = kRows * kIn / kMapThreads;
    static constexpr int kRPT = TH / 4 < 8 ? TH / 4 : 8;
    static constexpr int kSub = TH / (4 * kRPT);
    static_assert(kRows * kIn % kMapThreads == 0, "halo tile must split evenly over the threads");
    static_assert(kHaloPerThread <= 32, "in-image mask is 32 bits");
    // Moment inputs are kept as float2 pairs so one 64-bit shared access and one packed FMA
    // serve two quantities: (a-k, b-k) and ((a-k)(b-k), (a-b)^2).
    struct Smem {
        float2 sab[kRows][kIn + 1];
        float2 hab[kRows][kTile + 1];
        float2 hpq[kRows][kTile + 1];
        double red[kMapThreads / 32][6];
        float invx[kTile];    // 1 / in-plane tap weight of each output column of the tile
        float invy[TH];       // ... and of each output row
        float shift;          // the shift constant, when it is exchanged through shared memory
    };
    struct Regs {
        float a[kHaloPerThread], b[kHaloPerThread];
        float ka, kb;         // both images at the tile's first output pixel (kRegHeadroom)
        unsigned inmask;
    };
};

// Issues the loads of a tile's halo of both images into registers (element
// i = tid + 128 * it of the row-major halo); out-of-image elements read as 0.  Coherent
// loads (L2 only) are for planes written earlier in the same launch.
// kRegHeadroom is for kernels below their register limit.  There every thread also reads the
// tile's first output pixel: it is always inside the plane, and a warp makes one access.
// stage_halo<TH, true> then needs no shared-memory exchange of the shift constant, which
// saves a barrier per tile.  The bounds test takes one unsigned comparison per axis.  Both
// cost live registers.  The per-handler kernel gained 2.8% from them; the batch kernel, at
// its 128-register limit, lost 5%, so it keeps the plain forms.
template <int TH, bool kCoherent, bool kRegHeadroom>
__device__ __forceinline__ void load_halo(const TileRef& t, typename MapTile<TH>::Regs& r) {
    if (kRegHeadroom) {
        const int64_t o0 = (int64_t)t.Y0 * t.pitch + t.X0;
        r.ka = kCoherent ? __ldcg(t.a + o0) : __ldg(t.a + o0);
        r.kb = kCoherent ? __ldcg(t.b + o0) : __ldg(t.b + o0);
    }
    r.inmask = 0;
#pragma unroll
    for (int it = 0; it < MapTile<TH>::kHaloPerThread; it++) {
        const int i = threadIdx.x + it * kMapThreads;
        const int row = i / kIn, c = i - row * kIn;
        const int gx = t.X0 - kHalo + c, gy = t.Y0 - kHalo + row;
        const bool in = kRegHeadroom ? (unsigned)gx < (unsigned)t.w && (unsigned)gy < (unsigned)t.h
                                     : gx >= 0 && gx < t.w && gy >= 0 && gy < t.h;
        const int64_t o = in ? (int64_t)gy * t.pitch + gx : 0;
        if (kCoherent) {
            r.a[it] = in ? __ldcg(t.a + o) : 0.f;
            r.b[it] = in ? __ldcg(t.b + o) : 0.f;
        } else {
            r.a[it] = in ? __ldg(t.a + o) : 0.f;
            r.b[it] = in ? __ldg(t.b + o) : 0.f;
        }
        r.inmask |= (in ? 1u : 0u) << it;
    }
}

// Moves a loaded halo into shared memory, shifted by the tile constant k, and tabulates the
// renormalisation of the tile's output columns and rows (tile origin X0, Y0 in a w x h
// plane; positions past the plane, whose outputs are never used, take the last in-plane
// one).  Ends with a barrier, after which the registers are free for the next tile's loads.
template <int TH, bool kRegHeadroom>
__device__ __forceinline__ void stage_halo(typename MapTile<TH>::Smem& sm, const typename MapTile<TH>::Regs& r,
                                           int X0, int Y0, int w, int h) {
    const int tid = threadIdx.x;
    static_assert(kTile + TH <= kMapThreads, "one renormalisation entry per thread");
    if (tid < kTile)
        sm.invx[tid] = 1.0f / blur_norm(min(X0 + tid, w - 1), w);
    else if (tid < kTile + TH)
        sm.invy[tid - kTile] = 1.0f / blur_norm(min(Y0 + tid - kTile, h - 1), h);
    // Shift constant k: the mean of both images at the tile's first output pixel (always
    // inside the image): loaded by every thread with the halo (kRegHeadroom), or halo element
    // (8, 8), which thread 8 holds as its 4th element, passed through shared memory.
    // The renormalised blur maps constants to themselves, so moments of a-k, b-k give the
    // reference's blur(ab) - blur(a)blur(b) etc. in exact arithmetic, while in FP32 they
    // no longer cancel ~0.25-sized terms down to the ~1e-5 local covariances of smooth
    // regions.  k is symmetric in the two images, so identical inputs still give
    // bit-identical moments.
    float k;
    if (kRegHeadroom) {
        k = 0.5f * (r.ka + r.kb);
    } else {
        static_assert(kHalo * kIn + kHalo == 8 + 3 * kMapThreads, "shift element owner");
        if (tid == 8) sm.shift = 0.5f * (r.a[3] + r.b[3]);
        __syncthreads();
        k = sm.shift;
    }
    // Shifted halo; zero outside the plane, as the reference's zero padding
    // (src/ssimu2/gaussianblur.hpp:24-36): out-of-image taps add nothing and the
    // renormalisation divides by the in-image tap weights only.
#pragma unroll
    for (int it = 0; it < MapTile<TH>::kHaloPerThread; it++) {
        const int i = tid + it * kMapThreads;
        const int row = i / kIn, c = i - row * kIn;
        const bool in = (r.inmask >> it) & 1u;
        sm.sab[row][c] = in ? f2(r.a[it] - k, r.b[it] - k) : f2(0.f, 0.f);
    }
    __syncthreads();
}

// Halo of a 32 x 32 map tile read with 128-bit loads (per-handler and no-allocation maps
// kernels).  The halo is 48 rows of 12 float4 per image: halo column 0 is X0 - 8, a multiple
// of 8, and plane rows are padded to a multiple of 8 floats, so every float4 starts on a
// 16-byte boundary and a float4 that starts inside a row ends inside the row's padding.  A
// float4 that starts left of the plane or in a row outside it is not read; elements at or
// past the plane width are zeroed at staging (the padding holds no pixel).  Thread t holds
// positions t + 128 i (i < 5; the fifth only for t < 64) of both images: 10 loads per tile
// instead of 36 scalar ones.  The batch kernel, at its register limit, keeps load_halo.
struct HaloV4 {
    static constexpr int kRows = kTile + 2 * kHalo;
    static constexpr int kVec = kIn / 4;
    static constexpr int kPos = kRows * kVec;
    static constexpr int kSlots = (kPos + kMapThreads - 1) / kMapThreads;
    float4 a[kSlots], b[kSlots];
    float ka, kb;
    unsigned inmask;
};

__device__ __forceinline__ void load_halo_v4(const TileRef& t, HaloV4& r) {
    const int64_t o0 = (int64_t)t.Y0 * t.pitch + t.X0;
    r.ka = __ldg(t.a + o0);
    r.kb = __ldg(t.b + o0);
    r.inmask = 0;
#pragma unroll
    for (int it = 0; it < HaloV4::kSlots; it++) {
        const int j = threadIdx.x + it * kMapThreads;
        const int row = j / HaloV4::kVec, c4 = j - row * HaloV4::kVec;
        const int gx = t.X0 - kHalo + 4 * c4, gy = t.Y0 - kHalo + row;
        const bool in = j < HaloV4::kPos && (unsigned)gx < (unsigned)t.w && (unsigned)gy < (unsigned)t.h;
        const int64_t o = in ? (int64_t)gy * t.pitch + gx : 0;
        r.a[it] = in ? __ldg(reinterpret_cast<const float4*>(t.a + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
        r.b[it] = in ? __ldg(reinterpret_cast<const float4*>(t.b + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
        r.inmask |= (in ? 1u : 0u) << it;
    }
}

// stage_halo for a HaloV4: the same shift, renormalisation tables and zero padding.
__device__ __forceinline__ void stage_halo_v4(typename MapTile<kTile>::Smem& sm, const HaloV4& r, int X0, int Y0, int w,
                                              int h) {
    const int tid = threadIdx.x;
    if (tid < kTile)
        sm.invx[tid] = 1.0f / blur_norm(min(X0 + tid, w - 1), w);
    else if (tid < 2 * kTile)
        sm.invy[tid - kTile] = 1.0f / blur_norm(min(Y0 + tid - kTile, h - 1), h);
    const float k = 0.5f * (r.ka + r.kb);
#pragma unroll
    for (int it = 0; it < HaloV4::kSlots; it++) {
        const int j = tid + it * kMapThreads;
        if (j >= HaloV4::kPos) break;
        const int row = j / HaloV4::kVec, c4 = j - row * HaloV4::kVec;
        const int gx = X0 - kHalo + 4 * c4;
        const bool in = (r.inmask >> it) & 1u;
        const float av[4] = {r.a[it].x, r.a[it].y, r.a[it].z, r.a[it].w};
        const float bv[4] = {r.b[it].x, r.b[it].y, r.b[it].z, r.b[it].w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const bool ine = in && gx + e < w;
            sm.sab[row][4 * c4 + e] = ine ? f2(av[e] - k, bv[e] - k) : f2(0.f, 0.f);
        }
    }
    __syncthreads();
}

// The same 128-bit halo loads for the batch maps kernel, for tile heights 16, 32 and 64 and
// with coherent (L2) loads (the pyramids were written earlier in the same graph).  The shift
// constant is exchanged through shared memory: halo element (8, 8), the tile's first output
// pixel, is position 8 * 12 + 2, component x, held by thread 98.  Registers stay within the
// kernel's limit: 8, 10 or 16 float4 per thread.
template <int TH>
struct HaloV4T {
    static constexpr int kRows = TH + 2 * kHalo;
    static constexpr int kVec = kIn / 4;
    static constexpr int kPos = kRows * kVec;
    static constexpr int kSlots = (kPos + kMapThreads - 1) / kMapThreads;
    float4 a[kSlots], b[kSlots];
    unsigned inmask;
};

template <int TH, bool kCoherent>
__device__ __forceinline__ void load_halo_v4t(const TileRef& t, HaloV4T<TH>& r) {
    using H = HaloV4T<TH>;
    r.inmask = 0;
#pragma unroll
    for (int it = 0; it < H::kSlots; it++) {
        const int j = threadIdx.x + it * kMapThreads;
        const int row = j / H::kVec, c4 = j - row * H::kVec;
        const int gx = t.X0 - kHalo + 4 * c4, gy = t.Y0 - kHalo + row;
        const bool in = j < H::kPos && gx >= 0 && gx < t.w && gy >= 0 && gy < t.h;
        const int64_t o = in ? (int64_t)gy * t.pitch + gx : 0;
        if (kCoherent) {
            r.a[it] = in ? __ldcg(reinterpret_cast<const float4*>(t.a + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
            r.b[it] = in ? __ldcg(reinterpret_cast<const float4*>(t.b + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
            r.a[it] = in ? __ldg(reinterpret_cast<const float4*>(t.a + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
            r.b[it] = in ? __ldg(reinterpret_cast<const float4*>(t.b + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        r.inmask |= (in ? 1u : 0u) << it;
    }
}

template <int TH>
__device__ __forceinline__ void stage_halo_v4t(typename MapTile<TH>::Smem& sm, const HaloV4T<TH>& r, int X0, int Y0, int w,
                                               int h) {
    using H = HaloV4T<TH>;
    const int tid = threadIdx.x;
    if (tid < kTile)
        sm.invx[tid] = 1.0f / blur_norm(min(X0 + tid, w - 1), w);
    else if (tid < kTile + TH)
        sm.invy[tid - kTile] = 1.0f / blur_norm(min(Y0 + tid - kTile, h - 1), h);
    // shift constant: halo element (8, 8) is position 8 * 12 + 2, component 0, held by thread 98
    if (tid == kHalo * H::kVec + 2) sm.shift = 0.5f * (r.a[0].x + r.b[0].x);
    __syncthreads();
    const float k = sm.shift;
#pragma unroll
    for (int it = 0; it < H::kSlots; it++) {
        const int j = tid + it * kMapThreads;
        if (j >= H::kPos) break;
        const int row = j / H::kVec, c4 = j - row * H::kVec;
        const int gx = X0 - kHalo + 4 * c4;
        const bool in = (r.inmask >> it) & 1u;
        const float av[4] = {r.a[it].x, r.a[it].y, r.a[it].z, r.a[it].w};
        const float bv[4] = {r.b[it].x, r.b[it].y, r.b[it].z, r.b[it].w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const bool ine = in && gx + e < w;
            sm.sab[row][4 * c4 + e] = ine ? f2(av[e] - k, bv[e] - k) : f2(0.f, 0.f);
        }
    }
    __syncthreads();
}

// Blurs a staged tile and scores it: separable 17-tap blur of the four moment inputs,
// SSIM / artifact / detail-loss maps, and the tile's FP64 sums of x and x^4 of each map,
// written by threads 0-5 to out[0..5].  Ends with the reduction barrier; the caller must
// synchronise again before staging the next tile (the vertical pass reads sab).
template <int TH>
__device__ __forceinline__ void blur_score_tile(typename MapTile<TH>::Smem& sm, int X0, int Y0, int w, int h,
                                                double* out) {
    using MT = MapTile<TH>;
    const int tid = threadIdx.x;
    // Horizontal pass: kRows rows x 32 columns; a work item is four adjacent output columns
    // of one row; consecutive threads take consecutive rows (conflict-free 64-bit access).
    for (int u = tid; u < MT::kRows * (kTile / 4); u += kMapThreads) {
        const int cg = u / MT::kRows, r = u - cg * MT::kRows, c0 = cg * 4;
        float2 ab[20], pq[20];
#pragma unroll
        for (int j = 0; j < 20; j++) {
            ab[j] = sm.sab[r][c0 + j];
            const float d = ab[j].x - ab[j].y;
            pq[j] = f2(ab[j].x * ab[j].y, d * d);
        }
        float2 acc_ab[4], acc_pq[4];
#pragma unroll
        for (int o = 0; o < 4; o++) acc_ab[o] = acc_pq[o] = f2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 17; j++) {
            const float2 g = f2(c_gauss[j], c_gauss[j]);
#pragma unroll
            for (int o = 0; o < 4; o++) {
                acc_ab[o] = fma2(g, ab[j + o], acc_ab[o]);
                acc_pq[o] = fma2(g, pq[j + o], acc_pq[o]);
            }
        }
#pragma unroll
        for (int o = 0; o < 4; o++) {
            const float inv = sm.invx[c0 + o];
            sm.hab[r][c0 + o] = f2(acc_ab[o].x * inv, acc_ab[o].y * inv);
            sm.hpq[r][c0 + o] = f2(acc_pq[o].x * inv, acc_pq[o].y * inv);
        }
    }
    __syncthreads();

    // Vertical pass: each thread kRPT consecutive output rows of one column per sub-pass.
    constexpr int RPT = MT::kRPT;
    const int c = tid & 31;
    const int gx = X0 + c;
    double dsum[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int sub = 0; sub < MT::kSub; sub++) {
        const int r0 = sub * 4 * RPT + (tid >> 5) * RPT;
        float2 mab[RPT], mpq[RPT];
        {
            float2 col[RPT + 16];
#pragma unroll
            for (int j = 0; j < RPT + 16; j++) col[j] = sm.hab[r0 + j][c];
#pragma unroll
            for (int o = 0; o < RPT; o++) {
                float2 acc = f2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 17; j++) acc = fma2(f2(c_gauss[j], c_gauss[j]), col[o + j], acc);
                mab[o] = acc;
            }
#pragma unroll
            for (int j = 0; j < RPT + 16; j++) col[j] = sm.hpq[r0 + j][c];
#pragma unroll
            for (int o = 0; o < RPT; o++) {
                float2 acc = f2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 17; j++) acc = fma2(f2(c_gauss[j], c_gauss[j]), col[o + j], acc);
                mpq[o] = acc;
            }
        }
        float sum[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int o = 0; o < RPT; o++) {
            const int gy = Y0 + r0 + o;
            if (gx >= w || gy >= h) continue;
            const float inv = sm.invy[r0 + o];
            // Shifted means m1 = mu1 - k, m2 = mu2 - k, s12 = blur((a-k)(b-k)), D = blur((a-b)^2).
            const float m1 = mab[o].x * inv, m2 = mab[o].y * inv, s12 = mpq[o].x * inv, D = mpq[o].y * inv;
            // SSIM map of the reference (src/ssimu2/score.hpp:266-274),
            //   ssim = 1 - (1 - md^2) * N / (s1^2 + s2^2 + C),  N = 2 s12' + C,  md = mu1 - mu2,
            // rewritten without cancellation: with V = D - md^2 (the local variance of a - b),
            // s1^2 + s2^2 + C = V + N and therefore ssim = (V + md^2 N) / (V + N).  Identical
            // inputs give V = md = 0 and an SSIM of exactly 0.
            const float md = m1 - m2;
            const float md2 = md * md;
            const float N = fmaf(2.0f, s12 - m1 * m2, 0.0009f);
            const float V = D - md2;
            // V + N = s1^2 + s2^2 + C >= C > 0: the fast division (2 ulp) is safe here.
            const float ssim = fmaxf(__fdividef(fmaf(md2, N, V), V + N), 0.0f);
            // Artifact and detail-loss maps (score.hpp:276-281): (|b-mu2|+1)/(|a-mu1|+1) - 1,
            // evaluated as (|b-mu2| - |a-mu1|) / (|a-mu1| + 1) to avoid cancelling against 1.
            const float2 cv = sm.sab[r0 + o + kHalo][c + kHalo];
            const float ea = fabsf(cv.x - m1), eb = fabsf(cv.y - m2);
            const float v1 = __fdividef(eb - ea, ea + 1.0f);
            const float art = fmaxf(v1, 0.0f), det = fmaxf(-v1, 0.0f);
            const float s2 = ssim * ssim, a2 = art * art, d2 = det * det;
            sum[0] += ssim; sum[1] += art; sum[2] += det;
            sum[3] += s2 * s2; sum[4] += a2 * a2; sum[5] += d2 * d2;
        }
#pragma unroll
        for (int q = 0; q < 6; q++) dsum[q] += (double)sum[q];
    }
    // FP64 tree reduction of the tile.
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double v = dsum[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        dsum[q] = v;
    }
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 6; q++) sm.red[warp][q] = dsum[q];
    }
    __syncthreads();
    if (tid < 6) {
        double v = 0.0;
#pragma unroll
        for (int wi = 0; wi < kMapThreads / 32; wi++) v += sm.red[wi][tid];
        out[tid] = v;
    }
}

// The score of 108 features exactly as final_score computes it (src/ssimu2/score.hpp:442-460:
// float fmaf accumulation, float result).
__device__ __forceinline__ double score_from_features(const float* feat) {
    double s = 0.0;
    for (int i = 0; i < 108; i++) s = (double)fmaf((float)c_weights[i], feat[i], (float)s);
    s *= VSHIP_SSIMU2_SCALE;
    s = (VSHIP_SSIMU2_C3 * s * s) * s + VSHIP_SSIMU2_C1 * s - VSHIP_SSIMU2_C2 * s * s;
    s = s > 0.0 ? pow(s, VSHIP_SSIMU2_EXP) * -10.0 + 100.0 : 100.0;
    return (double)(float)s;
}

static void upload_gauss_constants() {
    float g[17], pre[18];
    pre[0] = 0.f;
    for (int i = 0; i < 17; i++) {
        g[i] = (float)std::exp(-(double)((8 - i) * (8 - i)) / (2.0 * 1.5 * 1.5));
        pre[i + 1] = pre[i] + g[i];
    }
    CUDA_CHECK(cudaMemcpyToSymbol(c_gauss, g, sizeof(g)));
    CUDA_CHECK(cudaMemcpyToSymbol(c_gauss_prefix, pre, sizeof(pre)));
}

// Level sizes of a width x height image and the offsets of the planes some map reads
// (level 0 keeps its Y plane, which the front tile writes unconditionally).
inline Pyramid make_pyramid(int width, int height) {
    Pyramid pyr{};
    int w = width, h = height;
    int64_t off = 0;
    for (int s = 0; s < kScales; s++) {
        pyr.w[s] = w;
        pyr.h[s] = h;
        pyr.pitch[s] = (int)round_up(w, 8);
        for (int p = 0; p < 3; p++) {
            const bool keep = plane_needed(p, s) || (s == 0 && p == 1);
            if (keep) {
                pyr.off[s][p] = off;
                off += round_up((int64_t)pyr.pitch[s] * h, 64);
            } else {
                pyr.off[s][p] = -1;
            }
        }
        w = (w - 1) / 2 + 1;
        h = (h - 1) / 2 + 1;
    }
    pyr.image_floats = round_up(off, 64);
    return pyr;
}

}  // namespace ssimu2
}  // namespace vship

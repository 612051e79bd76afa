// Learned SSIMULACRA2 surrogate for target-quality search.  No counterpart in the reference.
//
// A small convolutional network predicts a pair's SSIMULACRA2 score from the 1/8 and 1/16
// XYB pyramid levels of both images, which cost a fraction of the exact metric: the front
// tile in its coarse mode converts every pixel to linear RGB and averages, but computes XYB
// at levels 3 and 4 only, and no map is blurred.  A search consults the prediction first and
// calls the exact metric when the prediction lands within a margin of its threshold.
//
// Network (one set of weights applied to both levels):
//   input  6 channels: reference XYB (a) and distorted - reference (b - a), normalised per
//          channel with constants measured on the training set
//   conv1  3x3, 6 -> 16, ReLU        conv2  3x3, 16 -> 16, ReLU        conv3  1x1, 16 -> 8, ReLU
//   pool   per channel and level: mean of x and (mean of x^4 + 1e-8)^(1/4)   (32 features)
//   head   linear 32 -> 1; score = 70 + 20 * output
// Weights are FP16 on the device for the forward and backward kernels (FP32 accumulation);
// the optimiser keeps FP32 masters (Adam).  Training, inference and gradients run on the
// kernels of this file; the FP64 oracle in oracle/surrogate.py restates the same network.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "common.cuh"
#include "colour.cuh"
#include "frontend.cuh"
#include "metric_tables.h"
#include "ssimu2_device.cuh"
#include "engines.h"

namespace vship {
namespace surrogate {
namespace {

using ssimu2::FrontSmem;
using ssimu2::LinearIn;
using ssimu2::Pyramid;
using ssimu2::front_tile;

constexpr int kCin = 6, kC1 = 16, kC2 = 16, kC3 = 8;
constexpr int kFeat = 2 * 2 * kC3;  // (mean, 4-norm) x 8 channels x 2 levels
constexpr float kScoreShift = 70.f, kScoreScale = 20.f;
constexpr float kPoolEps = 1e-8f;

// Flat parameter vector (FP32 masters): offsets of each tensor.
constexpr int oW1 = 0;
constexpr int ob1 = oW1 + kC1 * kCin * 9;
constexpr int oW2 = ob1 + kC1;
constexpr int ob2 = oW2 + kC2 * kC1 * 9;
constexpr int oW3 = ob2 + kC2;
constexpr int ob3 = oW3 + kC3 * kC2;
constexpr int oWh = ob3 + kC3;
constexpr int obh = oWh + kFeat;
constexpr int kParams = obh + 1;  // 3369

constexpr int kTileSide = 16;      // conv tiles: 16 x 16 pixels, one thread each
constexpr int kConvThreads = 256;
constexpr int kMaxChunk = 64;      // pairs per coarse-front launch

// Geometry of one input level of a pair's input block (FP16, channel-major).
struct Level {
    int h, w;
    int64_t off;  // element offset inside a pair's block
};

// ------------------------------------------------------------------------------------------
// Coarse front: raw planes -> XYB levels 3 and 4 of both images; packing into net inputs
// ------------------------------------------------------------------------------------------

struct CoarseArgs {
    ColourParams cp[2];
    Pyramid pyr;                   // levels 3 and 4 stored, everything else -1
    float* out;                    // image i at out + i * pyr.image_floats
    int clip;                      // -1: images alternate reference / distorted; else every image is this clip
    RawImage raw[2 * kMaxChunk];
};

template <int kFast>
__global__ void __launch_bounds__(256) sg_coarse_front_kernel(const __grid_constant__ CoarseArgs a) {
    __shared__ FrontSmem fs;
    extern __shared__ __align__(16) float stage[];
    const int img = blockIdx.z, clip = a.clip < 0 ? (img & 1) : a.clip;
    const LinearIn lin{};
    front_tile<false, kFast, true>(fs, stage, a.cp[clip], a.raw[img], lin, a.pyr,
                                   a.out + (int64_t)img * a.pyr.image_floats, blockIdx.x, blockIdx.y);
}

// Per pair: [a_X, a_Y, a_B, b_X - a_X, b_Y - a_Y, b_B - a_B] at level 3, then at level 4.
__global__ void sg_pack_kernel(const float* __restrict__ coarse, Pyramid pyr, Level l3, Level l4, int64_t block,
                               __half* __restrict__ inputs) {
    const int pair = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n3 = l3.h * l3.w, n4 = l4.h * l4.w;
    if (i >= n3 + n4) return;
    const int L = i < n3 ? 3 : 4;
    const Level& lv = i < n3 ? l3 : l4;
    const int j = i < n3 ? i : i - n3;
    const int y = j / lv.w, x = j - y * lv.w;
    const float* A = coarse + (int64_t)(2 * pair) * pyr.image_floats;
    const float* B = A + pyr.image_floats;
    __half* out = inputs + (int64_t)pair * block + lv.off;
    const int64_t plane = (int64_t)lv.h * lv.w;
#pragma unroll
    for (int p = 0; p < 3; p++) {
        const int64_t o = pyr.off[L][p] + (int64_t)y * pyr.pitch[L] + x;
        const float va = A[o], vb = B[o];
        out[p * plane + j] = __float2half_rn(va);
        out[(3 + p) * plane + j] = __float2half_rn(vb - va);
    }
}

// Reference levels of one image, dense FP32: [3][h3][w3] then [3][h4][w4].
__global__ void sg_pack_reference_kernel(const float* __restrict__ coarse, Pyramid pyr, Level l3, Level l4,
                                         int64_t ref_floats, float* __restrict__ refs) {
    const int img = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n3 = l3.h * l3.w, n4 = l4.h * l4.w;
    if (i >= n3 + n4) return;
    const int L = i < n3 ? 3 : 4;
    const Level& lv = i < n3 ? l3 : l4;
    const int j = i < n3 ? i : i - n3;
    const int y = j / lv.w, x = j - y * lv.w;
    const float* A = coarse + (int64_t)img * pyr.image_floats;
    float* out = refs + (int64_t)img * ref_floats + (i < n3 ? 0 : 3 * n3);
    const int64_t plane = (int64_t)lv.h * lv.w;
#pragma unroll
    for (int p = 0; p < 3; p++) out[p * plane + j] = A[pyr.off[L][p] + (int64_t)y * pyr.pitch[L] + x];
}

// Network inputs of distorted images against prepared reference levels: the same values
// sg_pack_kernel writes for the pair.
__global__ void sg_pack_against_kernel(const float* __restrict__ coarse, Pyramid pyr, Level l3, Level l4,
                                       const float* __restrict__ refs, int64_t ref_floats, int64_t block,
                                       __half* __restrict__ inputs) {
    const int pair = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n3 = l3.h * l3.w, n4 = l4.h * l4.w;
    if (i >= n3 + n4) return;
    const int L = i < n3 ? 3 : 4;
    const Level& lv = i < n3 ? l3 : l4;
    const int j = i < n3 ? i : i - n3;
    const int y = j / lv.w, x = j - y * lv.w;
    const float* A = refs + (int64_t)pair * ref_floats + (i < n3 ? 0 : 3 * n3);
    const float* B = coarse + (int64_t)pair * pyr.image_floats;
    __half* out = inputs + (int64_t)pair * block + lv.off;
    const int64_t plane = (int64_t)lv.h * lv.w;
#pragma unroll
    for (int p = 0; p < 3; p++) {
        const float va = A[p * plane + j], vb = B[pyr.off[L][p] + (int64_t)y * pyr.pitch[L] + x];
        out[p * plane + j] = __float2half_rn(va);
        out[(3 + p) * plane + j] = __float2half_rn(vb - va);
    }
}

// ------------------------------------------------------------------------------------------
// Network kernels.  Activations are FP32 [n][c][h][w]; conv weights FP16 [cout][cin][k][k].
// ------------------------------------------------------------------------------------------

// Forward convolution + bias + ReLU (grid: 32 x 8 output tiles, samples).  With kHalfIn the
// input is the FP16 input block (sample stride `in_stride`), normalised on load as
// (x - shift[c]) * scale[c]; zero padding outside the level.  Register-blocked: each of the
// 64 threads makes 4 adjacent pixels of one row for all COUT channels, so one 128-bit shared
// load of 4 output channels' weights feeds 16 FMAs.  Every output accumulates bias, then
// input channel, then kernel row, then kernel column, one fmaf each, as a one-pixel loop would.
constexpr int kFwdTW = 32, kFwdTH = 8, kFwdThreads = (kFwdTW / 4) * kFwdTH;

// With kPool the layer also writes, per tile and channel, the sums of x and x^4 over the
// tile's pixels (pool[sample][tile][2 * COUT]) for the pooling that follows.
template <int K, int CIN, int COUT, bool kHalfIn, bool kPool = false>
__global__ void __launch_bounds__(kFwdThreads) sg_conv_fwd(const void* __restrict__ in, int64_t in_stride,
                                                           const float* __restrict__ norm, const __half* __restrict__ w,
                                                           const float* __restrict__ b, float* __restrict__ out,
                                                           int H, int W, int tiles_x, float* __restrict__ pool = nullptr) {
    static_assert(COUT % 4 == 0, "weights travel in groups of 4 output channels");
    constexpr int R = K / 2, SH = kFwdTH + K - 1, SW = kFwdTW + K - 1;
    constexpr int SP = (SW + 3) / 4 * 4;  // row pitch: 16-byte aligned rows
    __shared__ __align__(16) float s_in[CIN][SH][SP];
    __shared__ __align__(16) float s_w[CIN][K][K][COUT];
    const int n = blockIdx.y, tid = threadIdx.x;
    const int ty0 = (blockIdx.x / tiles_x) * kFwdTH, tx0 = (blockIdx.x % tiles_x) * kFwdTW;
    for (int i = tid; i < COUT * CIN * K * K; i += kFwdThreads) {  // [cout][cin][ky][kx] -> [cin][ky][kx][cout]
        const int o = i / (CIN * K * K), r = i - o * CIN * K * K;
        (&s_w[0][0][0][0])[r * COUT + o] = __half2float(w[i]);
    }
    const int64_t plane = (int64_t)H * W;
    // Input tile with halo: loads in groups of 16 per thread, all issued before any is stored.
    constexpr int kElems = CIN * SH * SW, kPer = (kElems + kFwdThreads - 1) / kFwdThreads, kGroup = 16;
    for (int base = 0; base < kPer; base += kGroup) {
        float v[kGroup];
#pragma unroll
        for (int j = 0; j < kGroup; j++) {
            const int i = tid + (base + j) * kFwdThreads;
            v[j] = 0.f;
            if (base + j < kPer && i < kElems) {
                const int c = i / (SH * SW), r = i - c * SH * SW, yy = r / SW, xx = r - yy * SW;
                const int gy = ty0 + yy - R, gx = tx0 + xx - R;
                if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
                    const int64_t o = (int64_t)c * plane + (int64_t)gy * W + gx;
                    if (kHalfIn)
                        v[j] = (__half2float(static_cast<const __half*>(in)[n * in_stride + o]) - norm[c]) * norm[CIN + c];
                    else
                        v[j] = __ldg(static_cast<const float*>(in) + n * in_stride + o);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kGroup; j++) {
            const int i = tid + (base + j) * kFwdThreads;
            if (base + j < kPer && i < kElems) {
                const int c = i / (SH * SW), r = i - c * SH * SW, yy = r / SW, xx = r - yy * SW;
                s_in[c][yy][xx] = v[j];
            }
        }
    }
    __syncthreads();
    const int ly = tid / (kFwdTW / 4), lx0 = (tid % (kFwdTW / 4)) * 4;
    const int gy = ty0 + ly, gx0 = tx0 + lx0;
    if (!kPool && (gy >= H || gx0 >= W)) return;  // with kPool every thread reaches the reduction
    float acc[4][COUT];
#pragma unroll
    for (int o = 0; o < COUT; o++) {
        const float bo = b[o];
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q][o] = bo;
    }
    for (int c = 0; c < CIN; c++)
#pragma unroll
        for (int ky = 0; ky < K; ky++) {
            float v[4 + K - 1];
            const float4 v4 = *reinterpret_cast<const float4*>(&s_in[c][ly + ky][lx0]);
            v[0] = v4.x; v[1] = v4.y; v[2] = v4.z; v[3] = v4.w;
#pragma unroll
            for (int e = 4; e < 4 + K - 1; e++) v[e] = s_in[c][ly + ky][lx0 + e];
#pragma unroll
            for (int kx = 0; kx < K; kx++)
#pragma unroll
                for (int o4 = 0; o4 < COUT / 4; o4++) {
                    const float4 wv = *reinterpret_cast<const float4*>(&s_w[c][ky][kx][4 * o4]);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        acc[q][4 * o4 + 0] = fmaf(wv.x, v[q + kx], acc[q][4 * o4 + 0]);
                        acc[q][4 * o4 + 1] = fmaf(wv.y, v[q + kx], acc[q][4 * o4 + 1]);
                        acc[q][4 * o4 + 2] = fmaf(wv.z, v[q + kx], acc[q][4 * o4 + 2]);
                        acc[q][4 * o4 + 3] = fmaf(wv.w, v[q + kx], acc[q][4 * o4 + 3]);
                    }
                }
        }
    const bool row_ok = gy < H;
    float* dst = out + (int64_t)n * COUT * plane + (int64_t)gy * W + gx0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (!row_ok || gx0 + q >= W) break;
#pragma unroll
        for (int o = 0; o < COUT; o++) dst[o * plane + q] = fmaxf(acc[q][o], 0.f);
    }
    if constexpr (kPool) {
        __shared__ float red[kFwdThreads / 32][2 * COUT];
        float s1[COUT], s4[COUT];
#pragma unroll
        for (int o = 0; o < COUT; o++) {
            s1[o] = s4[o] = 0.f;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float x = (row_ok && gx0 + q < W) ? fmaxf(acc[q][o], 0.f) : 0.f, x2 = x * x;
                s1[o] += x;
                s4[o] = fmaf(x2, x2, s4[o]);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                s1[o] += __shfl_xor_sync(0xffffffffu, s1[o], off);
                s4[o] += __shfl_xor_sync(0xffffffffu, s4[o], off);
            }
        }
        if ((tid & 31) == 0)
#pragma unroll
            for (int o = 0; o < COUT; o++) {
                red[tid >> 5][o] = s1[o];
                red[tid >> 5][COUT + o] = s4[o];
            }
        __syncthreads();
        if (tid < 2 * COUT) {
            float v = 0.f;
#pragma unroll
            for (int wi = 0; wi < kFwdThreads / 32; wi++) v += red[wi][tid];
            pool[((int64_t)n * gridDim.x + blockIdx.x) * 2 * COUT + tid] = v;
        }
    }
}

// Per sample: mean and 4-norm of each conv3 channel over the level from the tile sums of the
// last layer (fixed order: deterministic); also keeps mean(x^4) for the backward pass.
__global__ void __launch_bounds__(256) sg_pool_finish(const float* __restrict__ pool, int tiles, int HW,
                                                      float* __restrict__ feat, float* __restrict__ m4, int level) {
    __shared__ float red[8][2 * kC3];
    const int n = blockIdx.x, tid = threadIdx.x;
    const float* part = pool + (int64_t)n * tiles * 2 * kC3;
    float v[2 * kC3];
#pragma unroll
    for (int k = 0; k < 2 * kC3; k++) v[k] = 0.f;
    for (int t = tid; t < tiles; t += 256)
#pragma unroll
        for (int k = 0; k < 2 * kC3; k++) v[k] += part[t * 2 * kC3 + k];
#pragma unroll
    for (int k = 0; k < 2 * kC3; k++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
    if ((tid & 31) == 0)
#pragma unroll
        for (int k = 0; k < 2 * kC3; k++) red[tid >> 5][k] = v[k];
    __syncthreads();
    if (tid < 2 * kC3) {
        float t = 0.f;
        for (int wi = 0; wi < 8; wi++) t += red[wi][tid];
        t /= (float)HW;
        const int c = tid % kC3;
        if (tid < kC3) {
            feat[n * kFeat + level * 2 * kC3 + c] = t;
        } else {
            m4[n * 2 * kC3 + level * kC3 + c] = t;
            feat[n * kFeat + level * 2 * kC3 + kC3 + c] = sqrtf(sqrtf(t + kPoolEps));
        }
    }
}

// Gradient of the input of a conv + ReLU layer: din[c][y][x] = sum over o, taps of
// w[o][c][ky][kx] * g[o][y - ky + R][x - kx + R], with g = dout where out > 0.
template <int K, int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) sg_conv_bwd_data(const float* __restrict__ dout,
                                                                 const float* __restrict__ out,
                                                                 const __half* __restrict__ w, float* __restrict__ din,
                                                                 int H, int W, int tiles_x) {
    constexpr int R = K / 2, S = kTileSide + K - 1;
    __shared__ float s_g[COUT][S][S + 1];
    __shared__ float s_w[COUT * CIN * K * K];
    const int n = blockIdx.y, tid = threadIdx.x;
    const int ty0 = (blockIdx.x / tiles_x) * kTileSide, tx0 = (blockIdx.x % tiles_x) * kTileSide;
    for (int i = tid; i < COUT * CIN * K * K; i += kConvThreads) s_w[i] = __half2float(w[i]);
    const int64_t plane = (int64_t)H * W;
    for (int i = tid; i < COUT * S * S; i += kConvThreads) {
        const int o = i / (S * S), r = i - o * S * S, yy = r / S, xx = r - yy * S;
        const int gy = ty0 + yy - R, gx = tx0 + xx - R;
        float v = 0.f;
        if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
            const int64_t idx = (int64_t)n * COUT * plane + (int64_t)o * plane + (int64_t)gy * W + gx;
            v = out[idx] > 0.f ? dout[idx] : 0.f;
        }
        s_g[o][yy][xx] = v;
    }
    __syncthreads();
    const int ly = tid / kTileSide, lx = tid % kTileSide;
    const int gy = ty0 + ly, gx = tx0 + lx;
    if (gy >= H || gx >= W) return;
    float acc[CIN];
#pragma unroll
    for (int c = 0; c < CIN; c++) acc[c] = 0.f;
    for (int o = 0; o < COUT; o++)
#pragma unroll
        for (int ky = 0; ky < K; ky++)
#pragma unroll
            for (int kx = 0; kx < K; kx++) {
                const float g = s_g[o][ly + 2 * R - ky][lx + 2 * R - kx];
#pragma unroll
                for (int c = 0; c < CIN; c++) acc[c] = fmaf(s_w[(o * CIN + c) * K * K + ky * K + kx], g, acc[c]);
            }
    float* dst = din + (int64_t)n * CIN * plane + (int64_t)gy * W + gx;
#pragma unroll
    for (int c = 0; c < CIN; c++) dst[c * plane] = acc[c];
}

// Gradients of the weights and bias of a conv + ReLU layer, accumulated into dW / db.
// Persistent over (sample, tile); thread t owns the (output o = t / CIN, input c = t % CIN)
// channel pair with all K*K taps, and threads with c == 0 also the bias of o.
template <int K, int CIN, int COUT, bool kHalfIn>
__global__ void __launch_bounds__(kConvThreads) sg_conv_bwd_weight(const void* __restrict__ in, int64_t in_stride,
                                                                   const float* __restrict__ norm,
                                                                   const float* __restrict__ dout,
                                                                   const float* __restrict__ out,
                                                                   float* __restrict__ dW, float* __restrict__ db,
                                                                   int H, int W, int tiles_x, int tiles, int nsamples) {
    static_assert(CIN * COUT <= kConvThreads, "one (out, in) channel pair per thread");
    constexpr int R = K / 2, S = kTileSide + K - 1;
    __shared__ float s_in[CIN][S][S + 1];
    __shared__ float s_g[COUT][kTileSide * kTileSide];
    const int tid = threadIdx.x;
    const int o = tid / CIN, c = tid - (tid / CIN) * CIN;
    const bool owner = tid < CIN * COUT;
    float acc[K * K];
#pragma unroll
    for (int k = 0; k < K * K; k++) acc[k] = 0.f;
    float accb = 0.f;
    const int64_t plane = (int64_t)H * W;
    for (int item = blockIdx.x; item < tiles * nsamples; item += gridDim.x) {
        const int n = item / tiles, t = item - n * tiles;
        const int ty0 = (t / tiles_x) * kTileSide, tx0 = (t % tiles_x) * kTileSide;
        __syncthreads();
        for (int i = tid; i < CIN * S * S; i += kConvThreads) {
            const int cc = i / (S * S), r = i - cc * S * S, yy = r / S, xx = r - yy * S;
            const int gy = ty0 + yy - R, gx = tx0 + xx - R;
            float v = 0.f;
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
                const int64_t idx = (int64_t)cc * plane + (int64_t)gy * W + gx;
                if (kHalfIn)
                    v = (__half2float(static_cast<const __half*>(in)[n * in_stride + idx]) - norm[cc]) * norm[CIN + cc];
                else
                    v = static_cast<const float*>(in)[n * in_stride + idx];
            }
            s_in[cc][yy][xx] = v;
        }
        for (int i = tid; i < COUT * kTileSide * kTileSide; i += kConvThreads) {
            const int oo = i / (kTileSide * kTileSide), p = i - oo * kTileSide * kTileSide;
            const int gy = ty0 + p / kTileSide, gx = tx0 + p % kTileSide;
            float v = 0.f;
            if (gy < H && gx < W) {
                const int64_t idx = (int64_t)n * COUT * plane + (int64_t)oo * plane + (int64_t)gy * W + gx;
                v = out[idx] > 0.f ? dout[idx] : 0.f;
            }
            s_g[oo][p] = v;
        }
        __syncthreads();
        if (owner) {
            for (int p = 0; p < kTileSide * kTileSide; p++) {
                const float g = s_g[o][p];
                const int py = p / kTileSide, px = p % kTileSide;
#pragma unroll
                for (int ky = 0; ky < K; ky++)
#pragma unroll
                    for (int kx = 0; kx < K; kx++) acc[ky * K + kx] = fmaf(g, s_in[c][py + ky][px + kx], acc[ky * K + kx]);
                if (c == 0) accb += g;
            }
        }
    }
    if (owner) {
#pragma unroll
        for (int k = 0; k < K * K; k++) atomicAdd(dW + (o * CIN + c) * K * K + k, acc[k]);
        if (c == 0) atomicAdd(db + o, accb);
    }
}

// Head, loss and their gradients; one thread per sample, block reductions for the shared
// gradients.  With targets == nullptr only predictions are written.
__global__ void __launch_bounds__(256) sg_head(const float* __restrict__ feat, const float* __restrict__ params,
                                               const float* __restrict__ targets, float* __restrict__ pred, int n,
                                               float* __restrict__ dfeat, float* __restrict__ grads,
                                               float* __restrict__ loss) {
    __shared__ float red[kFeat + 2][8];
    const int i = blockIdx.x * 256 + threadIdx.x, tid = threadIdx.x;
    float y = 0.f, dy = 0.f, l = 0.f;
    float f[kFeat];
    if (i < n) {
        y = params[obh];
#pragma unroll
        for (int k = 0; k < kFeat; k++) {
            f[k] = feat[i * kFeat + k];
            y = fmaf(params[oWh + k], f[k], y);
        }
        if (pred) pred[i] = kScoreShift + kScoreScale * y;
        if (targets) {
            const float e = y - (targets[i] - kScoreShift) / kScoreScale;
            l = e * e / (float)n;
            dy = 2.f * e / (float)n;
#pragma unroll
            for (int k = 0; k < kFeat; k++) dfeat[i * kFeat + k] = dy * params[oWh + k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < kFeat; k++) f[k] = 0.f;
    }
    if (!targets) return;
    // Block sums of dy * f (head weights), dy (head bias) and the loss.
    for (int k = 0; k < kFeat + 2; k++) {
        float v = k < kFeat ? dy * f[k] : (k == kFeat ? dy : l);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if ((tid & 31) == 0) red[k][tid >> 5] = v;
    }
    __syncthreads();
    if (tid < kFeat + 2) {
        float v = 0.f;
        for (int wi = 0; wi < 8; wi++) v += red[tid][wi];
        if (tid < kFeat) atomicAdd(grads + oWh + tid, v);
        else if (tid == kFeat) atomicAdd(grads + obh, v);
        else atomicAdd(loss, v);
    }
}

// Gradient of conv3's output from the pooled features' gradients:
// d x = (dmean + dq * (m4 + eps)^(-3/4) * x^3) / HW.
__global__ void sg_pool_bwd(const float* __restrict__ act, const float* __restrict__ dfeat, const float* __restrict__ m4,
                            int HW, int level, float* __restrict__ dact) {
    const int n = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= HW) return;
    const float inv = 1.f / (float)HW;
#pragma unroll
    for (int c = 0; c < kC3; c++) {
        const int64_t idx = ((int64_t)n * kC3 + c) * HW + i;
        const float x = act[idx];
        const float dm = dfeat[n * kFeat + level * 2 * kC3 + c];
        const float dq = dfeat[n * kFeat + level * 2 * kC3 + kC3 + c];
        const float k = powf(m4[n * 2 * kC3 + level * kC3 + c] + kPoolEps, -0.75f);
        dact[idx] = (dm + dq * k * x * x * x) * inv;
    }
}

// Adam on the FP32 masters; refreshes the FP16 copies the kernels read.
__global__ void sg_adam(float* __restrict__ p, __half* __restrict__ p16, const float* __restrict__ g,
                        float* __restrict__ m, float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                        float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    p16[i] = __float2half_rn(pi);
}

// Copies the input blocks and targets of the samples idx[0..n) into a contiguous batch.
__global__ void sg_gather(const __half* __restrict__ inputs, int64_t block, const float* __restrict__ targets,
                          const int* __restrict__ idx, __half* __restrict__ out, float* __restrict__ tout) {
    const int b = blockIdx.y;
    const int64_t src = (int64_t)idx[b] * block;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < block; i += (int64_t)gridDim.x * blockDim.x)
        out[(int64_t)b * block + i] = inputs[src + i];
    if (blockIdx.x == 0 && threadIdx.x == 0) tout[b] = targets[idx[b]];
}

// acc[0] += v[0] (the running loss of an epoch, kept on the device).
__global__ void sg_add(float* acc, const float* v) { acc[0] += v[0]; }

__global__ void sg_to_half(const float* __restrict__ p, __half* __restrict__ h, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) h[i] = __float2half_rn(p[i]);
}

// ------------------------------------------------------------------------------------------
// Engine
// ------------------------------------------------------------------------------------------

inline int tiles_of(int h, int w) { return (int)(ceil_div(h, kTileSide) * ceil_div(w, kTileSide)); }

class Engine final : public SurrogateApi {
public:
    ~Engine() override { release(); }

    void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, int device) override {
        device_ = device;
        geo_[0] = make_geometry(src);
        geo_[1] = make_geometry(dis);
        if (geo_[0].generic() || geo_[1].generic())
            VSHIP_THROW(Vship_BadErrorType, "the surrogate takes colourspaces without resize or crop");
        if (geo_[0].OW != geo_[1].OW || geo_[0].OH != geo_[1].OH) VSHIP_THROW(Vship_DifferingInputType, "");
        for (int c = 0; c < 2; c++) cp_[c] = make_colour_params(c ? dis : src, geo_[c], false);
        const int W = (int)geo_[0].OW, H = (int)geo_[0].OH;
        // Coarse pyramid: levels 3 and 4, all three planes.
        pyr_ = ssimu2::make_pyramid(W, H);
        int64_t off = 0;
        for (int s = 0; s < ssimu2::kScales; s++)
            for (int p = 0; p < 3; p++) {
                if (s == 3 || s == 4) {
                    pyr_.off[s][p] = off;
                    off += round_up((int64_t)pyr_.pitch[s] * pyr_.h[s], 64);
                } else {
                    pyr_.off[s][p] = -1;
                }
            }
        pyr_.image_floats = round_up(off, 64);
        l3_ = Level{pyr_.h[3], pyr_.w[3], 0};
        l4_ = Level{pyr_.h[4], pyr_.w[4], (int64_t)kCin * l3_.h * l3_.w};
        block_ = l4_.off + (int64_t)kCin * l4_.h * l4_.w;
        CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        coarse_ = device_alloc<float>((size_t)(2 * kMaxChunk * pyr_.image_floats), "surrogate coarse pyramids");
        params_ = device_alloc<float>(kParams, "surrogate parameters");
        params16_ = device_alloc<__half>(kParams, "surrogate parameters (FP16)");
        grads_ = device_alloc<float>(kParams + 1, "surrogate gradients");
        adam_m_ = device_alloc<float>(kParams, "surrogate Adam moments");
        adam_v_ = device_alloc<float>(kParams, "surrogate Adam moments");
        norm_ = device_alloc<float>(2 * kCin, "surrogate input normalisation");
        host_params_.assign(kParams, 0.f);
        host_norm_.assign(2 * kCin, 0.f);
        for (int c = 0; c < kCin; c++) host_norm_[kCin + c] = 1.f;
        init_weights(1);
        upload_model();
    }

    int64_t input_elems() const override { return block_; }
    int num_params() const override { return kParams; }

    // Colour parameters of both clips for these strides (validated; a null stride array
    // skips its clip).
    void validate(const int64_t ls1[3], const int64_t ls2[3], ColourParams cp[2]) const {
        cp[0] = cp_[0];
        cp[1] = cp_[1];
        for (int c = 0; c < 2; c++) {
            const int64_t* ls = c ? ls2 : ls1;
            if (!ls) continue;
            for (int p = 0; p < 3; p++) {
                if (ls[p] < geo_[c].pw[p] * geo_[c].bytes) VSHIP_THROW(Vship_BadPointer, "lineSize smaller than one row of samples");
                if (ls[p] % geo_[c].bytes) cp[c].misaligned = 1;
            }
        }
    }

    // Levels 3 and 4 of `chunk` images into coarse_: pairs (clip -1: d1 and d2 interleaved),
    // or the images of one clip (0: d1, 1: d2).
    void coarse_front(int chunk, int clip, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t* ls1,
                      const int64_t* ls2, const ColourParams cp[2], cudaStream_t stream) {
        CoarseArgs& a = coarse_args_;
        a.cp[0] = cp[0];
        a.cp[1] = cp[1];
        a.pyr = pyr_;
        a.out = coarse_;
        a.clip = clip;
        const int per = clip < 0 ? 2 : 1;
        for (int i = 0; i < chunk; i++)
            for (int k = 0; k < per; k++) {
                const int c = clip < 0 ? k : clip;
                const uint8_t* const* src = c ? d2 : d1;
                RawImage& r = a.raw[per * i + k];
                for (int p = 0; p < 3; p++) {
                    if (!src[3 * i + p]) VSHIP_THROW(Vship_BadPointer, "null plane pointer");
                    r.p[p] = src[3 * i + p];
                    r.stride[p] = (c ? ls2 : ls1)[p];
                }
                if (misaligned_view(r, geo_[c])) a.cp[c].misaligned = 1;
            }
        const int f0 = fast_path_of(a.cp[0]), f1 = fast_path_of(a.cp[1]);
        const int fast = clip == 0 ? f0 : clip == 1 ? f1 : (f0 == f1 ? f0 : kFastGeneric);
        const int smem = (int)sizeof(float) * std::max(chroma_stage_floats(a.cp[0].subw, a.cp[0].subh),
                                                       chroma_stage_floats(a.cp[1].subw, a.cp[1].subh));
        auto kern = fast == kFastYuv420Bt709 ? sg_coarse_front_kernel<kFastYuv420Bt709>
                  : fast == kFastRgb8Srgb ? sg_coarse_front_kernel<kFastRgb8Srgb>
                                          : sg_coarse_front_kernel<kFastGeneric>;
        if (smem > 32 * 1024) CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        const dim3 grid((unsigned)ceil_div(pyr_.w[1], 32), (unsigned)ceil_div(pyr_.h[1], 32), (unsigned)(per * chunk));
        const int t = timer_.begin(0, "surrogate_coarse_front", stream);
        kern<<<grid, 256, smem, stream>>>(a);
        CUDA_CHECK(cudaGetLastError());
        timer_.end(t, stream);
    }

    void inputs(int n, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t ls1[3], const int64_t ls2[3],
                void* d_inputs, cudaStream_t stream) override {
        ColourParams cp[2];
        validate(ls1, ls2, cp);
        __half* out = static_cast<__half*>(d_inputs);
        for (int done = 0; done < n; done += kMaxChunk) {
            const int chunk = std::min(kMaxChunk, n - done);
            coarse_front(chunk, -1, d1 + 3 * done, d2 + 3 * done, ls1, ls2, cp, stream);
            const int npx = l3_.h * l3_.w + l4_.h * l4_.w;
            sg_pack_kernel<<<dim3((unsigned)ceil_div(npx, 256), (unsigned)chunk), 256, 0, stream>>>(
                coarse_, pyr_, l3_, l4_, block_, out + (int64_t)done * block_);
            CUDA_CHECK(cudaGetLastError());
        }
    }

    int64_t reference_floats() const override { return 3 * ((int64_t)l3_.h * l3_.w + (int64_t)l4_.h * l4_.w); }

    void references(int n, const uint8_t* const* d1, const int64_t ls1[3], float* d_refs, cudaStream_t stream) override {
        ColourParams cp[2];
        validate(ls1, nullptr, cp);
        for (int done = 0; done < n; done += kMaxChunk) {
            const int chunk = std::min(kMaxChunk, n - done);
            coarse_front(chunk, 0, d1 + 3 * done, nullptr, ls1, nullptr, cp, stream);
            const int npx = l3_.h * l3_.w + l4_.h * l4_.w;
            sg_pack_reference_kernel<<<dim3((unsigned)ceil_div(npx, 256), (unsigned)chunk), 256, 0, stream>>>(
                coarse_, pyr_, l3_, l4_, reference_floats(), d_refs + (int64_t)done * reference_floats());
            CUDA_CHECK(cudaGetLastError());
        }
    }

    void predict_against(int n, const float* d_refs, const uint8_t* const* d2, const int64_t ls2[3], float* d_pred,
                         cudaStream_t stream) override {
        ColourParams cp[2];
        validate(nullptr, ls2, cp);
        constexpr int kChunk = 256;
        if (!pred_inputs_) pred_inputs_ = device_alloc<__half>((size_t)kChunk * block_, "surrogate prediction inputs");
        for (int base = 0; base < n; base += kChunk) {
            const int count = std::min(kChunk, n - base);
            for (int done = 0; done < count; done += kMaxChunk) {
                const int chunk = std::min(kMaxChunk, count - done);
                const int first = base + done;
                coarse_front(chunk, 1, nullptr, d2 + 3 * first, nullptr, ls2, cp, stream);
                const int npx = l3_.h * l3_.w + l4_.h * l4_.w;
                sg_pack_against_kernel<<<dim3((unsigned)ceil_div(npx, 256), (unsigned)chunk), 256, 0, stream>>>(
                    coarse_, pyr_, l3_, l4_, d_refs + (int64_t)first * reference_floats(), reference_floats(), block_,
                    pred_inputs_ + (int64_t)done * block_);
                CUDA_CHECK(cudaGetLastError());
            }
            predict_inputs(count, pred_inputs_, d_pred + base, stream);
        }
    }

    void predict_inputs(int n, const void* d_inputs, float* d_pred, cudaStream_t stream) override {
        for (int done = 0; done < n; done += kBatchCap) {
            const int chunk = std::min(kBatchCap, n - done);
            ensure_batch(chunk);
            const int t = timer_.begin(1, "surrogate_forward", stream);
            forward(chunk, static_cast<const __half*>(d_inputs) + (int64_t)done * block_, stream);
            sg_head<<<(unsigned)ceil_div(chunk, 256), 256, 0, stream>>>(feat_, params_, nullptr, d_pred + done, chunk,
                                                                         nullptr, nullptr, nullptr);
            CUDA_CHECK(cudaGetLastError());
            timer_.end(t, stream);
        }
    }

    void predict(int n, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t ls1[3], const int64_t ls2[3],
                 float* d_pred, cudaStream_t stream) override {
        constexpr int kChunk = 256;
        if (!pred_inputs_) pred_inputs_ = device_alloc<__half>((size_t)kChunk * block_, "surrogate prediction inputs");
        for (int done = 0; done < n; done += kChunk) {
            const int chunk = std::min(kChunk, n - done);
            inputs(chunk, d1 + 3 * done, d2 + 3 * done, ls1, ls2, pred_inputs_, stream);
            predict_inputs(chunk, pred_inputs_, d_pred + done, stream);
        }
    }

    double gradients(int n, const void* d_inputs, const float* d_targets, float* grads_host) override {
        if (n > kBatchCap) VSHIP_THROW(Vship_BadErrorType, "gradient batches hold at most 1024 samples");
        ensure_batch(n);
        CUDA_CHECK(cudaMemsetAsync(grads_, 0, sizeof(float) * (kParams + 1), stream_));
        step_grads(n, static_cast<const __half*>(d_inputs), d_targets, stream_);
        std::vector<float> g(kParams + 1);
        CUDA_CHECK(cudaMemcpyAsync(g.data(), grads_, sizeof(float) * (kParams + 1), cudaMemcpyDeviceToHost, stream_));
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        if (grads_host) std::memcpy(grads_host, g.data(), sizeof(float) * kParams);
        return (double)g[kParams];
    }

    void train(int n, const void* d_inputs, const float* d_targets, int epochs, int batch, float lr, unsigned seed,
               float* loss_history) override {
        if (n < 1 || batch < 1 || batch > kBatchCap || epochs < 1)
            VSHIP_THROW(Vship_BadErrorType, "training needs n >= 1, 1 <= batch <= 1024, epochs >= 1");
        const __half* inputs = static_cast<const __half*>(d_inputs);
        fit_normalisation(n, inputs);
        init_weights(seed);
        upload_model();
        CUDA_CHECK(cudaMemsetAsync(adam_m_, 0, sizeof(float) * kParams, stream_));
        CUDA_CHECK(cudaMemsetAsync(adam_v_, 0, sizeof(float) * kParams, stream_));
        ensure_batch(batch);
        int* idx_d = device_alloc<int>((size_t)n, "surrogate sample order");
        __half* bin = nullptr;
        float* bt = nullptr;
        std::mt19937 rng(seed);
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        const int steps_per_epoch = std::max(1, n / batch);
        const int b = std::min(batch, n);
        const int total_steps = steps_per_epoch * epochs;
        int step = 0;
        const float b1 = 0.9f, b2 = 0.999f;
        try {
            bin = device_alloc<__half>((size_t)b * block_, "surrogate batch inputs");
            bt = device_alloc<float>((size_t)b, "surrogate batch targets");
            for (int e = 0; e < epochs; e++) {
                std::shuffle(order.begin(), order.end(), rng);
                CUDA_CHECK(cudaMemcpyAsync(idx_d, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream_));
                CUDA_CHECK(cudaMemsetAsync(loss_acc_, 0, sizeof(float), stream_));
                for (int s = 0; s < steps_per_epoch; s++, step++) {
                    sg_gather<<<dim3(64, (unsigned)b), 256, 0, stream_>>>(inputs, block_, d_targets, idx_d + s * b, bin, bt);
                    CUDA_CHECK(cudaGetLastError());
                    CUDA_CHECK(cudaMemsetAsync(grads_, 0, sizeof(float) * (kParams + 1), stream_));
                    step_grads(b, bin, bt, stream_);
                    // Cosine decay from lr to lr / 20.
                    const float t = (float)step / (float)std::max(1, total_steps - 1);
                    const float lr_t = lr * (0.05f + 0.95f * 0.5f * (1.f + std::cos(3.14159265f * t)));
                    const float c1 = 1.f - std::pow(b1, (float)(step + 1)), c2 = 1.f - std::pow(b2, (float)(step + 1));
                    sg_adam<<<(unsigned)ceil_div(kParams, 256), 256, 0, stream_>>>(params_, params16_, grads_, adam_m_,
                                                                                    adam_v_, kParams, lr_t, b1, b2, 1e-8f,
                                                                                    c1, c2);
                    CUDA_CHECK(cudaGetLastError());
                    sg_add<<<1, 1, 0, stream_>>>(loss_acc_, grads_ + kParams);
                    CUDA_CHECK(cudaGetLastError());
                }
                float l = 0.f;
                CUDA_CHECK(cudaMemcpyAsync(&l, loss_acc_, sizeof(float), cudaMemcpyDeviceToHost, stream_));
                CUDA_CHECK(cudaStreamSynchronize(stream_));
                if (loss_history) loss_history[e] = l / (float)steps_per_epoch;
            }
        } catch (...) {
            (void)cudaStreamSynchronize(stream_);
            device_free(idx_d);
            device_free(bin);
            device_free(bt);
            throw;
        }
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        device_free(idx_d);
        device_free(bin);
        device_free(bt);
        CUDA_CHECK(cudaMemcpy(host_params_.data(), params_, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    }

    int get_model(float* out, int max) override {
        const int total = kParams + 2 * kCin;
        if (out && max >= total) {
            CUDA_CHECK(cudaMemcpy(host_params_.data(), params_, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
            std::memcpy(out, host_params_.data(), sizeof(float) * kParams);
            std::memcpy(out + kParams, host_norm_.data(), sizeof(float) * 2 * kCin);
        }
        return total;
    }

    void set_model(const float* in, int count) override {
        if (count != kParams + 2 * kCin) VSHIP_THROW(Vship_BadErrorType, "model size mismatch");
        std::memcpy(host_params_.data(), in, sizeof(float) * kParams);
        std::memcpy(host_norm_.data(), in + kParams, sizeof(float) * 2 * kCin);
        upload_model();
    }

    KernelTimer& timer() override { return timer_; }

private:
    static constexpr int kBatchCap = 1024;

    void init_weights(unsigned seed) {
        std::mt19937 rng(seed ^ 0x5EEDu);
        auto he = [&](int off, int count, int fan_in) {
            std::normal_distribution<float> d(0.f, std::sqrt(2.f / (float)fan_in));
            for (int i = 0; i < count; i++) host_params_[off + i] = d(rng);
        };
        std::fill(host_params_.begin(), host_params_.end(), 0.f);
        he(oW1, kC1 * kCin * 9, kCin * 9);
        he(oW2, kC2 * kC1 * 9, kC1 * 9);
        he(oW3, kC3 * kC2, kC2);
        std::normal_distribution<float> d(0.f, 0.05f);
        for (int i = 0; i < kFeat; i++) host_params_[oWh + i] = d(rng);
        for (int i = 0; i < kC1; i++) host_params_[ob1 + i] = 0.01f;
        for (int i = 0; i < kC2; i++) host_params_[ob2 + i] = 0.01f;
        for (int i = 0; i < kC3; i++) host_params_[ob3 + i] = 0.01f;
    }

    void upload_model() {
        CUDA_CHECK(cudaMemcpy(params_, host_params_.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(norm_, host_norm_.data(), sizeof(float) * 2 * kCin, cudaMemcpyHostToDevice));
        sg_to_half<<<(unsigned)ceil_div(kParams, 256), 256>>>(params_, params16_, kParams);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaDeviceSynchronize());
    }

    // Per-channel shift and scale of the inputs, measured on up to 512 training samples:
    // reference channels to zero mean and unit deviation, difference channels to unit RMS.
    void fit_normalisation(int n, const __half* inputs) {
        const int k = std::min(n, 512);
        std::vector<__half> h((size_t)k * block_);
        CUDA_CHECK(cudaMemcpy(h.data(), inputs, sizeof(__half) * h.size(), cudaMemcpyDeviceToHost));
        for (int c = 0; c < kCin; c++) {
            double s = 0, s2 = 0, cnt = 0;
            for (int i = 0; i < k; i++)
                for (const Level* lv : {&l3_, &l4_}) {
                    const __half* p = h.data() + (size_t)i * block_ + lv->off + (int64_t)c * lv->h * lv->w;
                    for (int j = 0; j < lv->h * lv->w; j++) {
                        const double v = (double)__half2float(p[j]);
                        s += v;
                        s2 += v * v;
                        cnt += 1;
                    }
                }
            const double mean = s / cnt, var = std::max(s2 / cnt - mean * mean, 1e-12);
            if (c < 3) {
                host_norm_[c] = (float)mean;
                host_norm_[kCin + c] = (float)(1.0 / std::sqrt(var));
            } else {
                host_norm_[c] = 0.f;
                host_norm_[kCin + c] = (float)(1.0 / std::sqrt(std::max(s2 / cnt, 1e-12)));
            }
        }
    }

    void ensure_batch(int n) {
        if (n <= batch_cap_) return;
        CUDA_CHECK(cudaDeviceSynchronize());
        free_batch();
        const int64_t px = (int64_t)l3_.h * l3_.w + (int64_t)l4_.h * l4_.w;
        const size_t cap = (size_t)kBatchCap;
        act1_ = device_alloc<float>(cap * kC1 * px, "surrogate activations");
        act2_ = device_alloc<float>(cap * kC2 * px, "surrogate activations");
        act3_ = device_alloc<float>(cap * kC3 * px, "surrogate activations");
        d1_ = device_alloc<float>(cap * kC1 * px, "surrogate activation gradients");
        d2_ = device_alloc<float>(cap * kC2 * px, "surrogate activation gradients");
        d3_ = device_alloc<float>(cap * kC3 * px, "surrogate activation gradients");
        feat_ = device_alloc<float>(cap * kFeat, "surrogate features");
        dfeat_ = device_alloc<float>(cap * kFeat, "surrogate feature gradients");
        m4_ = device_alloc<float>(cap * 2 * kC3, "surrogate pooling moments");
        const int64_t tiles = std::max(ceil_div(l3_.w, kFwdTW) * ceil_div(l3_.h, kFwdTH),
                                       ceil_div(l4_.w, kFwdTW) * ceil_div(l4_.h, kFwdTH));
        pool_ = device_alloc<float>(cap * (size_t)tiles * 2 * kC3, "surrogate pooling partials");
        loss_acc_ = device_alloc<float>(2, "surrogate loss");
        batch_cap_ = kBatchCap;
    }

    // Activation base of a level inside the activation buffers (level 3 first, then 4).
    int64_t level_base(int level, int n, int channels) const {
        return level == 0 ? 0 : (int64_t)n * channels * l3_.h * l3_.w;
    }

    void forward(int n, const __half* in, cudaStream_t st) {
        for (int L = 0; L < 2; L++) {
            const Level& lv = L ? l4_ : l3_;
            const int H = lv.h, W = lv.w, tx = (int)ceil_div(W, kFwdTW);
            const dim3 grid((unsigned)(tx * ceil_div(H, kFwdTH)), (unsigned)n);
            float* a1 = act1_ + level_base(L, n, kC1);
            float* a2 = act2_ + level_base(L, n, kC2);
            float* a3 = act3_ + level_base(L, n, kC3);
            sg_conv_fwd<3, kCin, kC1, true><<<grid, kFwdThreads, 0, st>>>(in + lv.off, block_, norm_, params16_ + oW1,
                                                                       params_ + ob1, a1, H, W, tx);
            sg_conv_fwd<3, kC1, kC2, false><<<grid, kFwdThreads, 0, st>>>(a1, (int64_t)kC1 * H * W, nullptr,
                                                                        params16_ + oW2, params_ + ob2, a2, H, W, tx);
            sg_conv_fwd<1, kC2, kC3, false, true><<<grid, kFwdThreads, 0, st>>>(
                a2, (int64_t)kC2 * H * W, nullptr, params16_ + oW3, params_ + ob3, a3, H, W, tx, pool_);
            sg_pool_finish<<<(unsigned)n, 256, 0, st>>>(pool_, (int)grid.x, H * W, feat_, m4_, L);
            CUDA_CHECK(cudaGetLastError());
        }
    }

    // Forward, loss and all gradients of one batch into grads_ (grads_[kParams] = loss).
    void step_grads(int n, const __half* in, const float* targets, cudaStream_t st) {
        forward(n, in, st);
        sg_head<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(feat_, params_, targets, nullptr, n, dfeat_, grads_,
                                                             grads_ + kParams);
        CUDA_CHECK(cudaGetLastError());
        int sms = 148;
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
        for (int L = 0; L < 2; L++) {
            const Level& lv = L ? l4_ : l3_;
            const int H = lv.h, W = lv.w, tx = (int)ceil_div(W, kTileSide), tiles = tiles_of(H, W);
            const dim3 grid((unsigned)tiles, (unsigned)n);
            const unsigned wgrid = (unsigned)std::min(tiles * n, sms * 4);
            float* a1 = act1_ + level_base(L, n, kC1);
            float* a2 = act2_ + level_base(L, n, kC2);
            float* a3 = act3_ + level_base(L, n, kC3);
            float* g1 = d1_ + level_base(L, n, kC1);
            float* g2 = d2_ + level_base(L, n, kC2);
            float* g3 = d3_ + level_base(L, n, kC3);
            sg_pool_bwd<<<dim3((unsigned)ceil_div(H * W, 256), (unsigned)n), 256, 0, st>>>(a3, dfeat_, m4_, H * W, L, g3);
            sg_conv_bwd_weight<1, kC2, kC3, false><<<wgrid, kConvThreads, 0, st>>>(
                a2, (int64_t)kC2 * H * W, nullptr, g3, a3, grads_ + oW3, grads_ + ob3, H, W, tx, tiles, n);
            sg_conv_bwd_data<1, kC2, kC3><<<grid, kConvThreads, 0, st>>>(g3, a3, params16_ + oW3, g2, H, W, tx);
            sg_conv_bwd_weight<3, kC1, kC2, false><<<wgrid, kConvThreads, 0, st>>>(
                a1, (int64_t)kC1 * H * W, nullptr, g2, a2, grads_ + oW2, grads_ + ob2, H, W, tx, tiles, n);
            sg_conv_bwd_data<3, kC1, kC2><<<grid, kConvThreads, 0, st>>>(g2, a2, params16_ + oW2, g1, H, W, tx);
            sg_conv_bwd_weight<3, kCin, kC1, true><<<wgrid, kConvThreads, 0, st>>>(
                in + lv.off, block_, norm_, g1, a1, grads_ + oW1, grads_ + ob1, H, W, tx, tiles, n);
            CUDA_CHECK(cudaGetLastError());
        }
    }

    void free_batch() {
        for (float** p : {&act1_, &act2_, &act3_, &d1_, &d2_, &d3_, &feat_, &dfeat_, &m4_, &pool_, &loss_acc_}) {
            device_free(*p);
            *p = nullptr;
        }
        batch_cap_ = 0;
    }

    void release() {
        if (stream_) (void)cudaStreamSynchronize(stream_);
        (void)cudaDeviceSynchronize();
        free_batch();
        for (float** p : {&coarse_, &params_, &grads_, &adam_m_, &adam_v_, &norm_}) {
            device_free(*p);
            *p = nullptr;
        }
        device_free(params16_);
        params16_ = nullptr;
        device_free(pred_inputs_);
        pred_inputs_ = nullptr;
        timer_.destroy();
        if (stream_) (void)cudaStreamDestroy(stream_);
        stream_ = nullptr;
    }

    int device_ = 0;
    ClipGeometry geo_[2];
    ColourParams cp_[2];
    Pyramid pyr_{};
    Level l3_{}, l4_{};
    int64_t block_ = 0;
    cudaStream_t stream_ = nullptr;
    CoarseArgs coarse_args_{};
    float* coarse_ = nullptr;
    float* params_ = nullptr;
    __half* params16_ = nullptr;
    __half* pred_inputs_ = nullptr;
    float* grads_ = nullptr;
    float* adam_m_ = nullptr;
    float* adam_v_ = nullptr;
    float* norm_ = nullptr;
    std::vector<float> host_params_, host_norm_;
    int batch_cap_ = 0;
    float *act1_ = nullptr, *act2_ = nullptr, *act3_ = nullptr;
    float* pool_ = nullptr;  // per-tile channel sums of the last layer
    float *d1_ = nullptr, *d2_ = nullptr, *d3_ = nullptr;
    float *feat_ = nullptr, *dfeat_ = nullptr, *m4_ = nullptr, *loss_acc_ = nullptr;
    KernelTimer timer_;
};

}  // namespace
}  // namespace surrogate
}  // namespace vship

vship::SurrogateApi* vship::make_surrogate_engine() { return new vship::surrogate::Engine(); }

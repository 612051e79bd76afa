// Host side of the colour front-end: turns a Vship_Colorspace_t into ColourParams and the
// input geometry, stages host planes into device memory, and provides the optional
// resize + crop path (Converter::convert, src/gpuColorToLinear/vshipColor.hpp:36-146).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>

#include "common.cuh"
#include "colour.cuh"

namespace vship {

inline int sample_bytes(int s) {
    switch (s) {
    case Vship_SampleUINT8: return 1;
    case Vship_SampleFLOAT: return 4;
    case Vship_SampleHALF:
    case Vship_SampleUINT9:
    case Vship_SampleUINT10:
    case Vship_SampleUINT12:
    case Vship_SampleUINT14:
    case Vship_SampleUINT16: return 2;
    default: return 0;
    }
}

inline int sample_bits(int s) {
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

// Geometry of one input clip.
struct ClipGeometry {
    int64_t W = 0, H = 0;          // luma plane size as delivered
    int64_t pw[3] = {0, 0, 0}, ph[3] = {0, 0, 0};
    int64_t TW = 0, TH = 0;        // size after the optional resize
    int64_t OW = 0, OH = 0;        // size after crop: the metric's size
    int crop_top = 0, crop_left = 0;
    bool resized = false, cropped = false;
    int bytes = 0;
    bool generic() const { return resized || cropped; }
};

inline ClipGeometry make_geometry(const Vship_Colorspace_t& cs) {
    ClipGeometry g;
    g.bytes = sample_bytes(cs.sample);
    if (g.bytes == 0) VSHIP_THROW(Vship_BadErrorType, "unknown Vship_Sample_t value " + std::to_string((int)cs.sample));
    if (cs.width <= 0 || cs.height <= 0) VSHIP_THROW(Vship_BadErrorType, "width and height must be positive");
    if (cs.subsampling.subw < 0 || cs.subsampling.subw > 2 || cs.subsampling.subh < 0 || cs.subsampling.subh > 1)
        VSHIP_THROW(Vship_BadErrorType, "chroma subsampling must satisfy subw in [0,2] and subh in [0,1]");
    g.W = cs.width;
    g.H = cs.height;
    for (int c = 0; c < 3; c++) {
        g.pw[c] = c ? ((g.W - 1) >> cs.subsampling.subw) + 1 : g.W;
        g.ph[c] = c ? ((g.H - 1) >> cs.subsampling.subh) + 1 : g.H;
    }
    g.TW = cs.target_width == -1 ? g.W : cs.target_width;
    g.TH = cs.target_height == -1 ? g.H : cs.target_height;
    if (g.TW <= 0 || g.TH <= 0) VSHIP_THROW(Vship_BadErrorType, "target size must be positive or -1");
    g.resized = (g.TW != g.W || g.TH != g.H);
    g.cropped = cs.crop.top != 0 || cs.crop.bottom != 0 || cs.crop.left != 0 || cs.crop.right != 0;
    g.crop_top = cs.crop.top;
    g.crop_left = cs.crop.left;
    g.OW = g.TW - cs.crop.left - cs.crop.right;
    g.OH = g.TH - cs.crop.top - cs.crop.bottom;
    if (cs.crop.top < 0 || cs.crop.bottom < 0 || cs.crop.left < 0 || cs.crop.right < 0 || g.OW <= 0 || g.OH <= 0)
        VSHIP_THROW(Vship_BadErrorType, "crop rectangle leaves no pixels");
    return g;
}

inline ColourParams make_colour_params(const Vship_Colorspace_t& cs, const ClipGeometry& g, bool misaligned) {
    ColourParams cp{};
    cp.sample = cs.sample;
    cp.bytes = g.bytes;
    const int bits = sample_bits(cs.sample);
    cp.mask = bits >= 16 ? 0xFFFFu : ((1u << bits) - 1u);
    cp.misaligned = misaligned ? 1 : 0;
    cp.full_range = cs.range == Vship_RangeFull;
    cp.full_scale = 1.0f / (float)((1 << bits) - 1);
    cp.lim_scale = bits >= 8 ? 1.0f / (float)(1 << (bits - 8)) : 256.f;
    cp.yuv_chroma = cs.colorFamily == Vship_ColorYUV;
    cp.subw = cs.subsampling.subw;
    cp.subh = cs.subsampling.subh;
    cp.hcenter = (cs.chromaLocation == Vship_ChromaLoc_Center || cs.chromaLocation == Vship_ChromaLoc_Top);
    cp.vcenter = (cs.chromaLocation == Vship_ChromaLoc_Center || cs.chromaLocation == Vship_ChromaLoc_Left);
    cp.matrix = cs.YUVMatrix;
    cp.trc = cs.transferFunction;
    cp.primaries = cs.primaries;
    cp.skip_yuv = (cs.transferFunction == Vship_TRC_Linear && cs.YUVMatrix == Vship_MATRIX_RGB);
    cp.W = g.W;
    cp.H = g.H;
    cp.cw = g.pw[1];
    cp.ch = g.ph[1];
    return cp;
}

// Bytes of one dense device copy of an image (planes back to back, each 256-byte aligned).
inline int64_t dense_image_bytes(const ClipGeometry& g, int64_t plane_off[3]) {
    int64_t off = 0;
    for (int c = 0; c < 3; c++) {
        plane_off[c] = off;
        off += round_up(g.pw[c] * g.bytes * g.ph[c], 256);
    }
    return off;
}

// Device staging area of one input image; grows (never shrinks) when a caller's strides need
// more room than the dense layout allocated at Init.
struct StagingBuffer {
    uint8_t* ptr = nullptr;
    size_t cap = 0;
    void ensure(size_t n, cudaStream_t stream) {
        if (n <= cap) return;
        CUDA_CHECK(cudaStreamSynchronize(stream));
        device_free(ptr);
        ptr = nullptr;
        cap = 0;
        ptr = device_alloc<uint8_t>(n, "input staging");
        cap = n;
    }
    void free() {
        device_free(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

// Host planes of one image lie back to back in one allocation (as FFVship lays out its
// pinned frames): the whole frame can go in one copy that keeps the caller's strides.
inline bool contiguous_planes(const ClipGeometry& g, const uint8_t* const src[3], const int64_t line_size[3]) {
    return src[1] == src[0] + line_size[0] * g.ph[0] && src[2] == src[1] + line_size[1] * g.ph[1];
}

// Device bytes copy_host_image() writes for these host planes (validates them).
inline int64_t host_image_bytes(const ClipGeometry& g, const uint8_t* const src[3], const int64_t line_size[3]) {
    for (int c = 0; c < 3; c++) {
        if (src[c] == nullptr) VSHIP_THROW(Vship_BadPointer, "null plane pointer");
        if (line_size[c] < g.pw[c] * g.bytes) VSHIP_THROW(Vship_BadPointer, "lineSize smaller than one row of samples");
    }
    if (contiguous_planes(g, src, line_size)) {
        const int64_t bytes = line_size[0] * g.ph[0] + line_size[1] * g.ph[1] + line_size[2] * (g.ph[2] - 1) +
                              g.pw[2] * g.bytes;
        return round_up(bytes, 256);
    }
    int64_t off[3];
    return dense_image_bytes(g, off);
}

// Copies the three host planes of one image to `dst` (host_image_bytes() bytes, 256-byte
// aligned) and returns the device view.  Contiguous planes go in one copy and keep the
// caller's strides; otherwise each plane is copied densely.  Bytes past the last row of the
// last plane are never read (the copy size follows src/gpuColorToLinear/vshipColor.hpp:96).
inline RawImage copy_host_image(uint8_t* dst, const ClipGeometry& g, const uint8_t* const src[3],
                                const int64_t line_size[3], cudaStream_t stream) {
    int64_t row[3];
    for (int c = 0; c < 3; c++) row[c] = g.pw[c] * g.bytes;
    RawImage im;
    if (contiguous_planes(g, src, line_size)) {
        const int64_t bytes = line_size[0] * g.ph[0] + line_size[1] * g.ph[1] + line_size[2] * (g.ph[2] - 1) + row[2];
        CUDA_CHECK(cudaMemcpyAsync(dst, src[0], (size_t)bytes, cudaMemcpyHostToDevice, stream));
        for (int c = 0; c < 3; c++) {
            im.p[c] = dst + (src[c] - src[0]);
            im.stride[c] = line_size[c];
        }
        return im;
    }
    int64_t off[3];
    dense_image_bytes(g, off);
    for (int c = 0; c < 3; c++) {
        im.p[c] = dst + off[c];
        im.stride[c] = row[c];
        if (line_size[c] == row[c]) {
            CUDA_CHECK(cudaMemcpyAsync(dst + off[c], src[c], (size_t)(row[c] * g.ph[c]), cudaMemcpyHostToDevice, stream));
        } else {
            CUDA_CHECK(cudaMemcpy2DAsync(dst + off[c], (size_t)row[c], src[c], (size_t)line_size[c], (size_t)row[c],
                                         (size_t)g.ph[c], cudaMemcpyHostToDevice, stream));
        }
    }
    return im;
}

// Copies the three host planes of one image into a staging buffer (grown as needed) and
// returns the device view.
inline RawImage stage_host_image(StagingBuffer& buf, const ClipGeometry& g, const uint8_t* const src[3],
                                 const int64_t line_size[3], cudaStream_t stream) {
    buf.ensure((size_t)host_image_bytes(g, src, line_size), stream);
    return copy_host_image(buf.ptr, g, src, line_size, stream);
}

// A stride or a plane address that is not a multiple of the sample size makes the kernels
// use byte loads.
inline bool misaligned_planes(const uint8_t* const p[3], const int64_t stride[3], int bytes) {
    for (int c = 0; c < 3; c++)
        if (stride[c] % bytes || (reinterpret_cast<uintptr_t>(p[c]) % bytes)) return true;
    return false;
}

inline bool misaligned_view(const RawImage& im, const ClipGeometry& g) { return misaligned_planes(im.p, im.stride, g.bytes); }

// ---- generic path: ingest to planar linear RGB, then resize (horizontalResizeTranspose,
// ---- src/gpuColorToLinear/resize.hpp:26-48), crop by offset.

// Planar linear RGB of one image (BT.709 primaries, or the clip's own when kNative), one
// 64x64 luma tile per CTA with its chroma staged in shared memory (dynamic:
// chroma_stage_floats(subw, subh) floats).
template <bool kNative>
static __global__ void __launch_bounds__(256) ingest_linear_kernel(RawImage im, ColourParams cp, float* out, int64_t plane_stride) {
    extern __shared__ float stage_mem[];
    const int X0 = blockIdx.x * kStageTile, Y0 = blockIdx.y * kStageTile;
    ChromaStage st{};
    if (cp.subw || cp.subh) chroma_stage(im, cp, X0, Y0, stage_mem, st);
    for (int i = threadIdx.x; i < kStageTile * kStageTile; i += blockDim.x) {
        const int X = X0 + (i & (kStageTile - 1)), Y = Y0 + i / kStageTile;
        if (X >= cp.W || Y >= cp.H) continue;
        const float3 v = ingest_staged<kNative>(im, cp, st, X, Y, X0, Y0);
        const int64_t o = (int64_t)Y * cp.W + X;
        out[o] = v.x;
        out[plane_stride + o] = v.y;
        out[2 * plane_stride + o] = v.z;
    }
}

// Linear RGB of 8-bit R'G'B' sRGB planes (the kFastRgb8Srgb colourspaces): four pixels of a
// row per thread, one 32-bit load per plane when the four samples are 4-byte aligned and one
// float4 store per plane when the output is; each value is ingest_fast<kFastRgb8Srgb>'s.
static __global__ void __launch_bounds__(256) ingest_linear_rgb8_kernel(RawImage im, ColourParams cp, float* out,
                                                                       int64_t plane_stride) {
    const int64_t qw = (cp.W + 3) / 4;
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t Y = q / qw, X = (q - Y * qw) * 4;
    if (Y >= cp.H) return;
    const int n = (int)min((int64_t)4, cp.W - X);
    const int64_t o = Y * cp.W + X;
#pragma unroll
    for (int p = 0; p < 3; p++) {
        const uint8_t* src = im.p[p] + Y * im.stride[p] + X;
        float v[4];
        if (n == 4 && (reinterpret_cast<uintptr_t>(src) & 3) == 0) {
            const uchar4 u = __ldg(reinterpret_cast<const uchar4*>(src));
            v[0] = srgb_to_linear(range_luma((float)u.x, cp));
            v[1] = srgb_to_linear(range_luma((float)u.y, cp));
            v[2] = srgb_to_linear(range_luma((float)u.z, cp));
            v[3] = srgb_to_linear(range_luma((float)u.w, cp));
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) v[k] = k < n ? srgb_to_linear(range_luma((float)__ldg(src + k), cp)) : 0.f;
        }
        float* dst = out + p * plane_stride + o;
        if (n == 4 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
            *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (k < n) dst[k] = v[k];
        }
    }
}

inline void launch_ingest_linear(const RawImage& im, const ColourParams& cp, float* out, int64_t plane_stride, cudaStream_t st,
                                 bool native = false) {
    if (!native && fast_path_of(cp) == kFastRgb8Srgb) {
        const int64_t quads = (cp.W + 3) / 4 * cp.H;
        ingest_linear_rgb8_kernel<<<(unsigned)ceil_div(quads, 256), 256, 0, st>>>(im, cp, out, plane_stride);
        CUDA_CHECK(cudaGetLastError());
        return;
    }
    const dim3 grid((unsigned)ceil_div(cp.W, kStageTile), (unsigned)ceil_div(cp.H, kStageTile));
    const size_t smem = sizeof(float) * chroma_stage_floats(cp.subw, cp.subh);
    auto kernel = native ? ingest_linear_kernel<true> : ingest_linear_kernel<false>;
    if (smem > 48 * 1024) CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<grid, 256, smem, st>>>(im, cp, out, plane_stride);
    CUDA_CHECK(cudaGetLastError());
}

// One pass of the separable resize: rows of length sw resized to rw samples, written
// transposed (dst is rw x sh).  The source coordinate is formed in float as in the reference.
static __global__ void resize_transpose_kernel(const float* src, float* dst, int64_t sw, int64_t sh, int64_t rw) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rw * sh) return;
    const int64_t x = i % rw, y = i / rw;
    const float approx = (float)x * (float)sw / (float)rw;
    const int64_t b = (int64_t)approx;
    const float* row = src + y * sw;
    const float v1 = row[b];
    const float v0 = b - 1 >= 0 ? row[b - 1] : v1;
    const float v2 = b + 1 < sw ? row[b + 1] : v1;
    const float v3 = b + 2 < sw ? row[b + 2] : v2;
    dst[x * sh + y] = hermite(v1, (v2 - v0) / 2.f, v2, (v3 - v1) / 2.f, approx - (float)b);
}

// Linear RGB of the generic path: planes of TW x TH floats (after resize); the metric reads
// the crop window at offset crop_top * TW + crop_left with pitch TW.
struct GenericLinear {
    float* planes = nullptr;   // 3 * TW * TH
    float* scratch = nullptr;  // W*H*3 (ingest) + TW*H (resize intermediate)
    int64_t plane_floats = 0;

    void alloc(const ClipGeometry& g) {
        plane_floats = g.TW * g.TH;
        planes = device_alloc<float>((size_t)(3 * plane_floats), "resized linear planes");
        if (g.resized) scratch = device_alloc<float>((size_t)(3 * g.W * g.H + g.TW * g.H), "resize scratch");
    }
    void free() {
        device_free(planes);
        device_free(scratch);
        planes = scratch = nullptr;
    }
    void run(const RawImage& im, const ColourParams& cp, const ClipGeometry& g, cudaStream_t stream, bool native = false) {
        const int64_t n = g.W * g.H;
        float* lin = g.resized ? scratch : planes;
        const int64_t lin_stride = g.resized ? n : plane_floats;
        launch_ingest_linear(im, cp, lin, lin_stride, stream, native);
        if (!g.resized) return;
        float* mid = scratch + 3 * n;
        for (int c = 0; c < 3; c++) {
            resize_transpose_kernel<<<(unsigned)ceil_div(g.TW * g.H, 256), 256, 0, stream>>>(lin + c * n, mid, g.W, g.H, g.TW);
            CUDA_CHECK(cudaGetLastError());
            resize_transpose_kernel<<<(unsigned)ceil_div(g.TH * g.TW, 256), 256, 0, stream>>>(mid, planes + c * plane_floats, g.H, g.TW, g.TH);
            CUDA_CHECK(cudaGetLastError());
        }
    }
    const float* window() const { return planes; }
};

}  // namespace vship

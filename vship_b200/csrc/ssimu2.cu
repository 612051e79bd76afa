// SSIMULACRA2 engine for B200 (sm_100a).
//
// Per frame pair the reference (src/ssimu2/main.hpp:27-156, score.hpp:380-460) runs about
// 70 launches: colour conversion, 30 box downsamples, one XYB pass, 11 map kernels with
// 1-2 tree reductions each, then a blocking copy of 108 floats and the score on the host.
// This engine runs three kernels for any number of pairs of one handler:
//
//   1. ssimu2_front_kernel  raw planes -> linear RGB -> 6-level 2x box pyramid -> positive XYB
//                           (one 64x64 tile of level 0 per CTA; levels 1-5 of the tile are
//                           built in shared memory; only planes some map reads are stored)
//   2. ssimu2_maps_kernel   one launch over a work list of 32x32 output tiles of every
//                           unpruned (pair, plane, scale): 48x48 halo tiles of both images,
//                           separable 17-tap renormalised blur of a-k, b-k, (a-k)(b-k) and
//                           (a-b)^2 in shared memory (k: a per-tile shift), SSIM / artifact /
//                           detail-loss maps in a cancellation-free form, per-tile sums of x
//                           and x^4 in FP64
//   3. ssimu2_final_kernel  per pair: FP64 sum of tile partials, 4th roots, the 108 features
//                           and the score, computed like the reference's final_score
//
// Storage is FP32 end to end: storing levels in FP16 biases the SSIM 1-norms by ~1e-5 per
// pixel (quantisation noise adds ~2e-8 to each local variance), which moves the score by
// ~1e-2, ten times the accepted error.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"
#include "colour.cuh"
#include "frontend.cuh"
#include "metric_tables.h"
#include "ssimu2_device.cuh"
#include "engines.h"
#include "../../include/VshipAPI_ext.h"

namespace vship {
namespace ssimu2 {

constexpr int kMaxBatch = 64;  // pairs per launch

struct FrontArgs {
    ColourParams cp[2];      // [0] reference clip, [1] distorted clip
    const float* lin[2];     // generic path: linear RGB planes of the two clips (crop window)
    int64_t lin_plane[2];    // floats between planes
    int64_t lin_pitch[2];    // row pitch of the linear planes
    float* xyb;              // pyramid base; image i starts at xyb + i * pyr.image_floats
    Pyramid pyr;
    RawImage raw[2 * kMaxBatch];  // one per image (images alternate reference / distorted)
};

template <bool FromLinear, int kFast>
__global__ void __launch_bounds__(256, 4) ssimu2_front_kernel(const __grid_constant__ FrontArgs a) {
    __shared__ FrontSmem fs;
    extern __shared__ float stage_mem[];
    const int img = blockIdx.z;
    const int clip = img & 1;
    const LinearIn lin{a.lin[clip], a.lin_plane[clip], a.lin_pitch[clip]};
    front_tile<FromLinear, kFast>(fs, stage_mem, a.cp[clip], a.raw[img], lin, a.pyr,
                                  a.xyb + (int64_t)img * a.pyr.image_floats, blockIdx.x, blockIdx.y);
}

// One unpruned (pair, plane, scale) of the map work list.
struct MapSeg {
    const float* a;       // reference XYB plane
    const float* b;       // distorted XYB plane
    int w, h, pitch;
    int tiles_x;
    int tile_begin;       // first global tile index of this segment
    int ntiles;
    int slot;             // plane * 36 + scale * 6
    int on;               // bit k set: map k (ssim, artifact, detail-loss) is unpruned
};

// The work list of one pair, passed by value: the pairs of a batch differ only in their base
// pointer (pair p's reference plane is xyb + 2p * image_floats + off, its distorted plane
// image_floats further).
struct MapTemplate {
    struct Seg {
        int64_t off;
        int w, h, pitch, tiles_x, tile_begin;
    } seg[18];
    int nseg;
    int tiles_per_pair;
    const float* xyb;
    int64_t image_floats;
};

__device__ __forceinline__ TileRef locate_tile(const MapTemplate& mt, int tile) {
    const int pair = tile / mt.tiles_per_pair;
    const int lt = tile - pair * mt.tiles_per_pair;
    int s = 0;
#pragma unroll 1
    for (int i = 1; i < mt.nseg; i++)
        if (mt.seg[i].tile_begin <= lt) s = i;
    const MapTemplate::Seg& g = mt.seg[s];
    TileRef t;
    t.a = mt.xyb + (int64_t)(2 * pair) * mt.image_floats + g.off;
    t.b = t.a + mt.image_floats;
    t.w = g.w;
    t.h = g.h;
    t.pitch = g.pitch;
    const int l = lt - g.tile_begin;
    const int ty = l / g.tiles_x;
    t.X0 = (l - ty * g.tiles_x) * kTile;
    t.Y0 = ty * kTile;
    return t;
}

// Persistent: CTA b scores tiles b, b + gridDim.x, ...; the halo of the next tile is loaded
// into registers while the current one is blurred.
__global__ void __launch_bounds__(kMapThreads) ssimu2_maps_kernel(const __grid_constant__ MapTemplate mt, int total_tiles,
                                                                  double* __restrict__ partials) {
    using MT = MapTile<kTile>;
    __shared__ MT::Smem sm;
    int tile = blockIdx.x;
    if (tile >= total_tiles) return;
    TileRef cur = locate_tile(mt, tile);
    HaloV4 regs;
    load_halo_v4(cur, regs);

    while (true) {
        stage_halo_v4(sm, regs, cur.X0, cur.Y0, cur.w, cur.h);
        const int X0 = cur.X0, Y0 = cur.Y0, w = cur.w, h = cur.h;
        const int next = tile + gridDim.x;
        if (next < total_tiles) {
            cur = locate_tile(mt, next);
            load_halo_v4(cur, regs);
        }
        blur_score_tile<kTile>(sm, X0, Y0, w, h, partials + (int64_t)tile * 6);
        if (next >= total_tiles) break;
        tile = next;
        __syncthreads();
    }
}

// Per pair: FP64 totals of the tile partials, the 108 features, and the score exactly as
// final_score computes it (src/ssimu2/score.hpp:442-460: float fmaf accumulation, float
// result).
__global__ void __launch_bounds__(256) ssimu2_final_kernel(const MapSeg* __restrict__ segs, int segs_per_pair,
                                                           const double* __restrict__ partials,
                                                           double* __restrict__ scores, float* __restrict__ features) {
    // Every warp walks all segments and leaves its per-segment sums in shared memory, so the
    // segments need no barrier each; one barrier, then one thread per (segment, map) forms the
    // feature.  Per thread, per warp and across warps the additions are in the same order as
    // a segment-by-segment loop, so the sums are the same to the last bit.
    __shared__ double red[18][8][6];
    __shared__ float feat[108];
    const int pair = blockIdx.x, tid = threadIdx.x;
    for (int i = tid; i < 108; i += 256) feat[i] = 0.f;
    for (int s = 0; s < segs_per_pair; s++) {
        const MapSeg& sg = segs[pair * segs_per_pair + s];
        const int64_t begin = sg.tile_begin, ntiles = sg.ntiles;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        // Unrolled so that several tiles' loads are in flight; the additions stay in tile order.
#pragma unroll 4
        for (int t = tid; t < ntiles; t += 256) {
            const double* p = partials + (begin + t) * 6;
#pragma unroll
            for (int k = 0; k < 6; k++) acc[k] += p[k];
        }
#pragma unroll
        for (int k = 0; k < 6; k++) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
        }
        if ((tid & 31) == 0) {
#pragma unroll
            for (int k = 0; k < 6; k++) red[s][tid >> 5][k] = acc[k];
        }
    }
    __syncthreads();
    if (tid < 3 * segs_per_pair) {
        const int s = tid / 3, m = tid - 3 * s;
        const MapSeg& sg = segs[pair * segs_per_pair + s];
        const double n = (double)sg.w * (double)sg.h;
        double s1 = 0.0, s4 = 0.0;
        for (int w = 0; w < 8; w++) { s1 += red[s][w][m]; s4 += red[s][w][3 + m]; }
        const bool on = (sg.on >> m) & 1;
        feat[sg.slot + m] = on ? (float)(s1 / n) : 0.f;
        feat[sg.slot + 3 + m] = on ? (float)sqrt(sqrt(s4 / n)) : 0.f;
    }
    __syncthreads();
    if (features)
        for (int i = tid; i < 108; i += 256) features[(int64_t)pair * 108 + i] = feat[i];
    if (tid == 0) scores[pair] = score_from_features(feat);
}

// ------------------------------------------------------------------------------------------
// Engine
// ------------------------------------------------------------------------------------------

// Launches the front kernel on raw inputs, specialised when both clips share a fast format.
static void launch_front(const FrontArgs& fa, const ColourParams cp[2], dim3 grid, cudaStream_t st, KernelTimer* timer) {
    const int smem = (int)sizeof(float) * std::max(chroma_stage_floats(cp[0].subw, cp[0].subh),
                                                   chroma_stage_floats(cp[1].subw, cp[1].subh));
    const int f0 = fast_path_of(cp[0]), f1 = fast_path_of(cp[1]);
    const int fast = f0 == f1 ? f0 : kFastGeneric;
    auto kern = fast == kFastYuv420Bt709 ? ssimu2_front_kernel<false, kFastYuv420Bt709>
              : fast == kFastRgb8Srgb ? ssimu2_front_kernel<false, kFastRgb8Srgb>
                                      : ssimu2_front_kernel<false, kFastGeneric>;
    if (smem > 32 * 1024) CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int t = timer ? timer->begin(0, "ssimu2_front", st) : -1;
    kern<<<grid, 256, smem, st>>>(fa);
    CUDA_CHECK(cudaGetLastError());
    if (timer) timer->end(t, st);
}

// Work-list template of one pair for the maps kernel (same order as the per-pair segments
// of build_segments, which the final kernel walks).
static MapTemplate make_map_template(const Pyramid& pyr, const float* xyb) {
    MapTemplate mt{};
    int tile = 0;
    for (int s = 0; s < kScales; s++)
        for (int p = 0; p < 3; p++) {
            if (!plane_needed(p, s)) continue;
            MapTemplate::Seg& g = mt.seg[mt.nseg++];
            g.off = pyr.off[s][p];
            g.w = pyr.w[s];
            g.h = pyr.h[s];
            g.pitch = pyr.pitch[s];
            g.tiles_x = (int)ceil_div(g.w, kTile);
            g.tile_begin = tile;
            tile += g.tiles_x * (int)ceil_div(g.h, kTile);
        }
    mt.tiles_per_pair = tile;
    mt.xyb = xyb;
    mt.image_floats = pyr.image_floats;
    return mt;
}

class Engine final : public Ssimu2Api {
public:
    ~Engine() override { release(); }

    void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, int device) override {
        device_ = device;
        cs_[0] = src;
        cs_[1] = dis;
        geo_[0] = make_geometry(src);
        geo_[1] = make_geometry(dis);
        if (geo_[0].OW != geo_[1].OW || geo_[0].OH != geo_[1].OH)
            VSHIP_THROW(Vship_DifferingInputType, "");
        width_ = (int)geo_[0].OW;
        height_ = (int)geo_[0].OH;
        for (int c = 0; c < 2; c++) cp_[c] = make_colour_params(cs_[c], geo_[c], false);
        generic_ = geo_[0].generic() || geo_[1].generic();
        build_pyramid();
        CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        CUDA_CHECK(cudaEventCreateWithFlags(&last_done_, cudaEventDisableTiming));
        upload_gauss_constants();
        for (int c = 0; c < 2; c++) {
            int64_t off[3];
            staging_[c].ensure((size_t)dense_image_bytes(geo_[c], off), stream_);
            if (generic_) lin_[c].alloc(geo_[c]);
        }
        score_host_ = pinned_alloc<double>(1, "score");
        int sms = 0, per_sm = 0;
        CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ssimu2_maps_kernel, kMapThreads, 0));
        maps_grid_ = std::max(1, sms * std::max(1, per_sm));
        ensure_capacity(1);
    }

    double compute(const uint8_t* const s1[3], const uint8_t* const s2[3], const int64_t ls1[3], const int64_t ls2[3]) override {
        CUDA_CHECK(cudaStreamWaitEvent(stream_, last_done_, 0));
        RawImage raw[2];
        ColourParams cp[2] = {cp_[0], cp_[1]};
        for (int c = 0; c < 2; c++) {
            raw[c] = stage_host_image(staging_[c], geo_[c], c ? s2 : s1, c ? ls2 : ls1, stream_);
            cp[c].misaligned = misaligned_view(raw[c], geo_[c]) ? 1 : 0;
        }
        run_pairs(1, raw, cp, stream_, scores_d_, features_d_);
        CUDA_CHECK(cudaMemcpyAsync(score_host_, scores_d_, sizeof(double), cudaMemcpyDeviceToHost, stream_));
        CUDA_CHECK(cudaMemcpyAsync(last_features_, features_d_, sizeof(float) * 108, cudaMemcpyDeviceToHost, stream_));
        CUDA_CHECK(cudaEventRecord(last_done_, stream_));
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        return *score_host_;
    }

    void compute_device(int n, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t ls1[3],
                        const int64_t ls2[3], double* d_scores, float* d_features, cudaStream_t stream) override {
        if (n <= 0) return;
        if (generic_ && n > 1) {
            for (int i = 0; i < n; i++)
                compute_device(1, d1 + 3 * i, d2 + 3 * i, ls1, ls2, d_scores ? d_scores + i : nullptr,
                               d_features ? d_features + (int64_t)i * 108 : nullptr, stream);
            return;
        }
        ColourParams cp[2] = {cp_[0], cp_[1]};
        for (int c = 0; c < 2; c++) {
            const int64_t* ls = c ? ls2 : ls1;
            const uint8_t* const* src = c ? d2 : d1;
            for (int p = 0; p < 3; p++)
                if (ls[p] < geo_[c].pw[p] * geo_[c].bytes) VSHIP_THROW(Vship_BadPointer, "lineSize smaller than one row of samples");
            // the colour parameters are shared by the launch: one unaligned plane of any pair
            // (stride or address) switches that clip to byte loads
            for (int i = 0; i < n && !cp[c].misaligned; i++)
                if (misaligned_planes(src + 3 * i, ls, geo_[c].bytes)) cp[c].misaligned = 1;
        }
        cudaStream_t st = stream;  // NULL: the CUDA legacy default stream
        CUDA_CHECK(cudaStreamWaitEvent(st, last_done_, 0));
        std::vector<RawImage> raw(2 * kMaxBatch);
        int done = 0;
        while (done < n) {
            const int chunk = std::min(n - done, kMaxBatch);
            ensure_capacity(chunk);
            for (int i = 0; i < chunk; i++)
                for (int c = 0; c < 2; c++) {
                    const uint8_t* const* src = c ? d2 : d1;
                    const int64_t* ls = c ? ls2 : ls1;
                    for (int p = 0; p < 3; p++) {
                        if (src[3 * (done + i) + p] == nullptr) VSHIP_THROW(Vship_BadPointer, "null plane pointer");
                        raw[2 * i + c].p[p] = src[3 * (done + i) + p];
                        raw[2 * i + c].stride[p] = ls[p];
                    }
                }
            run_pairs(chunk, raw.data(), cp, st, d_scores ? d_scores + done : scores_d_,
                      d_features ? d_features + (int64_t)done * 108 : features_d_);
            done += chunk;
        }
        CUDA_CHECK(cudaEventRecord(last_done_, st));
    }

    void last_features(float out[108]) override { std::memcpy(out, last_features_, sizeof(last_features_)); }
    KernelTimer& timer() override { return timer_; }
    int width() const override { return width_; }
    int height() const override { return height_; }

private:
    void build_pyramid() {
        pyr_ = make_pyramid(width_, height_);
        tiles_per_pair_ = 0;
        segs_per_pair_ = 0;
        for (int s = 0; s < kScales; s++)
            for (int p = 0; p < 3; p++)
                if (plane_needed(p, s)) {
                    tiles_per_pair_ += (int)(ceil_div(pyr_.w[s], kTile) * ceil_div(pyr_.h[s], kTile));
                    segs_per_pair_++;
                }
    }

    // Work list of the map kernel for `npairs` pairs stored at the start of xyb_.
    std::vector<MapSeg> build_segments(int npairs) const {
        std::vector<MapSeg> segs;
        int tile = 0;
        for (int pr = 0; pr < npairs; pr++) {
            for (int s = 0; s < kScales; s++) {
                for (int p = 0; p < 3; p++) {
                    int on = 0;
                    for (int m = 0; m < 3; m++) on |= (map_on(p, s, m) ? 1 : 0) << m;
                    if (!on) continue;
                    MapSeg g{};
                    g.a = xyb_ + (int64_t)(2 * pr) * pyr_.image_floats + pyr_.off[s][p];
                    g.b = xyb_ + (int64_t)(2 * pr + 1) * pyr_.image_floats + pyr_.off[s][p];
                    g.w = pyr_.w[s];
                    g.h = pyr_.h[s];
                    g.pitch = pyr_.pitch[s];
                    g.tiles_x = (int)ceil_div(g.w, kTile);
                    g.ntiles = g.tiles_x * (int)ceil_div(g.h, kTile);
                    g.tile_begin = tile;
                    g.slot = p * 36 + s * 6;
                    g.on = on;
                    tile += g.ntiles;
                    segs.push_back(g);
                }
            }
        }
        return segs;
    }

    // Grows the batch buffers and rebuilds the work list for kMaxBatch pairs.  The work list
    // of the first n pairs is a prefix of it, so every batch size shares one table.
    void ensure_capacity(int npairs) {
        if (npairs <= cap_) return;
        const int ncap = npairs <= 1 ? 1 : kMaxBatch;
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        device_free(xyb_);
        device_free(partials_);
        device_free(segs_d_);
        device_free(scores_d_);
        device_free(features_d_);
        xyb_ = nullptr; partials_ = nullptr; segs_d_ = nullptr; scores_d_ = nullptr; features_d_ = nullptr;
        xyb_ = device_alloc<float>((size_t)(2 * ncap * pyr_.image_floats), "XYB pyramid");
        partials_ = device_alloc<double>((size_t)tiles_per_pair_ * 6 * ncap, "tile partials");
        segs_d_ = device_alloc<MapSeg>((size_t)segs_per_pair_ * ncap, "map work list");
        scores_d_ = device_alloc<double>((size_t)ncap, "scores");
        features_d_ = device_alloc<float>((size_t)108 * ncap, "features");
        const std::vector<MapSeg> segs = build_segments(ncap);
        CUDA_CHECK(cudaMemcpy(segs_d_, segs.data(), segs.size() * sizeof(MapSeg), cudaMemcpyHostToDevice));
        map_template_ = make_map_template(pyr_, xyb_);
        cap_ = ncap;
    }

    void run_pairs(int npairs, const RawImage* raw, const ColourParams cp[2], cudaStream_t st,
                   double* scores_d, float* features_d) {
        const int nimg = 2 * npairs;
        FrontArgs* fa = &front_args_;
        fa->cp[0] = cp[0];
        fa->cp[1] = cp[1];
        fa->xyb = xyb_;
        fa->pyr = pyr_;
        for (int i = 0; i < nimg; i++) fa->raw[i] = raw[i];
        const dim3 fgrid((unsigned)ceil_div(pyr_.w[1], 32), (unsigned)ceil_div(pyr_.h[1], 32), (unsigned)nimg);
        if (!generic_) {
            launch_front(*fa, cp, fgrid, st, &timer_);
        } else {
            // Resize/crop path (one pair): planar linear RGB first, then the pyramid reads the
            // crop window of each clip.
            for (int c = 0; c < 2; c++) {
                lin_[c].run(raw[c], cp[c], geo_[c], st);
                fa->lin[c] = lin_[c].planes + (int64_t)geo_[c].crop_top * geo_[c].TW + geo_[c].crop_left;
                fa->lin_plane[c] = geo_[c].TW * geo_[c].TH;
                fa->lin_pitch[c] = geo_[c].TW;
            }
            ssimu2_front_kernel<true, kFastGeneric><<<fgrid, 256, 0, st>>>(*fa);
            CUDA_CHECK(cudaGetLastError());
        }
        const int ntiles = tiles_per_pair_ * npairs;
        const int t1 = timer_.begin(1, "ssimu2_maps", st);
        ssimu2_maps_kernel<<<(unsigned)std::min(ntiles, maps_grid_), kMapThreads, 0, st>>>(map_template_, ntiles, partials_);
        CUDA_CHECK(cudaGetLastError());
        timer_.end(t1, st);
        const int t2 = timer_.begin(2, "ssimu2_final", st);
        ssimu2_final_kernel<<<(unsigned)npairs, 256, 0, st>>>(segs_d_, segs_per_pair_, partials_, scores_d, features_d);
        CUDA_CHECK(cudaGetLastError());
        timer_.end(t2, st);
    }

    void release() {
        if (stream_) (void)cudaStreamSynchronize(stream_);
        timer_.destroy();
        for (int c = 0; c < 2; c++) {
            staging_[c].free();
            lin_[c].free();
        }
        device_free(xyb_);
        device_free(partials_);
        device_free(segs_d_);
        device_free(scores_d_);
        device_free(features_d_);
        pinned_free(score_host_);
        xyb_ = nullptr; partials_ = nullptr; segs_d_ = nullptr; scores_d_ = nullptr; features_d_ = nullptr;
        score_host_ = nullptr;
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
    Vship_Colorspace_t cs_[2];
    ClipGeometry geo_[2];
    ColourParams cp_[2];
    bool generic_ = false;
    Pyramid pyr_{};
    int tiles_per_pair_ = 0, segs_per_pair_ = 0;
    int width_ = 0, height_ = 0;
    cudaStream_t stream_ = nullptr;
    StagingBuffer staging_[2];
    GenericLinear lin_[2];
    float* xyb_ = nullptr;
    double* partials_ = nullptr;
    MapSeg* segs_d_ = nullptr;
    double* scores_d_ = nullptr;
    float* features_d_ = nullptr;
    double* score_host_ = nullptr;
    float last_features_[108] = {};
    int cap_ = 0;
    FrontArgs front_args_{};
    MapTemplate map_template_{};
    int maps_grid_ = 0;
    cudaEvent_t last_done_ = nullptr;  // completion of the previous call, on whichever stream it ran
    KernelTimer timer_;
};

// ------------------------------------------------------------------------------------------
// Allocation-free scoring (VshipExt_ComputeSSIMU2NoAlloc)
//
// Some callers cannot call cudaMalloc: a process whose GPU memory is handed out up front by a
// fixed budget or pool (an allocation outside it fails or steals from another component), or
// a real-time loop that must not reach the driver's allocator, whose calls can block for
// milliseconds and synchronise the device.  For them this entry point
// scores one pair already in device memory with the same three kernels as the handler path,
// but with all of its scratch -- both XYB pyramids, the tile partials and the map work list
// -- in the file-scope array below.  The array is part of the library image: every GPU that
// loads the library holds its 32 MiB until the process exits.
// ------------------------------------------------------------------------------------------

constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 1920x1200 frames fit
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_lock;
static unsigned char* g_noalloc_base[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device.  The first call on a device
// resolves it with cudaGetSymbolAddress (the host-side name is only a stand-in for the
// device array) and loads the blur constants; later calls reuse the cached address.  The
// cache lives as long as the process: after cudaDeviceReset the address and the constants
// belong to a destroyed context, so the entry point must not be used on that device again.
static unsigned char* noalloc_scratch_for_current_device() {
    int dev = -1;
    CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        VSHIP_THROW(Vship_BadDeviceArgument, "device index beyond the no-allocation table");
    std::lock_guard<std::mutex> g(g_noalloc_lock);
    if (g_noalloc_base[dev] == nullptr) {
        void* ptr = nullptr;
        CUDA_CHECK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        upload_gauss_constants();
        g_noalloc_base[dev] = static_cast<unsigned char*>(ptr);
    }
    return g_noalloc_base[dev];
}

// The work list of one pair travels as kernel parameters and is stored into the scratch
// array on the device, so the entry point issues no copy from host memory.
struct SegList {
    MapSeg s[18];
};

__global__ void noalloc_store_segments_kernel(const __grid_constant__ SegList list, MapSeg* dst, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = list.s[i];
}

static void compute_no_alloc(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, double* d_score,
                             float* d_features, const uint8_t* const d1[3], const uint8_t* const d2[3],
                             const int64_t ls1[3], const int64_t ls2[3], cudaStream_t st) {
    if (!d_score || !d1 || !d2 || !ls1 || !ls2) VSHIP_THROW(Vship_BadPointer, "NULL argument");
    ClipGeometry geo[2] = {make_geometry(src), make_geometry(dis)};
    if (geo[0].OW != geo[1].OW || geo[0].OH != geo[1].OH) VSHIP_THROW(Vship_DifferingInputType, "");
    if (geo[0].generic() || geo[1].generic())
        VSHIP_THROW(Vship_BadErrorType, "resize and crop need per-handler buffers: use a handler");
    const Vship_Colorspace_t* cs[2] = {&src, &dis};
    ColourParams cp[2];
    for (int c = 0; c < 2; c++) {
        const int64_t* ls = c ? ls2 : ls1;
        const uint8_t* const* d = c ? d2 : d1;
        for (int p = 0; p < 3; p++) {
            if (d[p] == nullptr) VSHIP_THROW(Vship_BadPointer, "null plane pointer");
            if (ls[p] < geo[c].pw[p] * geo[c].bytes) VSHIP_THROW(Vship_BadPointer, "lineSize smaller than one row of samples");
        }
        cp[c] = make_colour_params(*cs[c], geo[c], misaligned_planes(d, ls, geo[c].bytes));
    }

    // Pyramid layout, tile count and work list of one pair, as the handler path builds them.
    Pyramid pyr{};
    int w = (int)geo[0].OW, h = (int)geo[0].OH;
    int64_t off = 0;
    for (int s = 0; s < kScales; s++) {
        pyr.w[s] = w;
        pyr.h[s] = h;
        pyr.pitch[s] = (int)round_up(w, 8);
        for (int p = 0; p < 3; p++) {
            if (plane_needed(p, s) || (s == 0 && p == 1)) {
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
    const size_t xyb_bytes = (size_t)(2 * pyr.image_floats) * sizeof(float);
    int ntiles = 0, nsegs = 0;
    for (int s = 0; s < kScales; s++)
        for (int p = 0; p < 3; p++)
            if (plane_needed(p, s)) {
                ntiles += (int)(ceil_div(pyr.w[s], kTile) * ceil_div(pyr.h[s], kTile));
                nsegs++;
            }
    const size_t part_off = round_up((int64_t)xyb_bytes, 256);
    const size_t seg_off = round_up((int64_t)(part_off + (size_t)ntiles * 6 * sizeof(double)), 256);
    const size_t need = seg_off + (size_t)nsegs * sizeof(MapSeg);
    if (need > kNoAllocScratchBytes)
        VSHIP_THROW(Vship_OutOfVRAM, "frame needs " + std::to_string(need) + " bytes of scratch; the no-allocation entry point has " +
                                         std::to_string(kNoAllocScratchBytes));

    unsigned char* base = noalloc_scratch_for_current_device();
    float* xyb = reinterpret_cast<float*>(base);
    double* partials = reinterpret_cast<double*>(base + part_off);
    MapSeg* segs_d = reinterpret_cast<MapSeg*>(base + seg_off);

    SegList list{};
    MapSeg* segs = list.s;
    int tile = 0, k = 0;
    for (int s = 0; s < kScales; s++)
        for (int p = 0; p < 3; p++) {
            int on = 0;
            for (int m = 0; m < 3; m++) on |= (map_on(p, s, m) ? 1 : 0) << m;
            if (!on) continue;
            MapSeg& g = segs[k++];
            g = MapSeg{};
            g.a = xyb + pyr.off[s][p];
            g.b = xyb + pyr.image_floats + pyr.off[s][p];
            g.w = pyr.w[s];
            g.h = pyr.h[s];
            g.pitch = pyr.pitch[s];
            g.tiles_x = (int)ceil_div(g.w, kTile);
            g.ntiles = g.tiles_x * (int)ceil_div(g.h, kTile);
            g.tile_begin = tile;
            g.slot = p * 36 + s * 6;
            g.on = on;
            tile += g.ntiles;
        }
    noalloc_store_segments_kernel<<<1, 32, 0, st>>>(list, segs_d, nsegs);
    CUDA_CHECK(cudaGetLastError());

    static FrontArgs fa;  // 6.6 KB of kernel arguments, kept off the caller's stack
    static std::mutex fa_lock;
    std::lock_guard<std::mutex> g(fa_lock);
    fa = FrontArgs{};
    fa.cp[0] = cp[0];
    fa.cp[1] = cp[1];
    fa.xyb = xyb;
    fa.pyr = pyr;
    for (int c = 0; c < 2; c++)
        for (int p = 0; p < 3; p++) {
            fa.raw[c].p[p] = (c ? d2 : d1)[p];
            fa.raw[c].stride[p] = (c ? ls2 : ls1)[p];
        }
    const dim3 fgrid((unsigned)ceil_div(pyr.w[1], 32), (unsigned)ceil_div(pyr.h[1], 32), 2u);
    launch_front(fa, cp, fgrid, st, nullptr);
    const MapTemplate mt = make_map_template(pyr, xyb);
    int sms = 0, per_sm = 0, dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ssimu2_maps_kernel, kMapThreads, 0));
    ssimu2_maps_kernel<<<(unsigned)std::min(ntiles, std::max(1, sms * per_sm)), kMapThreads, 0, st>>>(mt, ntiles, partials);
    CUDA_CHECK(cudaGetLastError());
    ssimu2_final_kernel<<<1, 256, 0, st>>>(segs_d, nsegs, partials, d_score, d_features);
    CUDA_CHECK(cudaGetLastError());
}

}  // namespace ssimu2

Ssimu2Api* make_ssimu2_engine() { return new ssimu2::Engine(); }

}  // namespace vship

extern "C" Vship_Exception VshipExt_ComputeSSIMU2NoAlloc(Vship_Colorspace_t src_colorspace, Vship_Colorspace_t dis_colorspace,
                                                         double* d_score, float* d_features, const uint8_t* const srcp1[3],
                                                         const uint8_t* const srcp2[3], const int64_t lineSize[3],
                                                         const int64_t lineSize2[3], void* stream) {
    try {
        vship::ssimu2::compute_no_alloc(src_colorspace, dis_colorspace, d_score, d_features, srcp1, srcp2, lineSize, lineSize2,
                                        (cudaStream_t)stream);
    } catch (const vship::Error& e) {
        vship::record_global_error(e);
        return e.code;
    } catch (const std::bad_alloc&) {
        vship::Error e(Vship_OutOfRAM, __FILE__, __LINE__, "VshipExt_ComputeSSIMU2NoAlloc");
        vship::record_global_error(e);
        return e.code;
    } catch (const std::exception& ex) {
        vship::Error e(Vship_BadErrorType, __FILE__, __LINE__, ex.what());
        vship::record_global_error(e);
        return e.code;
    }
    return Vship_NoError;
}

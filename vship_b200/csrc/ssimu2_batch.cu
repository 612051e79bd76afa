// SSIMULACRA2 over uneven batches: frame pairs of any resolutions and formats scored by one
// CUDA graph launch.  No counterpart in the reference, which scores one pair per call on a
// handler bound to one colourspace pair (src/ssimu2/main.hpp:80-156).
//
// The graph copies the batch's descriptors, clears the per-pair counters and runs two
// kernels over flat work lists that span every pair of the batch:
//
//   ssimu2_batch_front_kernel  one CTA per front tile of every image (raw planes -> linear RGB
//                              -> pyramid -> XYB, the per-handler front tile), which then
//                              counts the tile on its pair's counter
//   ssimu2_batch_tiles_kernel  one thread per map tile: the tile table (plane, position,
//                              size, partial slot) the map kernel reads instead of searching
//                              the descriptors
//   ssimu2_batch_maps_kernel   persistent: CTA b scores map tiles b, b + grid, ... of the
//                              list of every pair's tiles (blur, SSIM / artifact / detail-loss
//                              maps, per-tile sums: the per-handler map tile)
//   ssimu2_batch_final_kernel  one CTA per pair: features and score from the tile sums
//
// The map kernel depends on the front grid through a programmatic edge from its
// launch-completion port: it starts once every front CTA has begun, so its CTAs take over
// the front grid's last wave, and a map tile whose pair still has front tiles in flight
// waits for them (bounded in time) on the pair's counter.  Every front tile is then held by
// a running CTA that waits on nothing, and map tiles wait only on front tiles, so every wait
// ends; a wait that runs out sets an error word that the host reports.  Front CTAs run at
// the front code's own occupancy (256 threads, few registers), map CTAs at the map code's
// (128 threads, register-prefetched halos).  A fused single kernel was measured 1.6x
// slower: it runs the front tiles at the map code's register budget.
//
// The map tile height (16, 32 or 64 rows of 32 columns) trades halo overhead against shared
// memory and registers; the engine picks it by timing each on the batch, and keeps the
// choice per device and mix of resolutions in memory and in a JSON file.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#include <sys/stat.h>

#include "common.cuh"
#include "colour.cuh"
#include "frontend.cuh"
#include "metric_tables.h"
#include "ssimu2_device.cuh"
#include "engines.h"

namespace vship {
namespace ssimu2 {
namespace {

constexpr int kBatchMaxClasses = 16;     // distinct colourspace pairs per launch
constexpr int kBatchMaxPairs = 4096;     // pairs per launch
constexpr long long kWaitLimitNs = 2000000000LL;  // a dependency wait gives up after 2 s
constexpr unsigned kErrWaitTimeout = 1u;

// One unpruned (plane, scale) of a class: tiles of 32 x TH outputs.
struct BatchSeg {
    int64_t off;          // float offset of the plane in an image's pyramid
    int w, h, pitch;
    int tiles_x, tile_begin, ntiles;
    int slot;             // plane * 36 + scale * 6
    int on;               // bit k set: map k is unpruned
};

// Pairs sharing both colourspaces and the alignment of their sample views.
struct BatchClass {
    ColourParams cp[2];
    Pyramid pyr;
    int ftx, fty;         // front tiles (32 x 32 of level 1) per image
    int front_items;      // 2 * ftx * fty
    int tiles_per_pair;   // map tiles per pair
    int fast;             // front path of both clips
    int nseg;
    BatchSeg seg[18];
};

struct BatchPair {
    RawImage raw[2];
    int64_t xyb;          // float offset of the reference pyramid; the distorted one follows
    int64_t partial;      // first tile partial (6 doubles each)
    int cls;
};

// Header of the descriptor block copied to the device before each launch.  Both work lists
// are class-major: class c owns front items [front_start[c], front_start[c + 1]) and map
// tiles [maps_start[c], maps_start[c + 1]), pair by pair in the order of class_pairs.
struct BatchView {
    const BatchClass* cls;
    const BatchPair* pairs;
    const int* class_pairs;   // [npairs] pair indices grouped by class
    int nclasses, npairs;
    int front_total, maps_total;
    int pair_start[kBatchMaxClasses + 1];   // first class_pairs entry of each class
    int front_start[kBatchMaxClasses + 1];
    int maps_start[kBatchMaxClasses + 1];
    float* xyb;
    double* partials;
    double* scores;
    float* features;          // may be null
    uint4* tiles;             // [2 * maps_total] per map tile, written by ssimu2_batch_tiles_kernel
    unsigned* counters;       // [0] error (sticky), [1] front tiles done in all, [2, 2 + n) front tiles done
                              // per pair, then map tiles done per pair
};

// What a front CTA reads, passed as the kernel's parameter so that the colour parameters and
// pyramid geometry of its class come from the constant bank.
struct FrontParams {
    ColourParams cp[kBatchMaxClasses][2];
    Pyramid pyr[kBatchMaxClasses];
    int ftx[kBatchMaxClasses], fty[kBatchMaxClasses], fast[kBatchMaxClasses];
    int front_start[kBatchMaxClasses + 1];
    int pair_start[kBatchMaxClasses + 1];
    int nclasses;
    const int* class_pairs;
    const BatchPair* pairs;
    float* xyb;
    unsigned* counters;
};

// Class of work item x of a class-major list (start has nclasses + 1 entries).
__device__ __forceinline__ int class_of(const int* start, int nclasses, int x) {
    int c = 0;
    while (c + 1 < nclasses && x >= start[c + 1]) c++;
    return c;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Release-only counter update: it orders this CTA's earlier writes (made visible to thread 0
// by a barrier) before the increment without the acquire half of a full fence.
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ long long globaltimer_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Thread 0: waits until *ctr >= need.  Returns early (false) once the launch's error word is
// set, and sets it itself after kWaitLimitNs.
__device__ bool wait_at_least(const unsigned* ctr, unsigned need, unsigned* err) {
    if (ld_acquire(ctr) >= need) return true;
    const long long t0 = globaltimer_ns();
    for (;;) {
        __nanosleep(256);
        if (ld_acquire(ctr) >= need) return true;
        if (ld_acquire(err) != 0u) return false;
        if (globaltimer_ns() - t0 > kWaitLimitNs) {
            atomicCAS(err, 0u, kErrWaitTimeout);
            return false;
        }
    }
}

// One front tile per CTA.  kPath is the front path of every class of the launch, or -1 when
// the launch mixes paths (each CTA then follows its class's).
template <int kPath>
__global__ void __launch_bounds__(256, kPath == kFastRgb8Srgb || kPath == kFastYuv420Bt709 ? 5 : 4)
    ssimu2_batch_front_kernel(const __grid_constant__ FrontParams fp) {
    __shared__ FrontSmem fs;
    extern __shared__ __align__(16) float stage[];
    const int item = blockIdx.x;
    const int c = class_of(fp.front_start, fp.nclasses, item);
    const int per_img = fp.ftx[c] * fp.fty[c];
    const int rel = item - fp.front_start[c];
    const int k = rel / (2 * per_img);
    int local = rel - k * 2 * per_img;
    const int clip = local >= per_img ? 1 : 0;
    local -= clip * per_img;
    const int ty = local / fp.ftx[c], tx = local - ty * fp.ftx[c];
    const int p = __ldg(fp.class_pairs + fp.pair_start[c] + k);
    const BatchPair& bp = fp.pairs[p];
    const RawImage im = bp.raw[clip];
    const ColourParams& cp = fp.cp[c][clip];
    const Pyramid& pyr = fp.pyr[c];
    float* out = fp.xyb + bp.xyb + (int64_t)clip * pyr.image_floats;
    const LinearIn lin{};
    const int path = kPath >= 0 ? kPath : fp.fast[c];
    if (path == kFastRgb8Srgb)
        front_tile<false, kPath < 0 ? kFastRgb8Srgb : kPath>(fs, stage, cp, im, lin, pyr, out, tx, ty);
    else if (kPath < 0 && path == kFastYuv420Bt709)
        front_tile<false, kFastYuv420Bt709>(fs, stage, cp, im, lin, pyr, out, tx, ty);
    else if (kPath < 0)
        front_tile<false, kFastGeneric>(fs, stage, cp, im, lin, pyr, out, tx, ty);
    else
        front_tile<false, kPath>(fs, stage, cp, im, lin, pyr, out, tx, ty);
    __syncthreads();
    if (threadIdx.x == 0) {
        red_release_add(fp.counters + 2 + p, 1u);
        red_release_add(fp.counters + 1, 1u);
    }
}

// The tile table: one 32-byte entry per map tile of the launch,
//   [0].x = float offset of the reference plane in the pyramid buffer / 64
//   [0].y = tile column | tile row << 16
//   [0].z = partial slot
//   [0].w = pair
//   [1]   = plane width, height, pitch, image floats / 64
// so that a map CTA locates a tile with two independent loads issued a tile ahead instead
// of searching the descriptors.  Plane offsets are multiples of 64 floats (pyramid planes
// and images are 64-float aligned).
__global__ void __launch_bounds__(256) ssimu2_batch_tiles_kernel(const BatchView* __restrict__ vp) {
    const int m = blockIdx.x * 256 + threadIdx.x;
    if (m >= vp->maps_total) return;
    const int c = class_of(vp->maps_start, vp->nclasses, m);
    const BatchClass& bc = vp->cls[c];
    const int rel = m - vp->maps_start[c];
    const int k = rel / bc.tiles_per_pair;
    const int l = rel - k * bc.tiles_per_pair;
    const int p = vp->class_pairs[vp->pair_start[c] + k];
    const BatchPair& bp = vp->pairs[p];
    int s = 0;
    for (int i = 1; i < bc.nseg; i++)
        if (bc.seg[i].tile_begin <= l) s = i;
    const BatchSeg& g = bc.seg[s];
    const int lt = l - g.tile_begin;
    const int ty = lt / g.tiles_x;
    uint4 e0, e1;
    e0.x = (unsigned)((bp.xyb + g.off) >> 6);
    e0.y = (unsigned)(lt - ty * g.tiles_x) | ((unsigned)ty << 16);
    e0.z = (unsigned)(bp.partial + l);
    e0.w = (unsigned)p;
    e1.x = (unsigned)g.w;
    e1.y = (unsigned)g.h;
    e1.z = (unsigned)g.pitch;
    e1.w = (unsigned)(bc.pyr.image_floats >> 6);
    vp->tiles[2 * (int64_t)m] = e0;
    vp->tiles[2 * (int64_t)m + 1] = e1;
}

template <int TH>
__device__ __forceinline__ TileRef unpack_tile(const BatchView& v, uint4 e0, uint4 e1) {
    TileRef t;
    t.a = v.xyb + ((int64_t)e0.x << 6);
    t.b = t.a + ((int64_t)e1.w << 6);
    t.w = (int)e1.x;
    t.h = (int)e1.y;
    t.pitch = (int)e1.z;
    t.X0 = (int)(e0.y & 0xffffu) * kTile;
    t.Y0 = (int)(e0.y >> 16) * TH;
    return t;
}

constexpr int kFinalThreads = 256;

// Per pair: FP64 totals of the tile partials, the 108 features and the score (the
// per-handler final kernel's reduction over the pair's segments).
__global__ void __launch_bounds__(kFinalThreads) ssimu2_batch_final_kernel(const BatchView* __restrict__ vp) {
    // As the per-handler final kernel: per-segment warp sums in shared memory, one barrier,
    // one thread per (segment, map); the additions keep the segment-by-segment order.
    __shared__ double red[18][kFinalThreads / 32][6];
    __shared__ float feat[108];
    const int p = blockIdx.x, tid = threadIdx.x;
    const BatchPair& bp = vp->pairs[p];
    const BatchClass& bc = vp->cls[bp.cls];
    for (int i = tid; i < 108; i += kFinalThreads) feat[i] = 0.f;
    for (int s = 0; s < bc.nseg; s++) {
        const BatchSeg& g = bc.seg[s];
        double acc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 4
        for (int t = tid; t < g.ntiles; t += kFinalThreads) {
            const double* q = vp->partials + (bp.partial + g.tile_begin + t) * 6;
#pragma unroll
            for (int k = 0; k < 6; k++) acc[k] += q[k];
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
    if (tid < 3 * bc.nseg) {
        const int s = tid / 3, m = tid - 3 * s;
        const BatchSeg& g = bc.seg[s];
        const double n = (double)g.w * (double)g.h;
        double s1 = 0.0, s4 = 0.0;
        for (int wi = 0; wi < kFinalThreads / 32; wi++) { s1 += red[s][wi][m]; s4 += red[s][wi][3 + m]; }
        const bool on = (g.on >> m) & 1;
        feat[g.slot + m] = on ? (float)(s1 / n) : 0.f;
        feat[g.slot + 3 + m] = on ? (float)sqrt(sqrt(s4 / n)) : 0.f;
    }
    __syncthreads();
    if (vp->features)
        for (int i = tid; i < 108; i += kFinalThreads) vp->features[(int64_t)p * 108 + i] = feat[i];
    if (tid == 0) vp->scores[p] = score_from_features(feat);
}

// Tracks, per thread, which pyramids its halo loads may read: a pair is checked with an
// acquire load the first time the thread meets it, and all checks stop once every front
// tile of the launch is counted.
struct FrontGate {
    int ok_pair = -1;
    bool all = false;
    // Non-blocking: true when pair p's front tiles are all counted.
    __device__ __forceinline__ bool ready(const BatchView& v, int p) {
        if (all || p == ok_pair) return true;
        if (ld_acquire(v.counters + 1) >= (unsigned)v.front_total) {
            all = true;
            return true;
        }
        if (ld_acquire(v.counters + 2 + p) >= (unsigned)v.cls[v.pairs[p].cls].front_items) {
            ok_pair = p;
            return true;
        }
        return false;
    }
    // Blocking (bounded): waits for pair p's front tiles.
    __device__ __forceinline__ void wait(const BatchView& v, int p) {
        if (ready(v, p)) return;
        wait_at_least(v.counters + 2 + p, (unsigned)v.cls[v.pairs[p].cls].front_items, v.counters);
        ok_pair = p;
    }
};

// Persistent: CTA b scores map tiles b, b + gridDim.x, ... from the tile table, with the
// next tile's entry loaded a tile ahead and its halo prefetched into registers once its
// pair's front tiles are all counted.
template <int TH>
__global__ void __launch_bounds__(kMapThreads, TH == 64 ? 3 : 4) ssimu2_batch_maps_kernel(const BatchView* __restrict__ vp) {
    using MT = MapTile<TH>;
    extern __shared__ __align__(16) unsigned char dyn[];
    typename MT::Smem& sm = *reinterpret_cast<typename MT::Smem*>(dyn);
    __shared__ BatchView v;
    if (threadIdx.x == 0) v = *vp;
    __syncthreads();
    const int total = v.maps_total;
    const int stride = gridDim.x;
    int m = blockIdx.x;
    if (m >= total) return;
    FrontGate gate;
    const uint4* tiles = v.tiles;
    uint4 e0 = __ldg(tiles + 2 * (int64_t)m), e1 = __ldg(tiles + 2 * (int64_t)m + 1);
    uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
    if (m + stride < total) {
        n0 = __ldg(tiles + 2 * (int64_t)(m + stride));
        n1 = __ldg(tiles + 2 * (int64_t)(m + stride) + 1);
    }
    TileRef cur = unpack_tile<TH>(v, e0, e1);
    int pair = (int)e0.w;
    unsigned partial = e0.z;
    gate.wait(v, pair);
    HaloV4T<TH> regs;
    load_halo_v4t<TH, true>(cur, regs);
    bool have = true;
    for (;;) {
        if (!have) {
            gate.wait(v, pair);
            load_halo_v4t<TH, true>(cur, regs);
        }
        stage_halo_v4t<TH>(sm, regs, cur.X0, cur.Y0, cur.w, cur.h);
        const TileRef t = cur;
        const unsigned tpartial = partial;
        const int next = m + stride;
        have = false;
        if (next < total) {
            cur = unpack_tile<TH>(v, n0, n1);
            pair = (int)n0.w;
            partial = n0.z;
            if (next + stride < total) {
                n0 = __ldg(tiles + 2 * (int64_t)(next + stride));
                n1 = __ldg(tiles + 2 * (int64_t)(next + stride) + 1);
            }
            // Prefetch only when the next pair's pyramids are complete; otherwise wait after
            // this tile (never while holding it).
            if (gate.ready(v, pair)) {
                load_halo_v4t<TH, true>(cur, regs);
                have = true;
            }
        }
        blur_score_tile<TH>(sm, t.X0, t.Y0, t.w, t.h, v.partials + (int64_t)tpartial * 6);
        if (next >= total) break;
        m = next;
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------

bool same_colourspace(const Vship_Colorspace_t& a, const Vship_Colorspace_t& b) {
    return a.width == b.width && a.height == b.height && a.target_width == b.target_width &&
           a.target_height == b.target_height && a.sample == b.sample && a.range == b.range &&
           a.subsampling.subw == b.subsampling.subw && a.subsampling.subh == b.subsampling.subh &&
           a.chromaLocation == b.chromaLocation && a.colorFamily == b.colorFamily && a.YUVMatrix == b.YUVMatrix &&
           a.transferFunction == b.transferFunction && a.primaries == b.primaries && a.crop.top == b.crop.top &&
           a.crop.bottom == b.crop.bottom && a.crop.left == b.crop.left && a.crop.right == b.crop.right;
}

using KernelFn = void (*)(const BatchView*);

KernelFn maps_kernel_for(int rows) {
    switch (rows) {
        case 16: return ssimu2_batch_maps_kernel<16>;
        case 64: return ssimu2_batch_maps_kernel<64>;
        default: return ssimu2_batch_maps_kernel<32>;
    }
}

// Front kernel for a launch whose classes all take `path`, or the dispatching one (-1).
using FrontFn = void (*)(FrontParams);

FrontFn front_kernel_for(int path) {
    switch (path) {
        case kFastRgb8Srgb: return ssimu2_batch_front_kernel<kFastRgb8Srgb>;
        case kFastYuv420Bt709: return ssimu2_batch_front_kernel<kFastYuv420Bt709>;
        case kFastGeneric: return ssimu2_batch_front_kernel<kFastGeneric>;
        default: return ssimu2_batch_front_kernel<-1>;
    }
}

constexpr int kTileRowChoices[3] = {16, 32, 64};

// Tuned tile rows keyed by device and mix of resolutions, shared by all batch handlers.
std::mutex g_tune_lock;
std::map<std::string, int> g_tuned;

std::string tune_cache_path() {
    const char* env = std::getenv("VSHIP_TUNE_CACHE");
    if (env) return std::string(env);
    const char* xdg = std::getenv("XDG_CACHE_HOME");
    if (xdg && *xdg) return std::string(xdg) + "/vship_b200/ssimu2_tiles.json";
    const char* home = std::getenv("HOME");
    if (home && *home) return std::string(home) + "/.cache/vship_b200/ssimu2_tiles.json";
    return std::string();
}

// Reads a flat JSON object of string keys and integer values; malformed content is ignored.
std::map<std::string, int> read_tune_file(const std::string& path) {
    std::map<std::string, int> out;
    std::ifstream f(path);
    if (!f) return out;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string s = ss.str();
    size_t i = 0;
    while (true) {
        const size_t k0 = s.find('"', i);
        if (k0 == std::string::npos) break;
        const size_t k1 = s.find('"', k0 + 1);
        if (k1 == std::string::npos) break;
        const size_t colon = s.find(':', k1 + 1);
        if (colon == std::string::npos) break;
        const int val = std::atoi(s.c_str() + colon + 1);
        if (val == 16 || val == 32 || val == 64) out[s.substr(k0 + 1, k1 - k0 - 1)] = val;
        i = colon + 1;
    }
    return out;
}

void write_tune_file(const std::string& path, const std::map<std::string, int>& entries) {
    // Create the parent directories (mkdir -p); failures surface as an unopenable file.
    for (size_t p = path.find('/', 1); p != std::string::npos; p = path.find('/', p + 1))
        (void)mkdir(path.substr(0, p).c_str(), 0755);
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return;
        f << "{\n";
        size_t i = 0;
        for (const auto& kv : entries)
            f << "  \"" << kv.first << "\": " << kv.second << (++i < entries.size() ? ",\n" : "\n");
        f << "}\n";
    }
    std::rename(tmp.c_str(), path.c_str());
}

// Pairs of one launch: classes by colourspace pair, and each pair's class.
struct LaunchPlan {
    int first = 0, count = 0;
    std::vector<int> cls_of;             // per pair of the launch
    struct Cls {
        Vship_Colorspace_t cs[2];
        int misaligned[2];
        ClipGeometry geo[2];
        ColourParams cp[2];
        Pyramid pyr;
        int ftx, fty, stage_floats, npairs, fast;
    };
    std::vector<Cls> classes;
    int64_t xyb_floats = 0;
    int stage_floats = 0;
};

class BatchEngine final : public Ssimu2BatchApi {
public:
    ~BatchEngine() override { release(); }

    void init(int device) override {
        device_ = device;
        CUDA_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        CUDA_CHECK(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
        CUDA_CHECK(cudaEventCreateWithFlags(&last_done_, cudaEventDisableTiming));
        CUDA_CHECK(cudaEventCreateWithFlags(&blob_free_, cudaEventDisableTiming));
        for (int b = 0; b < 2; b++) {
            CUDA_CHECK(cudaEventCreateWithFlags(&copied_[b], cudaEventDisableTiming));
            CUDA_CHECK(cudaEventCreateWithFlags(&consumed_[b], cudaEventDisableTiming));
        }
        CUDA_CHECK(cudaEventCreate(&tune_ev_[0]));
        CUDA_CHECK(cudaEventCreate(&tune_ev_[1]));
        upload_gauss_constants();
        cudaDeviceProp prop{};
        CUDA_CHECK(cudaGetDeviceProperties(&prop, device));
        sms_ = prop.multiProcessorCount;
        device_name_ = prop.name;
        for (char& c : device_name_)
            if (c == '"' || c == '\\' || c == '|') c = '_';
        const size_t budget = (size_t)(0.4 * (double)prop.totalGlobalMem);
        budget_bytes_ = std::min<size_t>((size_t)24 << 30, budget);
        // Descriptor block: header, classes, pairs, pairs grouped by class.
        off_cls_ = round_up((int64_t)sizeof(BatchView), 256);
        off_pairs_ = round_up(off_cls_ + (int64_t)sizeof(BatchClass) * kBatchMaxClasses, 256);
        off_cpairs_ = round_up(off_pairs_ + (int64_t)sizeof(BatchPair) * kBatchMaxPairs, 256);
        blob_cap_ = (size_t)round_up(off_cpairs_ + (int64_t)sizeof(int) * kBatchMaxPairs, 256);
        blob_h_ = pinned_alloc<unsigned char>(blob_cap_, "batch descriptors");
        blob_d_ = device_alloc<unsigned char>(blob_cap_, "batch descriptors");
        kernel_arg_ = reinterpret_cast<const BatchView*>(blob_d_);
        counter_words_ = 2 + 2 * kBatchMaxPairs;
        counters_d_ = device_alloc<unsigned>((size_t)counter_words_, "batch counters");
        CUDA_CHECK(cudaMemset(counters_d_, 0, sizeof(unsigned) * counter_words_));
        err_h_ = pinned_alloc<unsigned>(1, "batch error word");
        *err_h_ = 0;
        CUDA_CHECK(cudaDeviceSynchronize());
    }

    void set_tile_rows(int rows) override {
        if (rows != 0 && rows != 16 && rows != 32 && rows != 64)
            VSHIP_THROW(Vship_BadErrorType, "tile rows must be 0 (automatic), 16, 32 or 64");
        rows_ = rows;
    }

    void compute_device(int n, const VshipExt_FramePair* pairs, double* d_scores, float* d_features,
                        cudaStream_t stream) override {
        check_error_word();
        if (n <= 0) return;
        if (!pairs || !d_scores) VSHIP_THROW(Vship_BadPointer, "NULL argument");
        CUDA_CHECK(cudaStreamWaitEvent(stream, last_done_, 0));
        int first = 0;
        while (first < n) {
            LaunchPlan plan = plan_launch(pairs, first, n);
            const int rows = choose_rows(plan, pairs, d_scores, d_features, stream);
            run(plan, pairs, rows, d_scores, d_features, stream, hold_front_);
            hold_front_ = false;
            first += plan.count;
        }
    }

    void compute(int n, const VshipExt_FramePair* pairs, double* scores, float* features) override {
        check_error_word();
        if (n <= 0) return;
        if (!pairs || !scores) VSHIP_THROW(Vship_BadPointer, "NULL argument");
        // Chunks of about kChunkBytes of input: chunk k is copied on copy_stream_ into
        // staging buffer k % 2 while chunk k - 1 is scored on stream_.
        constexpr int64_t kChunkBytes = (int64_t)256 << 20;
        std::vector<int64_t> bytes(n);
        for (int i = 0; i < n; i++) {
            int64_t b = 0;
            for (int c = 0; c < 2; c++) {
                const ClipGeometry g = make_geometry(c ? pairs[i].dis_colorspace : pairs[i].src_colorspace);
                b += host_image_bytes(g, c ? pairs[i].srcp2 : pairs[i].srcp1, c ? pairs[i].lineSize2 : pairs[i].lineSize);
            }
            bytes[i] = b;
        }
        ensure_outputs(n, features != nullptr);
        CUDA_CHECK(cudaStreamWaitEvent(stream_, last_done_, 0));
        std::vector<VshipExt_FramePair> dev;
        int first = 0, k = 0;
        while (first < n) {
            int last = first;
            int64_t chunk = 0;
            while (last < n && last - first < kBatchMaxPairs && (last == first || chunk + bytes[last] <= kChunkBytes))
                chunk += bytes[last++];
            const int b = k & 1;
            if ((int64_t)stage_cap_ < chunk) grow_staging((size_t)chunk);
            CUDA_CHECK(cudaStreamWaitEvent(copy_stream_, consumed_[b], 0));
            dev.assign(pairs + first, pairs + last);
            int64_t off = 0;
            for (int i = first; i < last; i++) {
                VshipExt_FramePair& d = dev[i - first];
                for (int c = 0; c < 2; c++) {
                    const Vship_Colorspace_t& cs = c ? pairs[i].dis_colorspace : pairs[i].src_colorspace;
                    const ClipGeometry g = make_geometry(cs);
                    const uint8_t* const* src = c ? pairs[i].srcp2 : pairs[i].srcp1;
                    const int64_t* ls = c ? pairs[i].lineSize2 : pairs[i].lineSize;
                    const int64_t nb = host_image_bytes(g, src, ls);
                    const RawImage im = copy_host_image(stage_[b] + off, g, src, ls, copy_stream_);
                    off += nb;
                    for (int p = 0; p < 3; p++) {
                        (c ? d.srcp2 : d.srcp1)[p] = im.p[p];
                        (c ? d.lineSize2 : d.lineSize)[p] = im.stride[p];
                    }
                }
            }
            CUDA_CHECK(cudaEventRecord(copied_[b], copy_stream_));
            CUDA_CHECK(cudaStreamWaitEvent(stream_, copied_[b], 0));
            compute_device(last - first, dev.data(), scores_d_ + first,
                           features ? features_d_ + (int64_t)first * 108 : nullptr, stream_);
            CUDA_CHECK(cudaEventRecord(consumed_[b], stream_));
            first = last;
            k++;
        }
        CUDA_CHECK(cudaMemcpyAsync(scores, scores_d_, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_));
        if (features)
            CUDA_CHECK(cudaMemcpyAsync(features, features_d_, sizeof(float) * 108 * n, cudaMemcpyDeviceToHost, stream_));
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        check_error_word();
    }

    int tile_rows() const override { return last_rows_; }
    void hold_front_tile() override { hold_front_ = true; }
    KernelTimer& timer() override { return timer_; }

private:
    struct Graph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t copy = nullptr;
        cudaGraphNode_t front = nullptr;
        cudaGraphNode_t tiles = nullptr;
        cudaGraphNode_t final = nullptr;
        cudaKernelNodeParams front_params{};
        cudaKernelNodeParams tiles_params{};
        cudaKernelNodeParams final_params{};
    };

    // Reports (once) a wait that ran out in an earlier launch.
    void check_error_word() {
        if (*err_h_ == 0) return;
        *err_h_ = 0;
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaMemset(counters_d_, 0, sizeof(unsigned)));
        VSHIP_THROW(Vship_HIPError, "a dependency wait inside a batch launch exceeded its time limit; "
                                    "the scores of that launch are not valid");
    }

    // Pairs [first, ...) that fit one launch: at most kBatchMaxPairs pairs and
    // kBatchMaxClasses classes (colourspace pair and sample alignment), with pyramids within
    // the memory budget.  Validates every pair's pointers and strides.
    LaunchPlan plan_launch(const VshipExt_FramePair* pairs, int first, int n) {
        LaunchPlan plan;
        plan.first = first;
        for (int i = first; i < n && i - first < kBatchMaxPairs; i++) {
            const VshipExt_FramePair& fp = pairs[i];
            ClipGeometry geo[2];
            int mis[2];
            for (int j = 0; j < 2; j++) {
                geo[j] = make_geometry(j ? fp.dis_colorspace : fp.src_colorspace);
                if (geo[j].generic())
                    VSHIP_THROW(Vship_BadErrorType, "batches take colourspaces without resize or crop (pair " +
                                                        std::to_string(i) + ")");
            }
            if (geo[0].OW != geo[1].OW || geo[0].OH != geo[1].OH)
                VSHIP_THROW(Vship_DifferingInputType, "pair " + std::to_string(i));
            for (int j = 0; j < 2; j++) {
                const uint8_t* const* src = j ? fp.srcp2 : fp.srcp1;
                const int64_t* ls = j ? fp.lineSize2 : fp.lineSize;
                RawImage raw;
                for (int q = 0; q < 3; q++) {
                    if (src[q] == nullptr) VSHIP_THROW(Vship_BadPointer, "null plane pointer (pair " + std::to_string(i) + ")");
                    if (ls[q] < geo[j].pw[q] * geo[j].bytes)
                        VSHIP_THROW(Vship_BadPointer, "lineSize smaller than one row of samples (pair " +
                                                          std::to_string(i) + ")");
                    raw.p[q] = src[q];
                    raw.stride[q] = ls[q];
                }
                mis[j] = misaligned_view(raw, geo[j]) ? 1 : 0;
            }
            int c = -1;
            for (size_t k = 0; k < plan.classes.size(); k++) {
                const auto& K = plan.classes[k];
                if (same_colourspace(K.cs[0], fp.src_colorspace) && same_colourspace(K.cs[1], fp.dis_colorspace) &&
                    K.misaligned[0] == mis[0] && K.misaligned[1] == mis[1]) {
                    c = (int)k;
                    break;
                }
            }
            if (c < 0) {
                if ((int)plan.classes.size() == kBatchMaxClasses) break;
                LaunchPlan::Cls k{};
                k.cs[0] = fp.src_colorspace;
                k.cs[1] = fp.dis_colorspace;
                int fast[2];
                for (int j = 0; j < 2; j++) {
                    k.misaligned[j] = mis[j];
                    k.geo[j] = geo[j];
                    k.cp[j] = make_colour_params(k.cs[j], k.geo[j], mis[j] != 0);
                    k.cp[j].misaligned = mis[j];
                    fast[j] = fast_path_of(k.cp[j]);
                    k.stage_floats = std::max(k.stage_floats, chroma_stage_floats(k.cp[j].subw, k.cp[j].subh));
                }
                k.fast = fast[0] == fast[1] ? fast[0] : kFastGeneric;
                k.pyr = make_pyramid((int)geo[0].OW, (int)geo[0].OH);
                k.ftx = (int)ceil_div(k.pyr.w[1], 32);
                k.fty = (int)ceil_div(k.pyr.h[1], 32);
                plan.classes.push_back(k);
                c = (int)plan.classes.size() - 1;
            }
            const int64_t add = 2 * plan.classes[c].pyr.image_floats;
            if (i > first && (size_t)(plan.xyb_floats + add) * sizeof(float) > budget_bytes_) {
                if (plan.classes[c].npairs == 0) plan.classes.pop_back();
                break;
            }
            plan.xyb_floats += add;
            plan.classes[c].npairs++;
            plan.stage_floats = std::max(plan.stage_floats, plan.classes[c].stage_floats);
            plan.cls_of.push_back(c);
            plan.count++;
        }
        return plan;
    }

    std::string tune_key(const LaunchPlan& plan) const {
        std::vector<std::string> parts;
        for (const auto& k : plan.classes) {
            int bucket = 1;
            while (bucket * 2 <= k.npairs) bucket *= 2;
            parts.push_back(std::to_string(k.pyr.w[0]) + "x" + std::to_string(k.pyr.h[0]) + ":f" +
                            std::to_string(k.fast) + ":n" + std::to_string(bucket));
        }
        std::sort(parts.begin(), parts.end());
        std::string key = device_name_ + "|ssimu2_batch";
        for (const auto& p : parts) key += "|" + p;
        return key;
    }

    int choose_rows(const LaunchPlan& plan, const VshipExt_FramePair* pairs, double* d_scores, float* d_features,
                    cudaStream_t stream) {
        if (rows_ != 0) return rows_;
        const std::string key = tune_key(plan);
        const std::string path = tune_cache_path();
        {
            std::lock_guard<std::mutex> g(g_tune_lock);
            auto it = g_tuned.find(key);
            if (it != g_tuned.end()) return it->second;
            if (!path.empty()) {
                const auto file = read_tune_file(path);
                auto f = file.find(key);
                if (f != file.end()) {
                    g_tuned[key] = f->second;
                    return f->second;
                }
            }
        }
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        CUDA_CHECK(cudaStreamIsCapturing(stream, &cap));
        if (cap != cudaStreamCaptureStatusNone) return 32;
        int best = 32;
        float best_ms = 0.f;
        for (int rows : kTileRowChoices) {
            run(plan, pairs, rows, d_scores, d_features, stream);  // warm-up
            CUDA_CHECK(cudaEventRecord(tune_ev_[0], stream));
            for (int r = 0; r < 2; r++) run(plan, pairs, rows, d_scores, d_features, stream);
            CUDA_CHECK(cudaEventRecord(tune_ev_[1], stream));
            CUDA_CHECK(cudaEventSynchronize(tune_ev_[1]));
            float ms = 0.f;
            CUDA_CHECK(cudaEventElapsedTime(&ms, tune_ev_[0], tune_ev_[1]));
            if (rows == kTileRowChoices[0] || ms < best_ms) {
                best = rows;
                best_ms = ms;
            }
        }
        std::lock_guard<std::mutex> g(g_tune_lock);
        g_tuned[key] = best;
        if (!path.empty()) {
            auto file = read_tune_file(path);
            file[key] = best;
            write_tune_file(path, file);
        }
        return best;
    }

    // Builds the descriptor block of a launch for `rows` in the pinned host copy and the
    // front kernel's parameters.  Returns the block's size; sets the partial count, front
    // tiles and map tiles of the launch, and the front path all its classes share (-1 if they
    // differ).
    size_t write_descriptors(const LaunchPlan& plan, const VshipExt_FramePair* pairs, int rows, double* d_scores,
                             float* d_features, int64_t& partials, int& front_total, int& maps_total, int& path) {
        BatchView* view = reinterpret_cast<BatchView*>(blob_h_);
        BatchClass* cls = reinterpret_cast<BatchClass*>(blob_h_ + off_cls_);
        BatchPair* bp = reinterpret_cast<BatchPair*>(blob_h_ + off_pairs_);
        int* class_pairs = reinterpret_cast<int*>(blob_h_ + off_cpairs_);
        BatchView v{};
        FrontParams& fp = front_params_;
        std::memset(&fp, 0, sizeof(fp));
        const int nc = (int)plan.classes.size();
        for (int c = 0; c < nc; c++) {
            const auto& k = plan.classes[c];
            BatchClass& bc = cls[c];
            std::memset(&bc, 0, sizeof(bc));
            bc.cp[0] = k.cp[0];
            bc.cp[1] = k.cp[1];
            bc.pyr = k.pyr;
            bc.ftx = k.ftx;
            bc.fty = k.fty;
            bc.front_items = 2 * k.ftx * k.fty;
            bc.fast = k.fast;
            int tile = 0;
            for (int s = 0; s < kScales; s++)
                for (int p = 0; p < 3; p++) {
                    int on = 0;
                    for (int m = 0; m < 3; m++) on |= (map_on(p, s, m) ? 1 : 0) << m;
                    if (!on) continue;
                    BatchSeg& g = bc.seg[bc.nseg++];
                    g.off = k.pyr.off[s][p];
                    g.w = k.pyr.w[s];
                    g.h = k.pyr.h[s];
                    g.pitch = k.pyr.pitch[s];
                    g.tiles_x = (int)ceil_div(g.w, kTile);
                    g.ntiles = g.tiles_x * (int)ceil_div(g.h, rows);
                    g.tile_begin = tile;
                    g.slot = p * 36 + s * 6;
                    g.on = on;
                    tile += g.ntiles;
                }
            bc.tiles_per_pair = tile;
            fp.cp[c][0] = k.cp[0];
            fp.cp[c][1] = k.cp[1];
            fp.pyr[c] = k.pyr;
            fp.ftx[c] = k.ftx;
            fp.fty[c] = k.fty;
            fp.fast[c] = k.fast;
            path = c == 0 ? k.fast : (path == k.fast ? path : -1);
        }
        // Pairs in batch order: device views and scratch offsets.
        int64_t xyb = 0, part = 0;
        for (int i = 0; i < plan.count; i++) {
            const VshipExt_FramePair& f = pairs[plan.first + i];
            const int c = plan.cls_of[i];
            BatchPair& q = bp[i];
            std::memset(&q, 0, sizeof(q));
            for (int j = 0; j < 2; j++)
                for (int p = 0; p < 3; p++) {
                    q.raw[j].p[p] = j ? f.srcp2[p] : f.srcp1[p];
                    q.raw[j].stride[p] = j ? f.lineSize2[p] : f.lineSize[p];
                }
            q.cls = c;
            q.xyb = xyb;
            q.partial = part;
            xyb += 2 * plan.classes[c].pyr.image_floats;
            part += cls[c].tiles_per_pair;
        }
        // Work lists: class-major, pairs of a class in batch order.
        int n = 0, front = 0, maps = 0;
        for (int c = 0; c < nc; c++) {
            v.pair_start[c] = fp.pair_start[c] = n;
            v.front_start[c] = fp.front_start[c] = front;
            v.maps_start[c] = maps;
            for (int i = 0; i < plan.count; i++)
                if (plan.cls_of[i] == c) class_pairs[n++] = i;
            const int np = n - v.pair_start[c];
            front += np * cls[c].front_items;
            maps += np * cls[c].tiles_per_pair;
        }
        v.pair_start[nc] = fp.pair_start[nc] = n;
        v.front_start[nc] = fp.front_start[nc] = front;
        v.maps_start[nc] = maps;
        partials = part;
        front_total = front;
        maps_total = maps;
        ensure_scratch(xyb, part, maps);
        v.cls = reinterpret_cast<const BatchClass*>(blob_d_ + off_cls_);
        v.pairs = reinterpret_cast<const BatchPair*>(blob_d_ + off_pairs_);
        v.class_pairs = reinterpret_cast<const int*>(blob_d_ + off_cpairs_);
        v.nclasses = nc;
        v.npairs = plan.count;
        v.front_total = front;
        v.maps_total = maps;
        v.xyb = xyb_;
        v.partials = partials_;
        v.scores = d_scores + plan.first;
        v.features = d_features ? d_features + (int64_t)plan.first * 108 : nullptr;
        v.counters = counters_d_;
        v.tiles = tiles_;
        *view = v;
        fp.nclasses = nc;
        fp.class_pairs = v.class_pairs;
        fp.pairs = v.pairs;
        fp.xyb = xyb_;
        fp.counters = counters_d_;
        return (size_t)(off_cpairs_ + (int64_t)sizeof(int) * plan.count);
    }

    // Grows the pyramid and partial buffers; waits for launches still using them.
    void ensure_scratch(int64_t xyb_floats, int64_t partials, int64_t tiles) {
        if (xyb_floats <= xyb_cap_ && partials <= partial_cap_ && tiles <= tiles_cap_) return;
        CUDA_CHECK(cudaEventSynchronize(last_done_));
        if (tiles > tiles_cap_) {
            device_free(tiles_);
            tiles_ = nullptr;
            tiles_cap_ = 0;
            tiles_ = device_alloc<uint4>((size_t)tiles * 2, "batch tile table");
            tiles_cap_ = tiles;
        }
        if (xyb_floats > xyb_cap_) {
            device_free(xyb_);
            xyb_ = nullptr;
            xyb_cap_ = 0;
            xyb_ = device_alloc<float>((size_t)xyb_floats, "batch XYB pyramids");
            xyb_cap_ = xyb_floats;
        }
        if (partials > partial_cap_) {
            device_free(partials_);
            partials_ = nullptr;
            partial_cap_ = 0;
            partials_ = device_alloc<double>((size_t)partials * 6, "batch tile partials");
            partial_cap_ = partials;
        }
    }

    void ensure_outputs(int n, bool features) {
        if (n > out_cap_ || (features && !features_d_)) {
            CUDA_CHECK(cudaEventSynchronize(last_done_));
            CUDA_CHECK(cudaStreamSynchronize(stream_));
            device_free(scores_d_);
            device_free(features_d_);
            scores_d_ = nullptr;
            features_d_ = nullptr;
            out_cap_ = std::max(n, out_cap_);
            scores_d_ = device_alloc<double>((size_t)out_cap_, "batch scores");
            features_d_ = device_alloc<float>((size_t)out_cap_ * 108, "batch features");
        }
    }

    void grow_staging(size_t bytes) {
        CUDA_CHECK(cudaStreamSynchronize(stream_));
        CUDA_CHECK(cudaStreamSynchronize(copy_stream_));
        for (int b = 0; b < 2; b++) {
            device_free(stage_[b]);
            stage_[b] = nullptr;
        }
        stage_cap_ = 0;
        for (int b = 0; b < 2; b++) stage_[b] = device_alloc<uint8_t>(bytes, "batch input staging");
        stage_cap_ = bytes;
    }

    size_t maps_smem_bytes(int rows) const {
        switch (rows) {
            case 16: return sizeof(MapTile<16>::Smem);
            case 64: return sizeof(MapTile<64>::Smem);
            default: return sizeof(MapTile<32>::Smem);
        }
    }

    // The graph of a launch shape: descriptor copy (its size set per launch), counter reset,
    // the front grid and the tile-table kernel (sizes set per launch), the persistent map
    // kernel behind the tile table and a programmatic edge from the front grid's
    // launch-completion port, the per-pair final kernel, and the error word's copy back to
    // the host.
    Graph& graph_for(int rows, int path, size_t front_smem) {
        const uint64_t key = ((uint64_t)rows << 40) | ((uint64_t)(path + 1) << 32) | (uint64_t)front_smem;
        auto it = graphs_.find(key);
        if (it != graphs_.end()) return it->second;
        KernelFn maps = maps_kernel_for(rows);
        FrontFn front = front_kernel_for(path);
        const size_t msmem = maps_smem_bytes(rows);
        CUDA_CHECK(cudaFuncSetAttribute(maps, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
        CUDA_CHECK(cudaFuncSetAttribute(front, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)front_smem));
        int per_sm = 0;
        CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, maps, kMapThreads, msmem));
        if (per_sm < 1) VSHIP_THROW(Vship_HIPError, "batch map kernel does not fit on a multiprocessor");
        Graph gr;
        CUDA_CHECK(cudaGraphCreate(&gr.graph, 0));
        CUDA_CHECK(cudaGraphAddMemcpyNode1D(&gr.copy, gr.graph, nullptr, 0, blob_d_, blob_h_, blob_cap_,
                                            cudaMemcpyHostToDevice));
        cudaGraphNode_t freed = nullptr, clear = nullptr, mapsn = nullptr, errcopy = nullptr;
        CUDA_CHECK(cudaGraphAddEventRecordNode(&freed, gr.graph, &gr.copy, 1, blob_free_));
        cudaMemsetParams ms{};
        ms.dst = counters_d_ + 1;
        ms.value = 0;
        ms.elementSize = sizeof(unsigned);
        ms.width = (size_t)counter_words_ - 1;
        ms.height = 1;
        CUDA_CHECK(cudaGraphAddMemsetNode(&clear, gr.graph, nullptr, 0, &ms));
        gr.front_params.func = (void*)front;
        gr.front_params.gridDim = dim3(1);
        gr.front_params.blockDim = dim3(256);
        gr.front_params.sharedMemBytes = (unsigned)front_smem;
        gr.front_params.kernelParams = front_args_;
        cudaGraphNode_t deps[2] = {gr.copy, clear};
        CUDA_CHECK(cudaGraphAddKernelNode(&gr.front, gr.graph, deps, 2, &gr.front_params));
        gr.tiles_params.func = (void*)ssimu2_batch_tiles_kernel;
        gr.tiles_params.gridDim = dim3(1);
        gr.tiles_params.blockDim = dim3(256);
        gr.tiles_params.sharedMemBytes = 0;
        gr.tiles_params.kernelParams = kernel_args_;
        CUDA_CHECK(cudaGraphAddKernelNode(&gr.tiles, gr.graph, &gr.copy, 1, &gr.tiles_params));
        cudaKernelNodeParams mp{};
        mp.func = (void*)maps;
        mp.gridDim = dim3((unsigned)(sms_ * per_sm));
        mp.blockDim = dim3(kMapThreads);
        mp.sharedMemBytes = (unsigned)msmem;
        mp.kernelParams = kernel_args_;
        CUDA_CHECK(cudaGraphAddKernelNode(&mapsn, gr.graph, &gr.tiles, 1, &mp));
        cudaGraphEdgeData edge{};
        edge.from_port = cudaGraphKernelNodePortLaunchCompletion;
        edge.type = cudaGraphDependencyTypeProgrammatic;
        if (cudaGraphAddDependencies_v2(gr.graph, &gr.front, &mapsn, &edge, 1) != cudaSuccess) {
            // Without programmatic edges the map kernel simply follows the whole front grid.
            (void)cudaGetLastError();
            CUDA_CHECK(cudaGraphAddDependencies(gr.graph, &gr.front, &mapsn, 1));
        }
        gr.final_params.func = (void*)ssimu2_batch_final_kernel;
        gr.final_params.gridDim = dim3(1);
        gr.final_params.blockDim = dim3(kFinalThreads);
        gr.final_params.sharedMemBytes = 0;
        gr.final_params.kernelParams = kernel_args_;
        CUDA_CHECK(cudaGraphAddKernelNode(&gr.final, gr.graph, &mapsn, 1, &gr.final_params));
        CUDA_CHECK(cudaGraphAddMemcpyNode1D(&errcopy, gr.graph, &gr.final, 1, err_h_, counters_d_, sizeof(unsigned),
                                            cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaGraphInstantiate(&gr.exec, gr.graph, 0));
        return graphs_.emplace(key, gr).first->second;
    }

    // hold: launch the front grid without its last tile, so that the map tiles of the last
    // pair wait for a pyramid that is never finished (the wait-limit test).
    void run(const LaunchPlan& plan, const VshipExt_FramePair* pairs, int rows, double* d_scores, float* d_features,
             cudaStream_t stream, bool hold = false) {
        // The pinned descriptor block is reused: wait until the previous launch has copied it.
        CUDA_CHECK(cudaEventSynchronize(blob_free_));
        int64_t partials = 0;
        int front_total = 0, maps_total = 0, path = -1;
        const size_t bytes =
            write_descriptors(plan, pairs, rows, d_scores, d_features, partials, front_total, maps_total, path);
        Graph& gr = graph_for(rows, path, sizeof(float) * (size_t)plan.stage_floats);
        CUDA_CHECK(cudaGraphExecMemcpyNodeSetParams1D(gr.exec, gr.copy, blob_d_, blob_h_, bytes, cudaMemcpyHostToDevice));
        cudaKernelNodeParams fp = gr.front_params;
        fp.gridDim = dim3((unsigned)(front_total - (hold ? 1 : 0)));  // front_total >= 2
        CUDA_CHECK(cudaGraphExecKernelNodeSetParams(gr.exec, gr.front, &fp));
        cudaKernelNodeParams tp = gr.tiles_params;
        tp.gridDim = dim3((unsigned)ceil_div(maps_total, 256));
        CUDA_CHECK(cudaGraphExecKernelNodeSetParams(gr.exec, gr.tiles, &tp));
        cudaKernelNodeParams qp = gr.final_params;
        qp.gridDim = dim3((unsigned)plan.count);
        CUDA_CHECK(cudaGraphExecKernelNodeSetParams(gr.exec, gr.final, &qp));
        const int t = timer_.begin(0, "ssimu2_batch", stream);
        CUDA_CHECK(cudaGraphLaunch(gr.exec, stream));
        timer_.end(t, stream);
        CUDA_CHECK(cudaEventRecord(last_done_, stream));
        last_rows_ = rows;
    }

    void release() {
        if (stream_) (void)cudaStreamSynchronize(stream_);
        if (copy_stream_) (void)cudaStreamSynchronize(copy_stream_);
        if (last_done_) (void)cudaEventSynchronize(last_done_);
        for (auto& kv : graphs_) {
            if (kv.second.exec) (void)cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) (void)cudaGraphDestroy(kv.second.graph);
        }
        graphs_.clear();
        timer_.destroy();
        device_free(xyb_);
        device_free(partials_);
        device_free(tiles_);
        device_free(blob_d_);
        device_free(counters_d_);
        device_free(scores_d_);
        device_free(features_d_);
        for (int b = 0; b < 2; b++) device_free(stage_[b]);
        if (blob_h_) (void)cudaFreeHost(blob_h_);
        if (err_h_) (void)cudaFreeHost(err_h_);
        for (cudaEvent_t e : {last_done_, blob_free_, copied_[0], copied_[1], consumed_[0], consumed_[1], tune_ev_[0], tune_ev_[1]})
            if (e) (void)cudaEventDestroy(e);
        if (stream_) (void)cudaStreamDestroy(stream_);
        if (copy_stream_) (void)cudaStreamDestroy(copy_stream_);
    }

    int device_ = 0, sms_ = 1;
    std::string device_name_;
    size_t budget_bytes_ = 0;
    int rows_ = 0, last_rows_ = 0;
    cudaStream_t stream_ = nullptr, copy_stream_ = nullptr;
    cudaEvent_t last_done_ = nullptr, blob_free_ = nullptr;
    cudaEvent_t copied_[2] = {}, consumed_[2] = {}, tune_ev_[2] = {};
    unsigned char* blob_h_ = nullptr;
    unsigned char* blob_d_ = nullptr;
    size_t blob_cap_ = 0;
    int64_t off_cls_ = 0, off_pairs_ = 0, off_cpairs_ = 0;
    unsigned* counters_d_ = nullptr;
    int counter_words_ = 0;
    unsigned* err_h_ = nullptr;
    bool hold_front_ = false;
    float* xyb_ = nullptr;
    int64_t xyb_cap_ = 0;
    double* partials_ = nullptr;
    int64_t partial_cap_ = 0;
    uint4* tiles_ = nullptr;
    int64_t tiles_cap_ = 0;
    double* scores_d_ = nullptr;
    float* features_d_ = nullptr;
    int out_cap_ = 0;
    uint8_t* stage_[2] = {nullptr, nullptr};
    size_t stage_cap_ = 0;
    std::map<uint64_t, Graph> graphs_;
    const BatchView* kernel_arg_ = nullptr;       // the map, tile and final kernels' parameter
    void* kernel_args_[1] = {&kernel_arg_};
    FrontParams front_params_{};                  // the front kernel's parameter, set per launch
    void* front_args_[1] = {&front_params_};
    KernelTimer timer_;
};

}  // namespace
}  // namespace ssimu2
}  // namespace vship

vship::Ssimu2BatchApi* vship::make_ssimu2_batch_engine() { return new vship::ssimu2::BatchEngine(); }

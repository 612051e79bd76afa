// VapourSynth plugin entry of the library (VapourSynthPluginInit2), so that scripts calling
// core.vship.SSIMULACRA2 / BUTTERAUGLI / GpuInfo keep working when this library replaces the
// reference's (src/VshipLib.cpp:62-68).  The filters mirror the reference's
// (src/ssimu2/vapoursynth.hpp, src/butter/vapoursynth.hpp): the same function names, argument
// strings and defaults, the same conversion of non-RGBS clips through the resize plugin
// (src/util/torgbs.hpp), the same frame properties and error codes; frames are scored through
// this library's own C ABI: SSIMULACRA2 and Butteraugli with a pool of `numStream` handlers
// shared by VapourSynth's worker threads, CVVDP with one handler that keeps the sequence's
// temporal state (src/cvvdp/vapoursynth.hpp).
#include <cuda_runtime.h>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "vs_abi.h"
#include "../../include/VshipAPI.h"

namespace vship {
namespace vsplugin {
namespace {

static_assert(offsetof(VsAbiApi, freeNode) == 7 * sizeof(void*), "VSAPI slot 8");
static_assert(offsetof(VsAbiApi, getVideoInfo) == 10 * sizeof(void*), "VSAPI slot 11");
static_assert(offsetof(VsAbiApi, freeFrame) == 16 * sizeof(void*), "VSAPI slot 17");
static_assert(offsetof(VsAbiApi, getReadPtr) == 22 * sizeof(void*), "VSAPI slot 23");
static_assert(offsetof(VsAbiApi, queryVideoFormat) == 32 * sizeof(void*), "VSAPI slot 33");
static_assert(offsetof(VsAbiApi, getFrameFilter) == 38 * sizeof(void*), "VSAPI slot 39");
static_assert(offsetof(VsAbiApi, setFilterError) == 42 * sizeof(void*), "VSAPI slot 43");
static_assert(offsetof(VsAbiApi, createMap) == 47 * sizeof(void*), "VSAPI slot 48");
static_assert(offsetof(VsAbiApi, mapSetError) == 51 * sizeof(void*), "VSAPI slot 52");
static_assert(offsetof(VsAbiApi, mapGetInt) == 59 * sizeof(void*), "VSAPI slot 60");
static_assert(offsetof(VsAbiApi, mapSetFloat) == 67 * sizeof(void*), "VSAPI slot 68");
static_assert(offsetof(VsAbiApi, mapGetData) == 69 * sizeof(void*), "VSAPI slot 70");
static_assert(offsetof(VsAbiApi, mapGetNode) == 73 * sizeof(void*), "VSAPI slot 74");
static_assert(offsetof(VsAbiApi, getPluginByID) == 83 * sizeof(void*), "VSAPI slot 84");
static_assert(offsetof(VsAbiApi, invoke) == 96 * sizeof(void*), "VSAPI slot 97");
static_assert(offsetof(VsAbiApi, getCoreInfo) == 101 * sizeof(void*), "VSAPI slot 102");

std::string error_message(Vship_Exception code) { return Error(code, __FILE__, __LINE__, "").message(); }

std::string global_error() {
    const int n = Vship_GetDetailedLastError(nullptr, 0);
    std::string s((size_t)std::max(n, 1), '\0');
    Vship_GetDetailedLastError(&s[0], n);
    return std::string(s.c_str());
}

// Handlers shared by the filter's frame requests: a frame takes a free one and gives it back.
struct Pool {
    std::mutex m;
    std::condition_variable cv;
    std::vector<int> free;
    int acquire() {
        std::unique_lock<std::mutex> l(m);
        cv.wait(l, [&] { return !free.empty(); });
        const int i = free.back();
        free.pop_back();
        return i;
    }
    void release(int i) {
        {
            std::lock_guard<std::mutex> g(m);
            free.push_back(i);
        }
        cv.notify_one();
    }
};

bool is_rgbs(const VsAbiVideoFormat& f) {
    return f.bitsPerSample == 32 && f.colorFamily == vsCfRGB && f.sampleType == vsStFloat;
}

bool same_video_info(const VsAbiVideoInfo* a, const VsAbiVideoInfo* b) {
    return a->height == b->height && a->width == b->width && a->format.colorFamily == b->format.colorFamily &&
           a->format.sampleType == b->format.sampleType && a->format.bitsPerSample == b->format.bitsPerSample &&
           a->format.subSamplingW == b->format.subSamplingW && a->format.subSamplingH == b->format.subSamplingH;
}

// A clip as planar float R'G'B' (src/util/torgbs.hpp): other formats go through the resize
// plugin's Bicubic with BT.709 (BT.470BG below 651 rows) limited-range input and full-range
// RGB output.  Consumes `source`; returns null with `err` set when the conversion fails.
VSNode* to_rgbs(VSNode* source, VSCore* core, const VsAbiApi* vsapi, std::string& err) {
    const VsAbiVideoInfo* vi = vsapi->getVideoInfo(source);
    if (is_rgbs(vi->format)) return source;
    const int matrix = vi->height > 650 ? 1 : 6;
    VSMap* args = vsapi->createMap();
    vsapi->mapConsumeNode(args, "clip", source, vsMaReplace);
    vsapi->mapSetInt(args, "matrix_in", matrix, vsMaReplace);
    vsapi->mapSetInt(args, "transfer_in", 1, vsMaReplace);
    vsapi->mapSetInt(args, "primaries_in", 1, vsMaReplace);
    vsapi->mapSetInt(args, "range_in", 0, vsMaReplace);
    vsapi->mapSetInt(args, "matrix", 0, vsMaReplace);
    vsapi->mapSetInt(args, "transfer", 1, vsMaReplace);
    vsapi->mapSetInt(args, "primaries", 1, vsMaReplace);
    vsapi->mapSetInt(args, "range", 1, vsMaReplace);
    vsapi->mapSetInt(args, "format", VS_ABI_MAKE_VIDEO_ID(vsCfRGB, vsStFloat, 32, 0, 0), vsMaReplace);
    VSPlugin* resize = vsapi->getPluginByID("com.vapoursynth.resize", core);
    VSNode* out = nullptr;
    if (!resize) {
        err = "the resize plugin (com.vapoursynth.resize) is needed to convert the clip to RGBS";
    } else {
        VSMap* ret = vsapi->invoke(resize, "Bicubic", args);
        const char* e = vsapi->mapGetError(ret);
        if (e) err = e;
        else out = vsapi->mapGetNode(ret, "clip", 0, nullptr);
        vsapi->freeMap(ret);
    }
    vsapi->freeMap(args);
    return out;
}

Vship_Colorspace_t rgbs_colorspace(const VsAbiVideoInfo* vi) {
    Vship_Colorspace_t cs{};
    cs.width = vi->width;
    cs.height = vi->height;
    cs.target_width = -1;
    cs.target_height = -1;
    cs.sample = Vship_SampleFLOAT;
    cs.range = Vship_RangeFull;
    cs.subsampling.subw = 0;
    cs.subsampling.subh = 0;
    cs.chromaLocation = Vship_ChromaLoc_Left;
    cs.colorFamily = Vship_ColorRGB;
    cs.YUVMatrix = Vship_MATRIX_RGB;
    cs.transferFunction = Vship_TRC_BT709;
    cs.primaries = Vship_PRIMARIES_BT709;
    return cs;
}

// Reference and distorted clips as RGBS with equal geometry, or an error set on `out`.
bool open_pair(const VSMap* in, VSMap* out, VSCore* core, const VsAbiApi* vsapi, VSNode*& ref, VSNode*& dis) {
    std::string err;
    ref = to_rgbs(vsapi->mapGetNode(in, "reference", 0, nullptr), core, vsapi, err);
    if (!ref) {
        vsapi->mapSetError(out, err.c_str());
        return false;
    }
    dis = to_rgbs(vsapi->mapGetNode(in, "distorted", 0, nullptr), core, vsapi, err);
    if (!dis) {
        vsapi->freeNode(ref);
        vsapi->mapSetError(out, err.c_str());
        return false;
    }
    const VsAbiVideoInfo* a = vsapi->getVideoInfo(ref);
    const VsAbiVideoInfo* b = vsapi->getVideoInfo(dis);
    Vship_Exception code = Vship_NoError;
    if (!same_video_info(a, b)) code = Vship_DifferingInputType;
    else if (!is_rgbs(a->format)) code = Vship_NonRGBSInput;
    if (code != Vship_NoError) {
        vsapi->mapSetError(out, error_message(code).c_str());
        vsapi->freeNode(ref);
        vsapi->freeNode(dis);
        return false;
    }
    return true;
}

int get_int(const VSMap* in, const char* key, int dflt, const VsAbiApi* vsapi) {
    int e = 0;
    const int64_t v = vsapi->mapGetInt(in, key, 0, &e);
    return e == vsPeSuccess ? (int)v : dflt;
}

// Handlers to create: numStream (default `dflt`), at most the core's threads, at least one.
int stream_count(const VSMap* in, VSCore* core, const VsAbiApi* vsapi, int dflt) {
    VsAbiCoreInfo info{};
    vsapi->getCoreInfo(core, &info);
    int n = get_int(in, "numStream", dflt < 0 ? info.numThreads : dflt, vsapi);
    n = std::min(n, info.numThreads);
    return std::max(n, 1);
}

struct FramePlanes {
    const uint8_t* p1[3];
    const uint8_t* p2[3];
    int64_t ls1[3], ls2[3];
};

FramePlanes planes_of(const VSFrame* a, const VSFrame* b, const VsAbiApi* vsapi) {
    FramePlanes f;
    for (int c = 0; c < 3; c++) {
        f.p1[c] = vsapi->getReadPtr(a, c);
        f.p2[c] = vsapi->getReadPtr(b, c);
        f.ls1[c] = (int64_t)vsapi->getStride(a, c);
        f.ls2[c] = (int64_t)vsapi->getStride(b, c);
    }
    return f;
}

// ------------------------------------------------------------------ SSIMULACRA2

struct Ssimu2Filter {
    VSNode* ref = nullptr;
    VSNode* dis = nullptr;
    std::vector<Vship_SSIMU2Handler> handlers;
    Pool pool;
};

const VSFrame* ssimu2_get_frame(int n, int reason, void* instance, void**, VSFrameContext* ctx, VSCore* core,
                                const VsAbiApi* vsapi) {
    Ssimu2Filter* d = static_cast<Ssimu2Filter*>(instance);
    if (reason == vsArInitial) {
        vsapi->requestFrameFilter(n, d->ref, ctx);
        vsapi->requestFrameFilter(n, d->dis, ctx);
        return nullptr;
    }
    if (reason != vsArAllFramesReady) return nullptr;
    const VSFrame* a = vsapi->getFrameFilter(n, d->ref, ctx);
    const VSFrame* b = vsapi->getFrameFilter(n, d->dis, ctx);
    VSFrame* dst = vsapi->copyFrame(b, core);
    FramePlanes f = planes_of(a, b, vsapi);
    double score = 0.0;
    const int k = d->pool.acquire();
    const Vship_Exception rc = Vship_ComputeSSIMU2(d->handlers[k], &score, f.p1, f.p2, f.ls1, f.ls2);
    std::string msg;
    if (rc != Vship_NoError) {
        const int len = Vship_SSIMU2GetDetailedLastError(d->handlers[k], nullptr, 0);
        msg.assign((size_t)std::max(len, 1), '\0');
        Vship_SSIMU2GetDetailedLastError(d->handlers[k], &msg[0], len);
    }
    d->pool.release(k);
    vsapi->freeFrame(a);
    vsapi->freeFrame(b);
    if (rc != Vship_NoError) {
        vsapi->freeFrame(dst);
        vsapi->setFilterError(msg.c_str(), ctx);
        return nullptr;
    }
    vsapi->mapSetFloat(vsapi->getFramePropertiesRW(dst), "_SSIMULACRA2", score, vsMaReplace);
    return dst;
}

void ssimu2_free(void* instance, VSCore*, const VsAbiApi* vsapi) {
    Ssimu2Filter* d = static_cast<Ssimu2Filter*>(instance);
    vsapi->freeNode(d->ref);
    vsapi->freeNode(d->dis);
    for (auto& h : d->handlers) Vship_SSIMU2Free(h);
    delete d;
}

void ssimu2_create(const VSMap* in, VSMap* out, void*, VSCore* core, const VsAbiApi* vsapi) {
    VSNode *ref, *dis;
    if (!open_pair(in, out, core, vsapi, ref, dis)) return;
    const int gpu = get_int(in, "gpu_id", 0, vsapi);
    if (Vship_GPUFullCheck(gpu) != Vship_NoError) {
        vsapi->mapSetError(out, global_error().c_str());
        vsapi->freeNode(ref);
        vsapi->freeNode(dis);
        return;
    }
    Ssimu2Filter* d = new Ssimu2Filter();
    d->ref = ref;
    d->dis = dis;
    const VsAbiVideoInfo* vi = vsapi->getVideoInfo(ref);
    const Vship_Colorspace_t cs = rgbs_colorspace(vi);
    const int streams = stream_count(in, core, vsapi, -1);
    for (int i = 0; i < streams; i++) {
        Vship_SSIMU2Handler h;
        if (Vship_SSIMU2Init2(&h, cs, cs, gpu) != Vship_NoError) {
            const int len = Vship_SSIMU2GetDetailedLastError(h, nullptr, 0);
            std::string msg((size_t)std::max(len, 1), '\0');
            Vship_SSIMU2GetDetailedLastError(h, &msg[0], len);
            Vship_SSIMU2Free(h);
            vsapi->mapSetError(out, msg.c_str());
            ssimu2_free(d, core, vsapi);
            return;
        }
        d->handlers.push_back(h);
        d->pool.free.push_back(i);
    }
    const VsAbiFilterDependency deps[2] = {{ref, vsRpStrictSpatial}, {dis, vsRpStrictSpatial}};
    vsapi->createVideoFilter(out, "vship", vi, ssimu2_get_frame, ssimu2_free, vsFmParallel, deps, 2, d, core);
}

// ------------------------------------------------------------------ Butteraugli

struct ButterFilter {
    VSNode* ref = nullptr;
    VSNode* dis = nullptr;
    int distmap = 0;
    VsAbiVideoFormat gray{};
    std::vector<Vship_ButteraugliHandler> handlers;
    Pool pool;
};

const VSFrame* butter_get_frame(int n, int reason, void* instance, void**, VSFrameContext* ctx, VSCore* core,
                                const VsAbiApi* vsapi) {
    ButterFilter* d = static_cast<ButterFilter*>(instance);
    if (reason == vsArInitial) {
        vsapi->requestFrameFilter(n, d->ref, ctx);
        vsapi->requestFrameFilter(n, d->dis, ctx);
        return nullptr;
    }
    if (reason != vsArAllFramesReady) return nullptr;
    const VSFrame* a = vsapi->getFrameFilter(n, d->ref, ctx);
    const VSFrame* b = vsapi->getFrameFilter(n, d->dis, ctx);
    VSFrame* dst = d->distmap ? vsapi->newVideoFrame(&d->gray, vsapi->getFrameWidth(a, 0), vsapi->getFrameHeight(a, 0),
                                                     nullptr, core)
                              : vsapi->copyFrame(b, core);
    FramePlanes f = planes_of(a, b, vsapi);
    Vship_ButteraugliScore score{};
    const int k = d->pool.acquire();
    const Vship_Exception rc =
        d->distmap ? Vship_ComputeButteraugli(d->handlers[k], &score, vsapi->getWritePtr(dst, 0),
                                              (int64_t)vsapi->getStride(dst, 0), f.p1, f.p2, f.ls1, f.ls2)
                   : Vship_ComputeButteraugli(d->handlers[k], &score, nullptr, 0, f.p1, f.p2, f.ls1, f.ls2);
    std::string msg;
    if (rc != Vship_NoError) {
        const int len = Vship_ButteraugliGetDetailedLastError(d->handlers[k], nullptr, 0);
        msg.assign((size_t)std::max(len, 1), '\0');
        Vship_ButteraugliGetDetailedLastError(d->handlers[k], &msg[0], len);
    }
    d->pool.release(k);
    vsapi->freeFrame(a);
    vsapi->freeFrame(b);
    if (rc != Vship_NoError) {
        vsapi->freeFrame(dst);
        vsapi->setFilterError(msg.c_str(), ctx);
        return nullptr;
    }
    VSMap* props = vsapi->getFramePropertiesRW(dst);
    vsapi->mapSetFloat(props, "_BUTTERAUGLI_QNorm", score.normQ, vsMaReplace);
    vsapi->mapSetFloat(props, "_BUTTERAUGLI_3Norm", score.norm3, vsMaReplace);
    vsapi->mapSetFloat(props, "_BUTTERAUGLI_INFNorm", score.norminf, vsMaReplace);
    return dst;
}

void butter_free(void* instance, VSCore*, const VsAbiApi* vsapi) {
    ButterFilter* d = static_cast<ButterFilter*>(instance);
    vsapi->freeNode(d->ref);
    vsapi->freeNode(d->dis);
    for (auto& h : d->handlers) Vship_ButteraugliFree(h);
    delete d;
}

void butter_create(const VSMap* in, VSMap* out, void*, VSCore* core, const VsAbiApi* vsapi) {
    VSNode *ref, *dis;
    if (!open_pair(in, out, core, vsapi, ref, dis)) return;
    int e = 0;
    double intensity = vsapi->mapGetFloat(in, "intensity_multiplier", 0, &e);
    if (e != vsPeSuccess) intensity = 203.0;
    const int gpu = get_int(in, "gpu_id", 0, vsapi);
    const int qnorm = get_int(in, "qnorm", 2, vsapi);
    if (Vship_GPUFullCheck(gpu) != Vship_NoError) {
        vsapi->mapSetError(out, global_error().c_str());
        vsapi->freeNode(ref);
        vsapi->freeNode(dis);
        return;
    }
    ButterFilter* d = new ButterFilter();
    d->ref = ref;
    d->dis = dis;
    d->distmap = get_int(in, "distmap", 0, vsapi);
    vsapi->queryVideoFormat(&d->gray, vsCfGray, vsStFloat, 32, 0, 0, core);
    const VsAbiVideoInfo* vi = vsapi->getVideoInfo(ref);
    VsAbiVideoInfo vout = *vi;
    if (d->distmap) vout.format = d->gray;
    const Vship_Colorspace_t cs = rgbs_colorspace(vi);
    const int streams = stream_count(in, core, vsapi, 4);
    for (int i = 0; i < streams; i++) {
        Vship_ButteraugliHandler h;
        if (Vship_ButteraugliInit2(&h, cs, cs, qnorm, (float)intensity, gpu) != Vship_NoError) {
            const int len = Vship_ButteraugliGetDetailedLastError(h, nullptr, 0);
            std::string msg((size_t)std::max(len, 1), '\0');
            Vship_ButteraugliGetDetailedLastError(h, &msg[0], len);
            Vship_ButteraugliFree(h);
            vsapi->mapSetError(out, msg.c_str());
            butter_free(d, core, vsapi);
            return;
        }
        d->handlers.push_back(h);
        d->pool.free.push_back(i);
    }
    const VsAbiFilterDependency deps[2] = {{ref, vsRpStrictSpatial}, {dis, vsRpStrictSpatial}};
    vsapi->createVideoFilter(out, "vship", &vout, butter_get_frame, butter_free, vsFmParallel, deps, 2, d, core);
}

// ------------------------------------------------------------------ CVVDP

// One handler: the metric keeps the sequence's temporal state, so frames are scored one at a
// time, in request order (src/cvvdp/vapoursynth.hpp:18-99).
struct CvvdpFilter {
    VSNode* ref = nullptr;
    VSNode* dis = nullptr;
    int distmap = 0;
    int64_t out_w = 0, out_h = 0;
    VsAbiVideoFormat gray{};
    Vship_CVVDPHandler handler{};
    bool alive = false;
    std::mutex m;
};

const VSFrame* cvvdp_get_frame(int n, int reason, void* instance, void**, VSFrameContext* ctx, VSCore* core,
                               const VsAbiApi* vsapi) {
    CvvdpFilter* d = static_cast<CvvdpFilter*>(instance);
    if (reason == vsArInitial) {
        vsapi->requestFrameFilter(n, d->ref, ctx);
        vsapi->requestFrameFilter(n, d->dis, ctx);
        return nullptr;
    }
    if (reason != vsArAllFramesReady) return nullptr;
    const VSFrame* a = vsapi->getFrameFilter(n, d->ref, ctx);
    const VSFrame* b = vsapi->getFrameFilter(n, d->dis, ctx);
    VSFrame* dst = d->distmap ? vsapi->newVideoFrame(&d->gray, (int)d->out_w, (int)d->out_h, nullptr, core)
                              : vsapi->copyFrame(b, core);
    FramePlanes f = planes_of(a, b, vsapi);
    double score = 0.0;
    Vship_Exception rc;
    std::string msg;
    {
        std::lock_guard<std::mutex> g(d->m);
        rc = d->distmap ? Vship_ComputeCVVDP(d->handler, &score, vsapi->getWritePtr(dst, 0), (int64_t)vsapi->getStride(dst, 0),
                                             f.p1, f.p2, f.ls1, f.ls2)
                        : Vship_ComputeCVVDP(d->handler, &score, nullptr, 0, f.p1, f.p2, f.ls1, f.ls2);
        if (rc != Vship_NoError) {
            const int len = Vship_CVVDPGetDetailedLastError(d->handler, nullptr, 0);
            msg.assign((size_t)std::max(len, 1), '\0');
            Vship_CVVDPGetDetailedLastError(d->handler, &msg[0], len);
        }
    }
    vsapi->freeFrame(a);
    vsapi->freeFrame(b);
    if (rc != Vship_NoError) {
        vsapi->freeFrame(dst);
        vsapi->setFilterError(msg.c_str(), ctx);
        return nullptr;
    }
    vsapi->mapSetFloat(vsapi->getFramePropertiesRW(dst), "_CVVDP", score, vsMaReplace);
    return dst;
}

void cvvdp_free(void* instance, VSCore*, const VsAbiApi* vsapi) {
    CvvdpFilter* d = static_cast<CvvdpFilter*>(instance);
    vsapi->freeNode(d->ref);
    vsapi->freeNode(d->dis);
    if (d->alive) Vship_CVVDPFree(d->handler);
    delete d;
}

std::string get_data(const VSMap* in, const char* key, const char* dflt, const VsAbiApi* vsapi) {
    int e = 0;
    const char* v = vsapi->mapGetData(in, key, 0, &e);
    return e == vsPeSuccess && v ? std::string(v) : std::string(dflt);
}

void cvvdp_create(const VSMap* in, VSMap* out, void*, VSCore* core, const VsAbiApi* vsapi) {
    VSNode *ref, *dis;
    if (!open_pair(in, out, core, vsapi, ref, dis)) return;
    const int gpu = get_int(in, "gpu_id", 0, vsapi);
    const int resize = get_int(in, "resizeToDisplay", 0, vsapi);
    const std::string model = get_data(in, "model_name", "standard_fhd", vsapi);
    const std::string json = get_data(in, "model_config_json", "", vsapi);
    if (Vship_GPUFullCheck(gpu) != Vship_NoError) {
        vsapi->mapSetError(out, global_error().c_str());
        vsapi->freeNode(ref);
        vsapi->freeNode(dis);
        return;
    }
    const VsAbiVideoInfo* vi = vsapi->getVideoInfo(ref);
    float fps = (float)vi->fpsNum / (float)vi->fpsDen;
    if (!(fps > 0) || fps > 100000.f) fps = 60.f;  // unknown or absurd rates (vapoursynth.hpp:179-183)
    CvvdpFilter* d = new CvvdpFilter();
    d->ref = ref;
    d->dis = dis;
    d->distmap = get_int(in, "distmap", 0, vsapi);
    const Vship_Colorspace_t cs = rgbs_colorspace(vi);
    if (Vship_CVVDPInit3(&d->handler, cs, cs, fps, resize != 0, model.c_str(), json.empty() ? nullptr : json.c_str(),
                         gpu) != Vship_NoError) {
        const int len = Vship_CVVDPGetDetailedLastError(d->handler, nullptr, 0);
        std::string msg((size_t)std::max(len, 1), '\0');
        Vship_CVVDPGetDetailedLastError(d->handler, &msg[0], len);
        Vship_CVVDPFree(d->handler);
        vsapi->mapSetError(out, msg.c_str());
        cvvdp_free(d, core, vsapi);
        return;
    }
    d->alive = true;
    Vship_CVVDPGetDistmapResolution(d->handler, &d->out_w, &d->out_h);
    vsapi->queryVideoFormat(&d->gray, vsCfGray, vsStFloat, 32, 0, 0, core);
    VsAbiVideoInfo vout = *vi;
    if (d->distmap) {
        vout.format = d->gray;
        vout.width = (int)d->out_w;
        vout.height = (int)d->out_h;
    }
    const VsAbiFilterDependency deps[2] = {{ref, vsRpStrictSpatial}, {dis, vsRpStrictSpatial}};
    vsapi->createVideoFilter(out, "vship", &vout, cvvdp_get_frame, cvvdp_free, vsFmParallelRequests, deps, 2, d, core);
}

// ------------------------------------------------------------------ GpuInfo

// Device description (src/VshipLib.cpp:9-59): every device's name without gpu_id, the chosen
// device's properties with it.
void gpu_info(const VSMap* in, VSMap* out, void*, VSCore*, const VsAbiApi* vsapi) {
    int count = 0;
    if (Vship_GetDeviceCount(&count) != Vship_NoError) {
        vsapi->mapSetError(out, global_error().c_str());
        return;
    }
    int e = 0;
    const int64_t id = vsapi->mapGetInt(in, "gpu_id", 0, &e);
    const int gpu = e == vsPeSuccess ? (int)id : 0;
    if (gpu < 0 || gpu >= count) {
        vsapi->mapSetError(out, error_message(Vship_BadDeviceArgument).c_str());
        return;
    }
    std::stringstream ss;
    cudaDeviceProp p{};
    if (e != vsPeSuccess) {
        for (int i = 0; i < count; i++) {
            if (cudaGetDeviceProperties(&p, i) != cudaSuccess) continue;
            ss << "GPU " << i << ": " << p.name << std::endl;
        }
    } else if (cudaGetDeviceProperties(&p, gpu) == cudaSuccess) {
        ss << "Name: " << p.name << std::endl;
        ss << "MultiProcessorCount: " << p.multiProcessorCount << std::endl;
        ss << "MaxSharedMemoryPerBlock: " << p.sharedMemPerBlock << " bytes" << std::endl;
        ss << "WarpSize: " << p.warpSize << std::endl;
        ss << "VRAMCapacity: " << ((float)p.totalGlobalMem) / 1000000000 << " GB" << std::endl;
        ss << "MemoryBusWidth: " << p.memoryBusWidth << " bits" << std::endl;
        ss << "Integrated: " << p.integrated << std::endl;
        ss << "PassKernelCheck : " << (int)(Vship_GPUFullCheck(gpu) == Vship_NoError) << std::endl;
    }
    const std::string s = ss.str();
    vsapi->mapSetData(out, "gpu_human_data", s.data(), (int)s.size(), vsDtUtf8, vsMaReplace);
}

}  // namespace
}  // namespace vsplugin
}  // namespace vship

extern "C" __attribute__((visibility("default"))) void VapourSynthPluginInit2(VSPlugin* plugin,
                                                                              const VsAbiPluginApi* vspapi) {
    using namespace vship::vsplugin;
    vspapi->configPlugin("com.lumen.vship", "vship", "VapourSynth SSIMULACRA2 on GPU", VS_ABI_MAKE_VERSION(4, 1),
                         VS_ABI_API_VERSION, 0, plugin);
    vspapi->registerFunction("SSIMULACRA2", "reference:vnode;distorted:vnode;numStream:int:opt;gpu_id:int:opt;",
                             "clip:vnode;", ssimu2_create, nullptr, plugin);
    vspapi->registerFunction("BUTTERAUGLI",
                             "reference:vnode;distorted:vnode;qnorm:int:opt;intensity_multiplier:float:opt;"
                             "distmap:int:opt;numStream:int:opt;gpu_id:int:opt;",
                             "clip:vnode;", butter_create, nullptr, plugin);
    vspapi->registerFunction("CVVDP",
                             "reference:vnode;distorted:vnode;model_name:data:opt;model_config_json:data:opt;"
                             "resizeToDisplay:int:opt;distmap:int:opt;gpu_id:int:opt;",
                             "clip:vnode;", cvvdp_create, nullptr, plugin);
    vspapi->registerFunction("GpuInfo", "gpu_id:int:opt;", "gpu_human_data:data;", gpu_info, nullptr, plugin);
}

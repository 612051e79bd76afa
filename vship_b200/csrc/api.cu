// The Vship C ABI (include/VshipAPI.h, include/VshipAPI_ext.h) over the B200 engines.
//
// Mirrors src/VshipLib.cpp:70-562 of the reference: handler tables with reusable ids, a
// global and a per-handler last error, the same error codes and message layout.  The
// differences are deliberate: a freed or never-initialised id gives
// Vship_BadHandler instead of undefined behaviour, a handler used by two threads at once
// gives Vship_BadHandler instead of a data race, and the global last error is guarded by a
// mutex.
#include <cuda_runtime.h>
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/VshipAPI.h"
#include "../../include/VshipAPI_ext.h"
#include "common.cuh"
#include "engines.h"

namespace vship {

const char* error_text(int code) {
    switch (code) {
    case Vship_NoError:
        return "NoError: When everything is right, you should not be searching for problems but appreciate what was given to you.";
    case Vship_OutOfVRAM:
        return "OutOfVRAM: Vship was not able to perform GPU memory allocation. (Advice) Reduce or Set numStream argument";
    case Vship_OutOfRAM:
        return "OutOfRAM: Vship was not able to allocate CPU memory. This is a rare error that should be reported. Check your RAM usage";
    case Vship_HIPError:
        return "InternalError: A GPU Call failed inside Vship. This may be due to a bad environment but is likely due to a bug in Vship.";
    case Vship_BadDisplayModel:
        return "BadDisplayModel: Vship was not able to find a corresponding model as specified. (Advice) See valid models in the doc or remove this option";
    case Vship_DifferingInputType:
        return "DifferingInputType: Vship received 2 videos with different properties. (Advice) verify that they have the same width, height and length";
    case Vship_NonRGBSInput:
        return "NonRGBSInput: Vship did not manage to get RGBS format of your inputs. This should not happen. (Advice) try converting yourself to RGBS";
    case Vship_BadPath:
        return "BadPath: Vship failed to open a file.";
    case Vship_BadJson:
        return "BadJson: Vship failed to parse the json";
    case Vship_DeviceCountError:
        return "DeviceCountError: Vship was unable to verify the number of GPU on your system. (Advice) Did you select the correct binary for your device AMD/NVIDIA. (Advice) if linux AMD, are you in video and render groups?";
    case Vship_NoDeviceDetected:
        return "NoDeviceDetected: Vship found no device on your system. (Advice) Did you select the correct binary for your device AMD/NVIDIA. (Advice) if linux AMD, are you in video and render groups?";
    case Vship_BadDeviceArgument:
        return "BadDeviceArgument: Vship received a bad gpu_id argument either you specified a number >= to your gpu count, either it was negative";
    case Vship_BadDeviceCode:
        return "BadDeviceCode: Vship was unable to run a simple GPU Kernel. This usually indicate that the code was compiled for the wrong architecture. (Advice) Try to compile vship yourself, eventually replace --offload-arch=native to your arch";
    case Vship_BadHandler:
        return "BadHandler: The handler used was not allocated. This indicates an issue in Vship API Usage. Did you call the Init function or altered the handler id?";
    case Vship_BadPointer:
        return "BadPointer: The pointer passed as an argument was not valid and returned an error. (Advice) If this happened while trying to free, was it allocated using the same method and not modified?";
    default:
        return "BadErrorType: There was an unknown error";
    }
}

namespace {

std::mutex g_error_lock;
Error g_last_error(Vship_NoError, "Your Heart", 0, "");
int g_default_gpu = 0;

void set_global_error(const Error& e) {
    std::lock_guard<std::mutex> g(g_error_lock);
    g_last_error = e;
}

// Writes `s` into out (at most len-1 bytes + NUL) and returns the size the full text needs
// (src/VshipLib.cpp:151-167).
int copy_message(const std::string& s, char* out, int len) {
    if (len <= 0 || out == nullptr) return (int)s.size() + 1;
    const int n = std::min(len - 1, (int)s.size());
    std::memcpy(out, s.data(), (size_t)n);
    out[n] = '\0';
    return (int)s.size() + 1;
}

// One handler: its engine, device and last error.  `busy` turns concurrent use of one
// handler into an error.
template <typename EngineT>
struct Slot {
    std::unique_ptr<EngineT> engine;
    int gpu = 0;
    bool ready = false;
    std::atomic<bool> busy{false};
    std::mutex err_lock;
    Error last_error{Vship_NoError, "Your Heart", 0, ""};

    void set_error(const Error& e) {
        std::lock_guard<std::mutex> g(err_lock);
        last_error = e;
    }
};

// Id allocator with a free list, like RessourceManager (src/util/concurrency.hpp:175-200);
// slots are never moved, so a pointer taken under the lock stays valid while in use.
template <typename EngineT>
struct Table {
    std::mutex lock;
    std::vector<std::unique_ptr<Slot<EngineT>>> slots;
    std::vector<unsigned> free_ids;

    unsigned allocate() {
        std::lock_guard<std::mutex> g(lock);
        if (free_ids.empty()) {
            slots.emplace_back(new Slot<EngineT>());
            free_ids.push_back((unsigned)slots.size() - 1);
        }
        const unsigned id = free_ids.back();
        free_ids.pop_back();
        return id;
    }
    Slot<EngineT>* get(unsigned id) {
        std::lock_guard<std::mutex> g(lock);
        if (id >= slots.size()) return nullptr;
        return slots[id].get();
    }
    void release(unsigned id) {
        std::lock_guard<std::mutex> g(lock);
        free_ids.push_back(id);
    }
};

Table<Ssimu2Api> g_ssimu2;
Table<ButterApi> g_butter;
Table<Ssimu2BatchApi> g_batch;
Table<SurrogateApi> g_surrogate;
Table<CvvdpApi> g_cvvdp;

template <typename EngineT>
Vship_Exception fail(Slot<EngineT>* s, const Error& e) {
    if (s) s->set_error(e);
    set_global_error(e);
    return e.code;
}

// Runs fn on a live handler with the device selected and the busy flag held.
template <typename EngineT, typename Fn>
Vship_Exception with_handler(Table<EngineT>& table, unsigned id, const char* where, Fn fn) {
    Slot<EngineT>* s = table.get(id);
    if (s == nullptr || !s->ready) {
        set_global_error(Error(Vship_BadHandler, __FILE__, __LINE__,
                               std::string("Handler internal state in ") + where +
                                   " is not valid, did you allocate or use after free?"));
        return Vship_BadHandler;
    }
    bool expected = false;
    if (!s->busy.compare_exchange_strong(expected, true)) {
        return fail(s, Error(Vship_BadHandler, __FILE__, __LINE__,
                             std::string("handler used by two threads at once in ") + where));
    }
    Vship_Exception rc = Vship_NoError;
    try {
        CUDA_CHECK(cudaSetDevice(s->gpu));
        fn(*s);
#ifdef VSHIP_BOUNDS_CHECK
        check_guards(where);
#endif
    } catch (const Error& e) {
        rc = fail(s, e);
    } catch (const std::bad_alloc&) {
        rc = fail(s, Error(Vship_OutOfRAM, __FILE__, __LINE__, where));
    } catch (const std::exception& e) {
        rc = fail(s, Error(Vship_BadErrorType, __FILE__, __LINE__, e.what()));
    }
    s->busy.store(false);
    return rc;
}

int device_count_or_throw() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(Vship_DeviceCountError, __FILE__, __LINE__);
    }
    if (count == 0) throw Error(Vship_NoDeviceDetected, __FILE__, __LINE__);
    return count;
}

#ifdef VSHIP_BOUNDS_CHECK
constexpr size_t kGuardBytes = 64u << 10;

struct GuardedBlock {
    unsigned char* base;   // start of the lower guard band
    size_t bytes;          // payload bytes
    std::string what;
    int device;
};

std::mutex g_guard_lock;
std::vector<GuardedBlock> g_guarded;
unsigned* g_guard_flag[64] = {};

__global__ void guard_check_kernel(const unsigned char* lo, const unsigned char* hi, size_t n, unsigned* bad) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (lo[i] != 0xFFu || hi[i] != 0xFFu) atomicOr(bad, 1u);
}
#endif

__global__ void kernel_test(int* out) { out[0] = 4320984; }

// One-thread sanity kernel (src/util/gpuhelper.hpp:40-54).
bool kernel_check() {
    int host = 0;
    int* dev = nullptr;
    CUDA_CHECK(cudaMalloc(&dev, sizeof(int)));
    CUDA_CHECK(cudaMemset(dev, 0, sizeof(int)));
    kernel_test<<<1, 1>>>(dev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&host, dev, sizeof(int), cudaMemcpyDeviceToHost);
    (void)cudaFree(dev);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return host == 4320984;
}

#ifdef VSHIP_BOUNDS_CHECK
}  // namespace

void* guarded_alloc(size_t bytes, const char* what) {
    unsigned char* p = nullptr;
    if (cudaMalloc(&p, bytes + 2 * kGuardBytes) != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(Vship_OutOfVRAM, __FILE__, __LINE__, std::string("cudaMalloc failed for ") + what);
    }
    CUDA_CHECK(cudaMemset(p, 0xFF, bytes + 2 * kGuardBytes));
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(g_guard_lock);
    g_guarded.push_back(GuardedBlock{p, bytes, what, dev});
    return p + kGuardBytes;
}

void guarded_free(void* user) {
    if (!user) return;
    std::lock_guard<std::mutex> g(g_guard_lock);
    for (size_t i = 0; i < g_guarded.size(); i++)
        if (g_guarded[i].base + kGuardBytes == user) {
            (void)cudaFree(g_guarded[i].base);
            g_guarded.erase(g_guarded.begin() + (long)i);
            return;
        }
}

void check_guards(const char* where) {
    CUDA_CHECK(cudaDeviceSynchronize());
    int dev = 0;
    CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(g_guard_lock);
    if (dev < 0 || dev >= 64) return;
    if (!g_guard_flag[dev]) CUDA_CHECK(cudaMalloc(&g_guard_flag[dev], sizeof(unsigned)));
    for (const GuardedBlock& b : g_guarded) {
        if (b.device != dev) continue;
        CUDA_CHECK(cudaMemset(g_guard_flag[dev], 0, sizeof(unsigned)));
        guard_check_kernel<<<64, 256>>>(b.base, b.base + kGuardBytes + b.bytes, kGuardBytes, g_guard_flag[dev]);
        CUDA_CHECK(cudaGetLastError());
        unsigned bad = 0;
        CUDA_CHECK(cudaMemcpy(&bad, g_guard_flag[dev], sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (bad)
            throw Error(Vship_HIPError, __FILE__, __LINE__,
                        std::string("a kernel wrote past the bounds of ") + b.what + " (found after " + where + ")");
    }
}

namespace {
#endif

template <typename EngineT, typename InitFn>
Vship_Exception init_handler(Table<EngineT>& table, unsigned* id_out, int gpu, InitFn init) {
    const unsigned id = table.allocate();
    *id_out = id;
    Slot<EngineT>* s = table.get(id);
    s->gpu = gpu;
    s->ready = false;
    s->engine.reset();
    try {
        CUDA_CHECK(cudaSetDevice(gpu));
        init(*s);
        s->ready = true;
    } catch (const Error& e) {
        s->engine.reset();
        s->ready = true;  // as in the reference, the id stays allocated until *Free
        s->set_error(e);
        set_global_error(e);
        return e.code;
    } catch (const std::bad_alloc&) {
        s->engine.reset();
        s->ready = true;
        Error e(Vship_OutOfRAM, __FILE__, __LINE__, "while creating a handler");
        s->set_error(e);
        set_global_error(e);
        return e.code;
    }
    return Vship_NoError;
}

template <typename EngineT>
Vship_Exception free_handler(Table<EngineT>& table, unsigned id, const char* where) {
    Slot<EngineT>* s = table.get(id);
    if (s == nullptr || !s->ready) {
        set_global_error(Error(Vship_BadHandler, __FILE__, __LINE__,
                               std::string("Handler internal state in ") + where +
                                   " is not valid, did you allocate or use after free?"));
        return Vship_BadHandler;
    }
    bool expected = false;
    if (!s->busy.compare_exchange_strong(expected, true))
        return fail(s, Error(Vship_BadHandler, __FILE__, __LINE__, std::string("handler in use during ") + where));
    Vship_Exception rc = Vship_NoError;
    try {
        CUDA_CHECK(cudaSetDevice(s->gpu));
        s->engine.reset();
    } catch (const Error& e) {
        rc = fail(s, e);
    }
    s->ready = false;
    s->busy.store(false);
    table.release(id);
    return rc;
}

template <typename EngineT>
int handler_error(Table<EngineT>& table, unsigned id, char* out, int len, const char* where) {
    Slot<EngineT>* s = table.get(id);
    if (s == nullptr || !s->ready) {
        set_global_error(Error(Vship_BadHandler, __FILE__, __LINE__,
                               std::string("Handler internal state in ") + where +
                                   " is not valid, did you allocate or use after free?"));
        return 0;
    }
    std::string msg;
    {
        std::lock_guard<std::mutex> g(s->err_lock);
        msg = s->last_error.message();
    }
    return copy_message(msg, out, len);
}

void require_engine(bool ok) {
    if (!ok) throw Error(Vship_BadHandler, __FILE__, __LINE__, "handler initialisation had failed");
}

template <typename EngineT>
int kernel_times(Table<EngineT>& table, unsigned id, VshipExt_KernelTime* out, int max, int reset) {
    int count = 0;
    Vship_Exception rc = with_handler(table, id, "kernel timing", [&](Slot<EngineT>& s) {
        require_engine((bool)s.engine);
        KernelTimer& t = s.engine->timer();
        t.collect();
        for (int k = 0; k < KernelTimer::kSlots; k++) {
            if (t.launches[k] == 0) continue;
            if (out && count < max) {
                std::memset(out[count].name, 0, sizeof(out[count].name));
                std::strncpy(out[count].name, t.names[k] ? t.names[k] : "", sizeof(out[count].name) - 1);
                out[count].launches = t.launches[k];
                out[count].total_ms = t.total_ms[k];
            }
            count++;
        }
        if (reset) t.reset();
    });
    return rc == Vship_NoError ? count : -1;
}

}  // namespace

void record_global_error(const Error& e) { set_global_error(e); }

}  // namespace vship

using namespace vship;

extern "C" {

Vship_Version Vship_GetVersion(void) {
    Vship_Version v;
    v.major = 4;
    v.minor = 1;
    v.minorMinor = 0;
    v.backend = Vship_Cuda;
    return v;
}

Vship_Exception Vship_GetDeviceCount(int* number) {
    try {
        const int n = device_count_or_throw();
        if (number) *number = n;
    } catch (const Error& e) {
        set_global_error(e);
        return e.code;
    }
    return Vship_NoError;
}

Vship_Exception Vship_SetDevice(int gpu_id) {
    int n = 0;
    const Vship_Exception rc = Vship_GetDeviceCount(&n);
    if (rc != Vship_NoError) return rc;
    if (gpu_id < 0 || gpu_id >= n) {
        set_global_error(Error(Vship_BadDeviceArgument, __FILE__, __LINE__, "In Vship_SetDevice"));
        return Vship_BadDeviceArgument;
    }
    g_default_gpu = gpu_id;
    return Vship_NoError;
}

Vship_Exception Vship_GetDeviceInfo(Vship_DeviceInfo* info, int gpu_id) {
    try {
        const int n = device_count_or_throw();
        if (gpu_id < 0 || gpu_id >= n) throw Error(Vship_BadDeviceArgument, __FILE__, __LINE__, "while using Vship_GetDeviceInfo");
        if (info == nullptr) throw Error(Vship_BadPointer, __FILE__, __LINE__, "device_info is NULL");
        cudaDeviceProp prop;
        CUDA_CHECK(cudaGetDeviceProperties(&prop, gpu_id));
        std::memcpy(info->name, prop.name, 256);
        info->VRAMSize = (uint64_t)prop.totalGlobalMem;
        info->integrated = prop.integrated;
        info->MultiProcessorCount = prop.multiProcessorCount;
        info->WarpSize = prop.warpSize;
    } catch (const Error& e) {
        set_global_error(e);
        return e.code;
    }
    return Vship_NoError;
}

Vship_Exception Vship_GPUFullCheck(int gpu_id) {
    try {
        const int n = device_count_or_throw();
        if (gpu_id < 0 || gpu_id >= n) throw Error(Vship_BadDeviceArgument, __FILE__, __LINE__);
        CUDA_CHECK(cudaSetDevice(gpu_id));
        if (!kernel_check()) throw Error(Vship_BadDeviceCode, __FILE__, __LINE__);
    } catch (const Error& e) {
        set_global_error(e);
        return e.code;
    }
    return Vship_NoError;
}

int Vship_GetErrorMessage(Vship_Exception exception, char* out_message, int len) {
    return copy_message(error_text(exception), out_message, len);
}

int Vship_GetDetailedLastError(char* out_message, int len) {
    std::string msg;
    {
        std::lock_guard<std::mutex> g(g_error_lock);
        msg = g_last_error.message();
    }
    return copy_message(msg, out_message, len);
}

Vship_Exception Vship_PinnedMalloc(void** ptr, uint64_t size) {
    if (ptr == nullptr || cudaMallocHost(ptr, size) != cudaSuccess) {
        (void)cudaGetLastError();
        set_global_error(Error(Vship_OutOfRAM, __FILE__, __LINE__, "In Vship_PinnedMalloc"));
        return Vship_OutOfRAM;
    }
    return Vship_NoError;
}

Vship_Exception Vship_PinnedFree(void* ptr) {
    if (cudaFreeHost(ptr) != cudaSuccess) {
        (void)cudaGetLastError();
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__,
                               "Failed to call hipHostFree on pointer given to Vship_PinnedFree"));
        return Vship_BadPointer;
    }
    return Vship_NoError;
}

// ---------------------------------------------------------------- SSIMULACRA2

Vship_Exception Vship_SSIMU2Init2(Vship_SSIMU2Handler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis, int gpu_id) {
    if (handler == nullptr) {
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__, "handler is NULL"));
        return Vship_BadPointer;
    }
    return init_handler(g_ssimu2, &handler->id, gpu_id, [&](Slot<Ssimu2Api>& s) {
        s.engine.reset(make_ssimu2_engine());
        s.engine->init(src, dis, gpu_id);
    });
}

Vship_Exception Vship_SSIMU2Init(Vship_SSIMU2Handler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis) {
    return Vship_SSIMU2Init2(handler, src, dis, g_default_gpu);
}

Vship_Exception Vship_SSIMU2Free(Vship_SSIMU2Handler handler) { return free_handler(g_ssimu2, handler.id, "Vship_SSIMU2Free"); }

Vship_Exception Vship_ComputeSSIMU2(Vship_SSIMU2Handler handler, double* score, const uint8_t* srcp1[3], const uint8_t* srcp2[3],
                                    const int64_t lineSize[3], const int64_t lineSize2[3]) {
    return with_handler(g_ssimu2, handler.id, "Vship_ComputeSSIMU2", [&](Slot<Ssimu2Api>& s) {
        require_engine((bool)s.engine);
        if (!score || !srcp1 || !srcp2 || !lineSize || !lineSize2) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        *score = s.engine->compute(srcp1, srcp2, lineSize, lineSize2);
    });
}

int Vship_SSIMU2GetDetailedLastError(Vship_SSIMU2Handler handler, char* out_message, int len) {
    return handler_error(g_ssimu2, handler.id, out_message, len, "Vship_SSIMU2GetDetailedLastError");
}

// ---------------------------------------------------------------- Butteraugli

Vship_Exception Vship_ButteraugliInit2(Vship_ButteraugliHandler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis,
                                       int Qnorm, float intensity_multiplier, int gpu_id) {
    if (handler == nullptr) {
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__, "handler is NULL"));
        return Vship_BadPointer;
    }
    return init_handler(g_butter, &handler->id, gpu_id, [&](Slot<ButterApi>& s) {
        s.engine.reset(make_butter_engine());
        s.engine->init(src, dis, Qnorm, intensity_multiplier, gpu_id);
    });
}

Vship_Exception Vship_ButteraugliInit(Vship_ButteraugliHandler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis,
                                      int Qnorm, float intensity_multiplier) {
    return Vship_ButteraugliInit2(handler, src, dis, Qnorm, intensity_multiplier, g_default_gpu);
}

Vship_Exception Vship_ButteraugliFree(Vship_ButteraugliHandler handler) {
    return free_handler(g_butter, handler.id, "Vship_ButteraugliFree");
}

Vship_Exception Vship_ComputeButteraugli(Vship_ButteraugliHandler handler, Vship_ButteraugliScore* score, const uint8_t* dstp,
                                         int64_t dststride, const uint8_t* srcp1[3], const uint8_t* srcp2[3],
                                         const int64_t lineSize[3], const int64_t lineSize2[3]) {
    return with_handler(g_butter, handler.id, "Vship_ComputeButteraugli", [&](Slot<ButterApi>& s) {
        require_engine((bool)s.engine);
        if (!score || !srcp1 || !srcp2 || !lineSize || !lineSize2) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        double norms[3];
        s.engine->compute(norms, const_cast<uint8_t*>(dstp), dststride, srcp1, srcp2, lineSize, lineSize2);
        score->normQ = norms[0];
        score->norm3 = norms[1];
        score->norminf = norms[2];
    });
}

int Vship_ButteraugliGetDetailedLastError(Vship_ButteraugliHandler handler, char* out_message, int len) {
    return handler_error(g_butter, handler.id, out_message, len, "Vship_ButteraugliGetDetailedLastError");
}

// ---------------------------------------------------------------- CVVDP

Vship_Exception Vship_CVVDPInit3(Vship_CVVDPHandler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis, float fps,
                                 bool resizeToDisplay, const char* model_key_cstr, const char* model_config_json_cstr,
                                 int gpu_id) {
    if (handler == nullptr || model_key_cstr == nullptr) {
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__, handler ? "model key is NULL" : "handler is NULL"));
        return Vship_BadPointer;
    }
    const std::string key(model_key_cstr);
    const std::string json(model_config_json_cstr ? model_config_json_cstr : "");
    return init_handler(g_cvvdp, &handler->id, gpu_id, [&](Slot<CvvdpApi>& s) {
        s.engine.reset(make_cvvdp_engine());
        s.engine->init(src, dis, fps, resizeToDisplay, key, json, gpu_id);
    });
}

Vship_Exception Vship_CVVDPInit2(Vship_CVVDPHandler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis, float fps,
                                 bool resizeToDisplay, const char* model_key_cstr, const char* model_config_json_cstr) {
    return Vship_CVVDPInit3(handler, src, dis, fps, resizeToDisplay, model_key_cstr, model_config_json_cstr, g_default_gpu);
}

Vship_Exception Vship_CVVDPInit(Vship_CVVDPHandler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis, float fps,
                                bool resizeToDisplay, const char* model_key_cstr) {
    return Vship_CVVDPInit2(handler, src, dis, fps, resizeToDisplay, model_key_cstr, nullptr);
}

Vship_Exception Vship_CVVDPFree(Vship_CVVDPHandler handler) { return free_handler(g_cvvdp, handler.id, "Vship_CVVDPFree"); }

Vship_Exception Vship_CVVDPGetDistmapResolution(Vship_CVVDPHandler handler, int64_t* width, int64_t* height) {
    return with_handler(g_cvvdp, handler.id, "Vship_CVVDPGetDistmapResolution", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        if (width) *width = s.engine->distmap_width();
        if (height) *height = s.engine->distmap_height();
    });
}

Vship_Exception Vship_ResetCVVDP(Vship_CVVDPHandler handler) {
    return with_handler(g_cvvdp, handler.id, "Vship_ResetCVVDP", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        s.engine->reset(false);
    });
}

Vship_Exception Vship_ResetScoreCVVDP(Vship_CVVDPHandler handler) {
    return with_handler(g_cvvdp, handler.id, "Vship_ResetScoreCVVDP", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        s.engine->reset(true);
    });
}

Vship_Exception Vship_LoadTemporalCVVDP(Vship_CVVDPHandler handler, const uint8_t* srcp1[3], const uint8_t* srcp2[3],
                                        const int64_t lineSize[3], const int64_t lineSize2[3]) {
    return with_handler(g_cvvdp, handler.id, "Vship_LoadTemporalCVVDP", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        if (!srcp1 || !srcp2 || !lineSize || !lineSize2) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->load_temporal(srcp1, srcp2, lineSize, lineSize2);
    });
}

Vship_Exception Vship_ComputeCVVDP(Vship_CVVDPHandler handler, double* score, const uint8_t* dstp, int64_t dststride,
                                   const uint8_t* srcp1[3], const uint8_t* srcp2[3], const int64_t lineSize[3],
                                   const int64_t lineSize2[3]) {
    return with_handler(g_cvvdp, handler.id, "Vship_ComputeCVVDP", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        if (!score || !srcp1 || !srcp2 || !lineSize || !lineSize2) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        *score = s.engine->compute(const_cast<uint8_t*>(dstp), dststride, srcp1, srcp2, lineSize, lineSize2);
    });
}

int Vship_CVVDPGetDetailedLastError(Vship_CVVDPHandler handler, char* out_message, int len) {
    return handler_error(g_cvvdp, handler.id, out_message, len, "Vship_CVVDPGetDetailedLastError");
}

// ---------------------------------------------------------------- extensions

Vship_Exception VshipExt_ComputeSSIMU2Device(Vship_SSIMU2Handler handler, int n, double* d_scores, float* d_features,
                                             const uint8_t* const* srcp1, const uint8_t* const* srcp2,
                                             const int64_t lineSize[3], const int64_t lineSize2[3], void* stream) {
    return with_handler(g_ssimu2, handler.id, "VshipExt_ComputeSSIMU2Device", [&](Slot<Ssimu2Api>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative pair count");
        if (n > 0 && (!d_scores || !srcp1 || !srcp2 || !lineSize || !lineSize2))
            throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->compute_device(n, srcp1, srcp2, lineSize, lineSize2, d_scores, d_features, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SSIMU2LastFeatures(Vship_SSIMU2Handler handler, float features[108]) {
    return with_handler(g_ssimu2, handler.id, "VshipExt_SSIMU2LastFeatures", [&](Slot<Ssimu2Api>& s) {
        require_engine((bool)s.engine);
        if (!features) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->last_features(features);
    });
}

Vship_Exception VshipExt_ComputeButteraugliDevice(Vship_ButteraugliHandler handler, double* d_norms, float* d_distmap,
                                                  int64_t dststride, const uint8_t* const srcp1[3],
                                                  const uint8_t* const srcp2[3], const int64_t lineSize[3],
                                                  const int64_t lineSize2[3], void* stream) {
    return with_handler(g_butter, handler.id, "VshipExt_ComputeButteraugliDevice", [&](Slot<ButterApi>& s) {
        require_engine((bool)s.engine);
        if (!d_norms || !srcp1 || !srcp2 || !lineSize || !lineSize2) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->compute_device(d_norms, d_distmap, dststride, srcp1, srcp2, lineSize, lineSize2, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SSIMU2KernelTiming(Vship_SSIMU2Handler handler, int enable) {
    return with_handler(g_ssimu2, handler.id, "VshipExt_SSIMU2KernelTiming", [&](Slot<Ssimu2Api>& s) {
        require_engine((bool)s.engine);
        s.engine->timer().enable(enable != 0);
    });
}

int VshipExt_SSIMU2KernelTimes(Vship_SSIMU2Handler handler, VshipExt_KernelTime* out, int max, int reset) {
    return kernel_times(g_ssimu2, handler.id, out, max, reset);
}

Vship_Exception VshipExt_ButteraugliKernelTiming(Vship_ButteraugliHandler handler, int enable) {
    return with_handler(g_butter, handler.id, "VshipExt_ButteraugliKernelTiming", [&](Slot<ButterApi>& s) {
        require_engine((bool)s.engine);
        s.engine->timer().enable(enable != 0);
    });
}

int VshipExt_ButteraugliKernelTimes(Vship_ButteraugliHandler handler, VshipExt_KernelTime* out, int max, int reset) {
    return kernel_times(g_butter, handler.id, out, max, reset);
}

Vship_Exception VshipExt_ButteraugliTestTmaTimeout(Vship_ButteraugliHandler handler) {
    return with_handler(g_butter, handler.id, "VshipExt_ButteraugliTestTmaTimeout", [&](Slot<ButterApi>& s) {
        require_engine((bool)s.engine);
        if (!s.engine->test_tma_timeout())
            throw Error(Vship_BadDeviceArgument, __FILE__, __LINE__,
                        "this handler's resolution does not use the tensor-map column pass");
    });
}

Vship_Exception VshipExt_SSIMU2Resolution(Vship_SSIMU2Handler handler, int64_t* width, int64_t* height) {
    return with_handler(g_ssimu2, handler.id, "VshipExt_SSIMU2Resolution", [&](Slot<Ssimu2Api>& s) {
        require_engine((bool)s.engine);
        if (width) *width = s.engine->width();
        if (height) *height = s.engine->height();
    });
}

Vship_Exception VshipExt_ButteraugliResolution(Vship_ButteraugliHandler handler, int64_t* width, int64_t* height) {
    return with_handler(g_butter, handler.id, "VshipExt_ButteraugliResolution", [&](Slot<ButterApi>& s) {
        require_engine((bool)s.engine);
        if (width) *width = s.engine->width();
        if (height) *height = s.engine->height();
    });
}

Vship_Exception VshipExt_CVVDPDisplayModel(const char* model_key, const char* model_config_json, VshipExt_CVVDPDisplay* out) {
    if (model_key == nullptr || out == nullptr) {
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument"));
        return Vship_BadPointer;
    }
    try {
        cvvdp_display_model(model_key, model_config_json ? model_config_json : "", out);
    } catch (const Error& e) {
        set_global_error(e);
        return e.code;
    }
    return Vship_NoError;
}

Vship_Exception VshipExt_CVVDPGeometry(Vship_CVVDPHandler handler, int* bands, int* ring_frames) {
    return with_handler(g_cvvdp, handler.id, "VshipExt_CVVDPGeometry", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        if (bands) *bands = s.engine->bands();
        if (ring_frames) *ring_frames = s.engine->ring_frames();
    });
}

Vship_Exception VshipExt_CVVDPKernelTiming(Vship_CVVDPHandler handler, int enable) {
    return with_handler(g_cvvdp, handler.id, "VshipExt_CVVDPKernelTiming", [&](Slot<CvvdpApi>& s) {
        require_engine((bool)s.engine);
        s.engine->timer().enable(enable != 0);
    });
}

int VshipExt_CVVDPKernelTimes(Vship_CVVDPHandler handler, VshipExt_KernelTime* out, int max, int reset) {
    return kernel_times(g_cvvdp, handler.id, out, max, reset);
}

// ---------------------------------------------------------------- uneven batches

Vship_Exception VshipExt_SSIMU2BatchInit(VshipExt_SSIMU2BatchHandler* handler, int gpu_id) {
    if (handler == nullptr) {
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__, "handler is NULL"));
        return Vship_BadPointer;
    }
    return init_handler(g_batch, &handler->id, gpu_id, [&](Slot<Ssimu2BatchApi>& s) {
        s.engine.reset(make_ssimu2_batch_engine());
        s.engine->init(gpu_id);
    });
}

Vship_Exception VshipExt_SSIMU2BatchFree(VshipExt_SSIMU2BatchHandler handler) {
    return free_handler(g_batch, handler.id, "VshipExt_SSIMU2BatchFree");
}

int VshipExt_SSIMU2BatchGetDetailedLastError(VshipExt_SSIMU2BatchHandler handler, char* out_message, int len) {
    return handler_error(g_batch, handler.id, out_message, len, "VshipExt_SSIMU2BatchGetDetailedLastError");
}

Vship_Exception VshipExt_ComputeSSIMU2BatchDevice(VshipExt_SSIMU2BatchHandler handler, int n, const VshipExt_FramePair* pairs,
                                                  double* d_scores, float* d_features, void* stream) {
    return with_handler(g_batch, handler.id, "VshipExt_ComputeSSIMU2BatchDevice", [&](Slot<Ssimu2BatchApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative pair count");
        if (n > 0 && (!pairs || !d_scores)) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->compute_device(n, pairs, d_scores, d_features, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_ComputeSSIMU2Batch(VshipExt_SSIMU2BatchHandler handler, int n, const VshipExt_FramePair* pairs,
                                            double* scores, float* features) {
    return with_handler(g_batch, handler.id, "VshipExt_ComputeSSIMU2Batch", [&](Slot<Ssimu2BatchApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative pair count");
        if (n > 0 && (!pairs || !scores)) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->compute(n, pairs, scores, features);
    });
}

Vship_Exception VshipExt_SSIMU2BatchSetTileRows(VshipExt_SSIMU2BatchHandler handler, int rows) {
    return with_handler(g_batch, handler.id, "VshipExt_SSIMU2BatchSetTileRows", [&](Slot<Ssimu2BatchApi>& s) {
        require_engine((bool)s.engine);
        s.engine->set_tile_rows(rows);
    });
}

Vship_Exception VshipExt_SSIMU2BatchTileRows(VshipExt_SSIMU2BatchHandler handler, int* rows) {
    return with_handler(g_batch, handler.id, "VshipExt_SSIMU2BatchTileRows", [&](Slot<Ssimu2BatchApi>& s) {
        require_engine((bool)s.engine);
        if (!rows) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        *rows = s.engine->tile_rows();
    });
}

Vship_Exception VshipExt_SSIMU2BatchTestHoldFrontTile(VshipExt_SSIMU2BatchHandler handler) {
    return with_handler(g_batch, handler.id, "VshipExt_SSIMU2BatchTestHoldFrontTile", [&](Slot<Ssimu2BatchApi>& s) {
        require_engine((bool)s.engine);
        s.engine->hold_front_tile();
    });
}

Vship_Exception VshipExt_SSIMU2BatchKernelTiming(VshipExt_SSIMU2BatchHandler handler, int enable) {
    return with_handler(g_batch, handler.id, "VshipExt_SSIMU2BatchKernelTiming", [&](Slot<Ssimu2BatchApi>& s) {
        require_engine((bool)s.engine);
        s.engine->timer().enable(enable != 0);
    });
}

int VshipExt_SSIMU2BatchKernelTimes(VshipExt_SSIMU2BatchHandler handler, VshipExt_KernelTime* out, int max, int reset) {
    return kernel_times(g_batch, handler.id, out, max, reset);
}

// ---------------------------------------------------------------- learned surrogate

Vship_Exception VshipExt_SurrogateInit(VshipExt_SurrogateHandler* handler, Vship_Colorspace_t src, Vship_Colorspace_t dis,
                                       int gpu_id) {
    if (handler == nullptr) {
        set_global_error(Error(Vship_BadPointer, __FILE__, __LINE__, "handler is NULL"));
        return Vship_BadPointer;
    }
    return init_handler(g_surrogate, &handler->id, gpu_id, [&](Slot<SurrogateApi>& s) {
        s.engine.reset(make_surrogate_engine());
        s.engine->init(src, dis, gpu_id);
    });
}

Vship_Exception VshipExt_SurrogateFree(VshipExt_SurrogateHandler handler) {
    return free_handler(g_surrogate, handler.id, "VshipExt_SurrogateFree");
}

int VshipExt_SurrogateGetDetailedLastError(VshipExt_SurrogateHandler handler, char* out_message, int len) {
    return handler_error(g_surrogate, handler.id, out_message, len, "VshipExt_SurrogateGetDetailedLastError");
}

Vship_Exception VshipExt_SurrogateInputSize(VshipExt_SurrogateHandler handler, int64_t* elems) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateInputSize", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (!elems) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        *elems = s.engine->input_elems();
    });
}

Vship_Exception VshipExt_SurrogateInputs(VshipExt_SurrogateHandler handler, int n, const uint8_t* const* srcp1,
                                         const uint8_t* const* srcp2, const int64_t lineSize[3], const int64_t lineSize2[3],
                                         void* d_inputs, void* stream) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateInputs", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative pair count");
        if (n > 0 && (!srcp1 || !srcp2 || !lineSize || !lineSize2 || !d_inputs))
            throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->inputs(n, srcp1, srcp2, lineSize, lineSize2, d_inputs, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SurrogatePredictInputs(VshipExt_SurrogateHandler handler, int n, const void* d_inputs,
                                                float* d_pred, void* stream) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogatePredictInputs", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative sample count");
        if (n > 0 && (!d_inputs || !d_pred)) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->predict_inputs(n, d_inputs, d_pred, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SurrogatePredict(VshipExt_SurrogateHandler handler, int n, const uint8_t* const* srcp1,
                                          const uint8_t* const* srcp2, const int64_t lineSize[3],
                                          const int64_t lineSize2[3], float* d_pred, void* stream) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogatePredict", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative pair count");
        if (n > 0 && (!srcp1 || !srcp2 || !lineSize || !lineSize2 || !d_pred))
            throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->predict(n, srcp1, srcp2, lineSize, lineSize2, d_pred, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SurrogateReferenceSize(VshipExt_SurrogateHandler handler, int64_t* floats) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateReferenceSize", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (!floats) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        *floats = s.engine->reference_floats();
    });
}

Vship_Exception VshipExt_SurrogateReferences(VshipExt_SurrogateHandler handler, int n, const uint8_t* const* srcp1,
                                             const int64_t lineSize[3], float* d_refs, void* stream) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateReferences", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative frame count");
        if (n > 0 && (!srcp1 || !lineSize || !d_refs)) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->references(n, srcp1, lineSize, d_refs, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SurrogatePredictAgainst(VshipExt_SurrogateHandler handler, int n, const float* d_refs,
                                                 const uint8_t* const* srcp2, const int64_t lineSize2[3], float* d_pred,
                                                 void* stream) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogatePredictAgainst", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (n < 0) throw Error(Vship_BadPointer, __FILE__, __LINE__, "negative pair count");
        if (n > 0 && (!d_refs || !srcp2 || !lineSize2 || !d_pred))
            throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->predict_against(n, d_refs, srcp2, lineSize2, d_pred, (cudaStream_t)stream);
    });
}

Vship_Exception VshipExt_SurrogateTrain(VshipExt_SurrogateHandler handler, int n, const void* d_inputs,
                                        const float* d_targets, int epochs, int batch, float lr, unsigned seed,
                                        float* loss_history) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateTrain", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (!d_inputs || !d_targets) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->train(n, d_inputs, d_targets, epochs, batch, lr, seed, loss_history);
    });
}

Vship_Exception VshipExt_SurrogateGradients(VshipExt_SurrogateHandler handler, int n, const void* d_inputs,
                                            const float* d_targets, float* grads, double* loss) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateGradients", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (n < 1 || !d_inputs || !d_targets) throw Error(Vship_BadPointer, __FILE__, __LINE__, "bad argument");
        const double l = s.engine->gradients(n, d_inputs, d_targets, grads);
        if (loss) *loss = l;
    });
}

int VshipExt_SurrogateModel(VshipExt_SurrogateHandler handler, float* out, int max) {
    int count = -1;
    Vship_Exception rc = with_handler(g_surrogate, handler.id, "VshipExt_SurrogateModel", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        count = s.engine->get_model(out, max);
    });
    return rc == Vship_NoError ? count : -1;
}

Vship_Exception VshipExt_SurrogateSetModel(VshipExt_SurrogateHandler handler, const float* model, int count) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateSetModel", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        if (!model) throw Error(Vship_BadPointer, __FILE__, __LINE__, "NULL argument");
        s.engine->set_model(model, count);
    });
}

Vship_Exception VshipExt_SurrogateKernelTiming(VshipExt_SurrogateHandler handler, int enable) {
    return with_handler(g_surrogate, handler.id, "VshipExt_SurrogateKernelTiming", [&](Slot<SurrogateApi>& s) {
        require_engine((bool)s.engine);
        s.engine->timer().enable(enable != 0);
    });
}

int VshipExt_SurrogateKernelTimes(VshipExt_SurrogateHandler handler, VshipExt_KernelTime* out, int max, int reset) {
    return kernel_times(g_surrogate, handler.id, out, max, reset);
}

#ifdef VSHIP_BOUNDS_CHECK
// Bounds-check build only: checks the guard-band checker itself on the current device.  It
// allocates a guarded 1 KiB buffer and, when `corrupt` is non-zero, changes one byte of its
// upper guard band from the host (cudaMemset inside the allocation: no kernel steps out of
// bounds), then runs the guard check.  Returns its code: Vship_NoError for an intact band,
// Vship_HIPError when the change was found.
__attribute__((visibility("default"))) Vship_Exception VshipExt_BoundsCheckProbe(int corrupt) {
    unsigned char* p = nullptr;
    Vship_Exception rc = Vship_NoError;
    try {
        p = static_cast<unsigned char*>(guarded_alloc(1024, "the probe buffer"));
        if (corrupt) CUDA_CHECK(cudaMemset(p + 1024 + 100, 0x00, 1));
        check_guards("VshipExt_BoundsCheckProbe");
    } catch (const Error& e) {
        set_global_error(e);
        rc = e.code;
    }
    guarded_free(p);
    return rc;
}
#endif

}  // extern "C"

// Shared host/device utilities of the B200 Vship engine: error type, CUDA checks, small
// math helpers.  Everything here is internal; the public surface is include/VshipAPI.h.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <sstream>

#include "../../include/VshipAPI.h"

namespace vship {

// Generic text of each error code.  The wording is part of the observable API (callers
// parse it), so it follows the reference's errorMessage() (src/util/VshipExceptions.hpp:41-92).
const char* error_text(int code);

// An error raised inside the engine: code, origin and free-form detail.  getMessage()
// produces the same layout as the reference's VshipError::getErrorMessage
// (src/util/VshipExceptions.hpp:104-112): header line, generic text, origin line, detail.
struct Error {
    Vship_Exception code = Vship_NoError;
    std::string file = "";
    int line = 0;
    std::string detail = "";

    Error() = default;
    Error(Vship_Exception c, const char* f, int l, std::string d = "") : code(c), file(f), line(l), detail(std::move(d)) {}

    std::string message() const {
        std::ostringstream ss;
        ss << "VshipException\n" << error_text(code) << "\n - At line " << line << " of " << file << "\n";
        if (!detail.empty()) ss << "Detail: " << detail << "\n";
        return ss.str();
    }
};

#define VSHIP_THROW(code, detail) throw ::vship::Error((code), __FILE__, __LINE__, (detail))

#define CUDA_CHECK(expr)                                                                    \
    do {                                                                                    \
        cudaError_t err_ = (expr);                                                          \
        if (err_ != cudaSuccess) {                                                          \
            (void)cudaGetLastError();                                                       \
            throw ::vship::Error(Vship_HIPError, __FILE__, __LINE__, cudaGetErrorString(err_)); \
        }                                                                                   \
    } while (0)

#ifdef VSHIP_BOUNDS_CHECK
// Bounds-check build (the stand-in for compute-sanitizer, which is not available on the GPU
// pool): every device buffer the engines allocate gets a 64 KiB guard band on each side, and
// the buffer and its guards start filled with 0xFF bytes (a NaN in every float and double).
// A kernel that writes past either end of a buffer leaves a guard byte changed, which
// check_guards() finds after each API call and reports as Vship_HIPError; a kernel that reads
// past an end, or reads a float it never wrote, carries a NaN into the scores.  Defined in
// api.cu.
void* guarded_alloc(size_t bytes, const char* what);
void guarded_free(void* p);
void check_guards(const char* where);
#endif

// Device allocation that reports OutOfVRAM like the reference (src/ssimu2/main.hpp:127-133).
template <typename T>
inline T* device_alloc(size_t count, const char* what) {
#ifdef VSHIP_BOUNDS_CHECK
    return static_cast<T*>(guarded_alloc((count ? count : 1) * sizeof(T), what));
#endif
    void* p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(Vship_OutOfVRAM, __FILE__, __LINE__, std::string("cudaMalloc failed for ") + what);
    }
    return static_cast<T*>(p);
}

template <typename T>
inline T* pinned_alloc(size_t count, const char* what) {
    void* p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocHost(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(Vship_OutOfRAM, __FILE__, __LINE__, std::string("cudaMallocHost failed for ") + what);
    }
    return static_cast<T*>(p);
}

inline void device_free(void* p) {
#ifdef VSHIP_BOUNDS_CHECK
    guarded_free(p);
    return;
#endif
    if (p) (void)cudaFree(p);
}

inline void pinned_free(void* p) {
    if (p) (void)cudaFreeHost(p);
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Optional per-kernel CUDA-event timing, used by bench.py to compute a kernel's achieved
// bandwidth from its own launch durations.  Disabled by default (no events recorded).
struct KernelTimer {
    static constexpr int kSlots = 8;
    bool enabled = false;
    const char* names[kSlots] = {};
    int launches[kSlots] = {};
    double total_ms[kSlots] = {};
    cudaEvent_t pending_start[64];
    cudaEvent_t pending_stop[64];
    int pending_slot[64];
    int npending = 0;
    bool created = false;

    void enable(bool on) {
        if (on && !created) {
            for (int i = 0; i < 64; i++) {
                CUDA_CHECK(cudaEventCreate(&pending_start[i]));
                CUDA_CHECK(cudaEventCreate(&pending_stop[i]));
            }
            created = true;
        }
        enabled = on;
    }
    void destroy() {
        if (!created) return;
        for (int i = 0; i < 64; i++) {
            (void)cudaEventDestroy(pending_start[i]);
            (void)cudaEventDestroy(pending_stop[i]);
        }
        created = false;
    }
    // Starts timing slot `slot` on `stream`; returns the pending index or -1.
    int begin(int slot, const char* name, cudaStream_t stream) {
        if (!enabled) return -1;
        if (npending == 64) collect();
        names[slot] = name;
        int i = npending++;
        pending_slot[i] = slot;
        CUDA_CHECK(cudaEventRecord(pending_start[i], stream));
        return i;
    }
    void end(int i, cudaStream_t stream) {
        if (i < 0) return;
        CUDA_CHECK(cudaEventRecord(pending_stop[i], stream));
    }
    // Folds all recorded intervals into the totals (synchronises on the events).
    void collect() {
        for (int i = 0; i < npending; i++) {
            float ms = 0.f;
            CUDA_CHECK(cudaEventSynchronize(pending_stop[i]));
            CUDA_CHECK(cudaEventElapsedTime(&ms, pending_start[i], pending_stop[i]));
            launches[pending_slot[i]] += 1;
            total_ms[pending_slot[i]] += ms;
        }
        npending = 0;
    }
    void reset() {
        collect();
        for (int s = 0; s < kSlots; s++) { launches[s] = 0; total_ms[s] = 0; }
    }
};

}  // namespace vship

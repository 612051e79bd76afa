/*
 * VshipAPI_ext.h -- additions of the B200 engine to the Vship C ABI.
 *
 * None of these entry points exists in the reference library; they are additive and never
 * change the behaviour of the functions in VshipAPI.h.  They serve callers that keep frames
 * in device memory (a decoder writing to the GPU, a batch scorer) and the benchmark, which
 * needs per-kernel timings.
 */
#ifndef VSHIP_B200_API_EXT_H
#define VSHIP_B200_API_EXT_H

#include "VshipAPI.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Scores n frame pairs whose planes are already in device memory of the handler's GPU.
 * srcp1 and srcp2 are host arrays of 3*n device plane pointers (pair i uses entries 3i..3i+2),
 * with the same byte strides for every pair.  Work is queued on `stream` (a cudaStream_t;
 * NULL is the CUDA legacy default stream) and the call returns without waiting: d_scores (device,
 * n doubles) and d_features (device, n*108 floats, may be NULL) are valid once the stream has
 * reached this point.  Up to 64 pairs run in one launch of each kernel. */
EXPORTPREPROCESS Vship_Exception VshipExt_ComputeSSIMU2Device(Vship_SSIMU2Handler handler, int n, double* d_scores,
                                                               float* d_features, const uint8_t* const* srcp1,
                                                               const uint8_t* const* srcp2, const int64_t lineSize[3],
                                                               const int64_t lineSize2[3], void* stream);

/* The 108 SSIMULACRA2 features (plane*36 + scale*6 + norm*3 + map) of the handler's last
 * Vship_ComputeSSIMU2 call; pruned features are 0. */
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2LastFeatures(Vship_SSIMU2Handler handler, float features[108]);

/* Butteraugli of one frame pair already in device memory, queued on `stream`.  d_norms
 * (device, 3 doubles) receives {normQ, norm3, norminf}; d_distmap (device, may be NULL) the
 * FP32 distortion map with row stride dststride bytes (a multiple of 4). */
EXPORTPREPROCESS Vship_Exception VshipExt_ComputeButteraugliDevice(Vship_ButteraugliHandler handler, double* d_norms,
                                                                    float* d_distmap, int64_t dststride,
                                                                    const uint8_t* const srcp1[3], const uint8_t* const srcp2[3],
                                                                    const int64_t lineSize[3], const int64_t lineSize2[3],
                                                                    void* stream);

/* Per-kernel CUDA-event timing of a handler (off by default).  When enabled, every kernel
 * launch of the handler is bracketed by events on its stream. */
typedef struct VshipExt_KernelTime {
    char name[32];
    int launches;
    double total_ms;
} VshipExt_KernelTime;

EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2KernelTiming(Vship_SSIMU2Handler handler, int enable);
/* Writes up to max entries (kernels launched at least once since timing was enabled or last
 * reset) and returns their number; reset != 0 clears the totals afterwards.  Synchronises. */
EXPORTPREPROCESS int VshipExt_SSIMU2KernelTimes(Vship_SSIMU2Handler handler, VshipExt_KernelTime* out, int max, int reset);
EXPORTPREPROCESS Vship_Exception VshipExt_ButteraugliKernelTiming(Vship_ButteraugliHandler handler, int enable);
EXPORTPREPROCESS int VshipExt_ButteraugliKernelTimes(Vship_ButteraugliHandler handler, VshipExt_KernelTime* out, int max, int reset);

/* Metric resolution (after resize and crop) of a handler. */
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2Resolution(Vship_SSIMU2Handler handler, int64_t* width, int64_t* height);
EXPORTPREPROCESS Vship_Exception VshipExt_ButteraugliResolution(Vship_ButteraugliHandler handler, int64_t* width, int64_t* height);

#ifdef __cplusplus
}
#endif

#endif /* VSHIP_B200_API_EXT_H */

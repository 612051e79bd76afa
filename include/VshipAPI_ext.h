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
/* Test hook for the bounded waits of the low-frequency blur's column pass, which loads its
 * boxes with tensor-map copies when the plane width is a multiple of 4: in the next call one
 * box barrier of the reference image's full-scale pass is armed with no copy behind it, so its
 * wait gives up after a short limit and sets the handler's error word; Vship_ComputeButteraugli
 * then fails with Vship_HIPError (VshipExt_ComputeButteraugliDevice reports it on the next
 * call), and the calls after it are whole again.  Nothing faults and the context stays
 * usable.  Vship_BadDeviceArgument when the handler's resolution does not use that pass. */
EXPORTPREPROCESS Vship_Exception VshipExt_ButteraugliTestTmaTimeout(Vship_ButteraugliHandler handler);
EXPORTPREPROCESS int VshipExt_ButteraugliKernelTimes(Vship_ButteraugliHandler handler, VshipExt_KernelTime* out, int max, int reset);

/* Scores one frame pair already in device memory without allocating anything, for callers
 * that cannot call cudaMalloc: a process whose GPU memory is handed out up front by a fixed
 * budget or pool (an allocation outside it fails or takes memory another component was
 * promised), or a real-time loop that must never enter the driver's allocator (a cudaMalloc
 * can block for milliseconds and synchronise the device).  This function has no counterpart
 * in the reference library.
 *
 * It runs on the current device, with no handler: the colourspaces are passed directly
 * (resize and crop are not supported here; use a handler for those).  Inputs are three device
 * plane pointers per image with byte strides; d_score (device, 1 double) and d_features
 * (device, 108 floats, may be NULL) receive the results; work is queued on `stream` (NULL is
 * the legacy default stream) and the call returns without waiting.
 *
 * All scratch -- both XYB pyramids, the tile sums and the work list -- lives in a fixed
 * 32 MiB array inside the library, which every GPU that loads the library holds until the
 * process exits.  Frames up to 1920x1200 fit; larger frames are rejected with Vship_OutOfVRAM
 * and a detail giving the bytes needed.  The first call on each device looks up the array's
 * device address and loads the blur constants (synchronous driver calls), so make that first
 * call before any stream capture.  Every call shares the one array per device: calls whose
 * work overlaps on the GPU (different streams, or host threads without ordering) race and
 * corrupt each other's results; serialise them.  Each call writes every scratch byte it
 * reads, so nothing left by a previous call leaks into a result.  The device address and the
 * blur constants are cached per device for the life of the process: after cudaDeviceReset do
 * not call this entry point on that device again. */
EXPORTPREPROCESS Vship_Exception VshipExt_ComputeSSIMU2NoAlloc(Vship_Colorspace_t src_colorspace,
                                                                Vship_Colorspace_t dis_colorspace, double* d_score,
                                                                float* d_features, const uint8_t* const srcp1[3],
                                                                const uint8_t* const srcp2[3], const int64_t lineSize[3],
                                                                const int64_t lineSize2[3], void* stream);

/* ---- Uneven batches --------------------------------------------------------------------
 * No counterpart in the reference, which scores one pair per call through a handler bound to
 * one colourspace pair.  A batch handler scores any number of pairs whose colourspaces may
 * all differ (resolutions, formats) in one persistent launch replayed from a CUDA graph: one
 * work list holds the front tiles of every image, then the map tiles of every pair, then
 * each pair's final reduction, and a map tile starts once both pyramids of its pair are
 * built.  Resize and crop (target_width/height other than -1, or a non-zero crop) are not
 * supported in batches; use a per-colourspace handler for those. */

/* One frame pair of a batch: both colourspaces, three plane pointers per image and the row
 * strides in bytes (device pointers for VshipExt_ComputeSSIMU2BatchDevice, host pointers for
 * VshipExt_ComputeSSIMU2Batch). */
typedef struct VshipExt_FramePair {
    Vship_Colorspace_t src_colorspace;
    Vship_Colorspace_t dis_colorspace;
    const uint8_t* srcp1[3];
    const uint8_t* srcp2[3];
    int64_t lineSize[3];
    int64_t lineSize2[3];
} VshipExt_FramePair;

typedef struct VshipExt_SSIMU2BatchHandler {
    unsigned int id;
} VshipExt_SSIMU2BatchHandler;

EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2BatchInit(VshipExt_SSIMU2BatchHandler* handler, int gpu_id);
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2BatchFree(VshipExt_SSIMU2BatchHandler handler);
EXPORTPREPROCESS int VshipExt_SSIMU2BatchGetDetailedLastError(VshipExt_SSIMU2BatchHandler handler, char* out_message, int len);

/* n device-resident pairs, queued on `stream` (NULL: the legacy default stream) without
 * waiting.  d_scores (device, n doubles) receives the scores, d_features (device, 108 n
 * floats, may be NULL) the features.  Device buffers grow to the largest batch seen
 * (allocation synchronises the device).  With automatic tile rows (the default) the first
 * batch of a new mix of resolutions times each tile shape and synchronises; do that before
 * any stream capture, or fix the rows with VshipExt_SSIMU2BatchSetTileRows.  Wait-time
 * limits inside the launch are reported by the next call on the handler. */
EXPORTPREPROCESS Vship_Exception VshipExt_ComputeSSIMU2BatchDevice(VshipExt_SSIMU2BatchHandler handler, int n,
                                                                    const VshipExt_FramePair* pairs, double* d_scores,
                                                                    float* d_features, void* stream);
/* n host-resident pairs (pageable or pinned): copies them in chunks that overlap with the
 * scoring of the previous chunk, writes n scores (host) and, when features is not NULL,
 * 108 n features (host), and returns when they are written. */
EXPORTPREPROCESS Vship_Exception VshipExt_ComputeSSIMU2Batch(VshipExt_SSIMU2BatchHandler handler, int n,
                                                              const VshipExt_FramePair* pairs, double* scores,
                                                              float* features);
/* Rows of the map tiles: 16, 32 or 64, or 0 to choose by timing (the default).  Timed
 * choices are kept per device and mix of resolutions in memory and in the JSON file named by
 * the VSHIP_TUNE_CACHE environment variable (default
 * $XDG_CACHE_HOME/vship_b200/ssimu2_tiles.json or ~/.cache/vship_b200/ssimu2_tiles.json;
 * an empty value disables the file). */
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2BatchSetTileRows(VshipExt_SSIMU2BatchHandler handler, int rows);
/* Rows used by the last batch (0 before the first). */
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2BatchTileRows(VshipExt_SSIMU2BatchHandler handler, int* rows);
/* Test hook for the launch's bounded dependency waits: the next launch of this handler runs
 * its front grid without its last tile, so the map tiles of that pair wait for a pyramid that
 * is never finished.  The wait gives up after its 2 s limit and sets the launch's error word;
 * VshipExt_ComputeSSIMU2Batch then fails with Vship_HIPError (VshipExt_ComputeSSIMU2BatchDevice
 * reports it on the next call), and the launches after it are whole again.  Nothing faults
 * and the context stays usable. */
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2BatchTestHoldFrontTile(VshipExt_SSIMU2BatchHandler handler);
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2BatchKernelTiming(VshipExt_SSIMU2BatchHandler handler, int enable);
EXPORTPREPROCESS int VshipExt_SSIMU2BatchKernelTimes(VshipExt_SSIMU2BatchHandler handler, VshipExt_KernelTime* out,
                                                     int max, int reset);

/* ---- Learned surrogate ------------------------------------------------------------------
 * No counterpart in the reference.  A small convolutional network predicts SSIMULACRA2 from
 * the 1/8 and 1/16 XYB pyramid levels of both images (the coarse levels cost a fraction of
 * the exact metric), for searches such as target-quality encoding that need many scores but
 * only their side of a threshold: consult the prediction, and call the exact metric when it
 * lands within a margin of the threshold.  A handler is bound to one colourspace pair (no
 * resize or crop); its network runs at any resolution, so a model trained on one handler can
 * be set on another.  Training, inference and gradients run on the library's own kernels. */
typedef struct VshipExt_SurrogateHandler {
    unsigned int id;
} VshipExt_SurrogateHandler;

EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateInit(VshipExt_SurrogateHandler* handler, Vship_Colorspace_t src_colorspace,
                                                        Vship_Colorspace_t dis_colorspace, int gpu_id);
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateFree(VshipExt_SurrogateHandler handler);
EXPORTPREPROCESS int VshipExt_SurrogateGetDetailedLastError(VshipExt_SurrogateHandler handler, char* out_message, int len);
/* FP16 elements of one pair's network input. */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateInputSize(VshipExt_SurrogateHandler handler, int64_t* elems);
/* Network inputs of n device-resident pairs (3 plane pointers per image, as
 * VshipExt_ComputeSSIMU2Device) into d_inputs (device, n * InputSize FP16), on `stream`. */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateInputs(VshipExt_SurrogateHandler handler, int n,
                                                          const uint8_t* const* srcp1, const uint8_t* const* srcp2,
                                                          const int64_t lineSize[3], const int64_t lineSize2[3],
                                                          void* d_inputs, void* stream);
/* Predicted scores (device floats) of n prepared inputs, or of n device-resident pairs. */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogatePredictInputs(VshipExt_SurrogateHandler handler, int n,
                                                                 const void* d_inputs, float* d_pred, void* stream);
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogatePredict(VshipExt_SurrogateHandler handler, int n,
                                                           const uint8_t* const* srcp1, const uint8_t* const* srcp2,
                                                           const int64_t lineSize[3], const int64_t lineSize2[3],
                                                           float* d_pred, void* stream);
/* Searches probe one reference frame against many distortions of it: prepare the references'
 * coarse levels once (device floats, ReferenceSize each, n references back to back), then
 * predict distorted frames against them (pair i uses reference i); the predictions equal
 * those of VshipExt_SurrogatePredict on the same pairs, at about half the cost. */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateReferenceSize(VshipExt_SurrogateHandler handler, int64_t* floats);
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateReferences(VshipExt_SurrogateHandler handler, int n,
                                                              const uint8_t* const* srcp1, const int64_t lineSize[3],
                                                              float* d_refs, void* stream);
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogatePredictAgainst(VshipExt_SurrogateHandler handler, int n,
                                                                  const float* d_refs, const uint8_t* const* srcp2,
                                                                  const int64_t lineSize2[3], float* d_pred, void* stream);
/* Trains the network from scratch (seeded) on n prepared inputs and their exact scores
 * (device floats): Adam, cosine learning-rate decay from lr to lr / 20, MSE on the scores.
 * loss_history (host, may be NULL) receives the mean loss of each epoch.  Synchronous. */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateTrain(VshipExt_SurrogateHandler handler, int n, const void* d_inputs,
                                                         const float* d_targets, int epochs, int batch, float lr,
                                                         unsigned int seed, float* loss_history);
/* Loss and its gradients (host floats, one per parameter) for the current model on n <= 1024
 * prepared inputs; the model is not changed. */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateGradients(VshipExt_SurrogateHandler handler, int n,
                                                             const void* d_inputs, const float* d_targets, float* grads,
                                                             double* loss);
/* The model as floats (parameters, then the input normalisation): returns its length and
 * fills `out` when max is at least that; -1 on error.  SetModel loads such a vector. */
EXPORTPREPROCESS int VshipExt_SurrogateModel(VshipExt_SurrogateHandler handler, float* out, int max);
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateSetModel(VshipExt_SurrogateHandler handler, const float* model, int count);
/* Per-kernel CUDA-event timing of a surrogate handler (coarse front, network forward). */
EXPORTPREPROCESS Vship_Exception VshipExt_SurrogateKernelTiming(VshipExt_SurrogateHandler handler, int enable);
EXPORTPREPROCESS int VshipExt_SurrogateKernelTimes(VshipExt_SurrogateHandler handler, VshipExt_KernelTime* out, int max,
                                                   int reset);

/* Metric resolution (after resize and crop) of a handler. */
EXPORTPREPROCESS Vship_Exception VshipExt_SSIMU2Resolution(Vship_SSIMU2Handler handler, int64_t* width, int64_t* height);
EXPORTPREPROCESS Vship_Exception VshipExt_ButteraugliResolution(Vship_ButteraugliHandler handler, int64_t* width, int64_t* height);

/* ---- CVVDP display models (no reference counterpart) --------------------------------------
 * The display a CVVDP handler would use for (model_key, model_config_json), resolved exactly as
 * Vship_CVVDPInit2 resolves it (built-in model, then the JSON file's entry of that name), with
 * the derived pixels per degree and black / reflected luminance.  Host only: needs no GPU.
 * Errors: Vship_BadDisplayModel, Vship_BadPath, Vship_BadJson, Vship_BadPointer (null key or
 * output), reported through the global last error. */
typedef struct VshipExt_CVVDPDisplay {
    int64_t width, height; /* resolution in pixels */
    int hdr;               /* 0: SDR display (sRGB encoding), 1: HDR */
    float viewing_distance_meters, diagonal_size_inches;
    float max_luminance, contrast, E_ambient, k_refl, exposure;
    float ppd;             /* pixels per visual degree */
    float black_level;     /* max_luminance / contrast, cd/m^2 */
    float reflected_level; /* E_ambient * k_refl / pi, cd/m^2 */
} VshipExt_CVVDPDisplay;
EXPORTPREPROCESS Vship_Exception VshipExt_CVVDPDisplayModel(const char* model_key, const char* model_config_json,
                                                            VshipExt_CVVDPDisplay* out);
/* Pyramid bands and ring length (frames) of a CVVDP handler. */
EXPORTPREPROCESS Vship_Exception VshipExt_CVVDPGeometry(Vship_CVVDPHandler handler, int* bands, int* ring_frames);
EXPORTPREPROCESS Vship_Exception VshipExt_CVVDPKernelTiming(Vship_CVVDPHandler handler, int enable);
EXPORTPREPROCESS int VshipExt_CVVDPKernelTimes(Vship_CVVDPHandler handler, VshipExt_KernelTime* out, int max, int reset);

#ifdef __cplusplus
}
#endif

#endif /* VSHIP_B200_API_EXT_H */

// Internal interfaces between the C ABI layer (api.cu) and the metric engines.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"
#include "../../include/VshipAPI_ext.h"

namespace vship {

// SSIMULACRA2 engine of one handler (replaces ssimu2::SSIMU2ComputingImplementation,
// src/ssimu2/main.hpp:80-156).  All device memory is allocated by init.
struct Ssimu2Api {
    virtual ~Ssimu2Api() = default;
    virtual void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, int device) = 0;
    // Host planes; blocks until the score is known.
    virtual double compute(const uint8_t* const s1[3], const uint8_t* const s2[3], const int64_t ls1[3],
                           const int64_t ls2[3]) = 0;
    // n pairs already in device memory (3 plane pointers per image); asynchronous on `stream`.
    virtual void compute_device(int n, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t ls1[3],
                                const int64_t ls2[3], double* d_scores, float* d_features, cudaStream_t stream) = 0;
    virtual void last_features(float out[108]) = 0;
    virtual KernelTimer& timer() = 0;
    virtual int width() const = 0;
    virtual int height() const = 0;
};

// Butteraugli engine of one handler (replaces butter::ButterComputingImplementation,
// src/butter/main.hpp:183-231).
struct ButterApi {
    virtual ~ButterApi() = default;
    virtual void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, int qnorm, float intensity,
                      int device) = 0;
    // Host planes; dstp (nullable) receives the FP32 distortion map with row stride dststride.
    virtual void compute(double norms[3], uint8_t* dstp, int64_t dststride, const uint8_t* const s1[3],
                         const uint8_t* const s2[3], const int64_t ls1[3], const int64_t ls2[3]) = 0;
    // One pair already in device memory; asynchronous on `stream`.  d_norms receives 3 doubles,
    // d_distmap (nullable) the map with row stride dststride bytes.
    virtual void compute_device(double* d_norms, float* d_distmap, int64_t dststride, const uint8_t* const d1[3],
                                const uint8_t* const d2[3], const int64_t ls1[3], const int64_t ls2[3],
                                cudaStream_t stream) = 0;
    // Test hook: the next call's full-scale low-frequency column pass of the reference image
    // leaves one box barrier armed with no load behind it, so that wait runs out.  False when
    // this handler's resolution does not use the tensor-map pass.
    virtual bool test_tma_timeout() = 0;
    virtual KernelTimer& timer() = 0;
    virtual int width() const = 0;
    virtual int height() const = 0;
};

// SSIMULACRA2 over uneven batches (no reference counterpart): pairs of any colourspaces in
// one persistent launch replayed from a CUDA graph.
struct Ssimu2BatchApi {
    virtual ~Ssimu2BatchApi() = default;
    virtual void init(int device) = 0;
    // Device-resident pairs; asynchronous on `stream`.
    virtual void compute_device(int n, const VshipExt_FramePair* pairs, double* d_scores, float* d_features,
                                cudaStream_t stream) = 0;
    // Host-resident pairs; blocks until scores (and features, when not null) are written.
    virtual void compute(int n, const VshipExt_FramePair* pairs, double* scores, float* features) = 0;
    virtual void set_tile_rows(int rows) = 0;
    virtual int tile_rows() const = 0;
    // Test hook: the next launch leaves its last front tile unlaunched (one launch only).
    virtual void hold_front_tile() = 0;
    virtual KernelTimer& timer() = 0;
};

// Learned SSIMULACRA2 surrogate bound to one colourspace pair (no reference counterpart).
struct SurrogateApi {
    virtual ~SurrogateApi() = default;
    virtual void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, int device) = 0;
    virtual int64_t input_elems() const = 0;   // FP16 elements of one pair's network input
    virtual int num_params() const = 0;
    // Network inputs of n device-resident pairs into d_inputs (n * input_elems() FP16).
    virtual void inputs(int n, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t ls1[3],
                        const int64_t ls2[3], void* d_inputs, cudaStream_t stream) = 0;
    virtual void predict_inputs(int n, const void* d_inputs, float* d_pred, cudaStream_t stream) = 0;
    // Inputs and predictions of n device-resident pairs (internal input buffer).
    virtual void predict(int n, const uint8_t* const* d1, const uint8_t* const* d2, const int64_t ls1[3],
                         const int64_t ls2[3], float* d_pred, cudaStream_t stream) = 0;
    // Levels 1/8 and 1/16 of n reference images (FP32, reference_floats() each), and
    // predictions of n distorted images against such prepared references.
    virtual int64_t reference_floats() const = 0;
    virtual void references(int n, const uint8_t* const* d1, const int64_t ls1[3], float* d_refs,
                            cudaStream_t stream) = 0;
    virtual void predict_against(int n, const float* d_refs, const uint8_t* const* d2, const int64_t ls2[3],
                                 float* d_pred, cudaStream_t stream) = 0;
    // Loss and gradients (FP32, num_params()) of the current weights on n samples.
    virtual double gradients(int n, const void* d_inputs, const float* d_targets, float* grads_host) = 0;
    virtual void train(int n, const void* d_inputs, const float* d_targets, int epochs, int batch, float lr,
                       unsigned seed, float* loss_history) = 0;
    // Model = parameters then input normalisation (shift[6], scale[6]); returns its length.
    virtual int get_model(float* out, int max) = 0;
    virtual void set_model(const float* in, int count) = 0;
    virtual KernelTimer& timer() = 0;
};

// CVVDP engine of one handler (replaces cvvdp::CVVDPComputingImplementation,
// src/cvvdp/main.hpp:161-398): a ring of past frames per clip and the running temporal score.
struct CvvdpApi {
    virtual ~CvvdpApi() = default;
    virtual void init(const Vship_Colorspace_t& src, const Vship_Colorspace_t& dis, float fps, bool resize_to_display,
                      const std::string& model_key, const std::string& model_config_json, int device) = 0;
    // Adds a frame pair to the ring, scores it and returns the JOD of the sequence so far;
    // dstp (nullable) receives the distortion map (rows of dststride bytes).
    virtual double compute(uint8_t* dstp, int64_t dststride, const uint8_t* const s1[3], const uint8_t* const s2[3],
                           const int64_t ls1[3], const int64_t ls2[3]) = 0;
    // Adds a frame pair to the ring without scoring it.
    virtual void load_temporal(const uint8_t* const s1[3], const uint8_t* const s2[3], const int64_t ls1[3],
                               const int64_t ls2[3]) = 0;
    // Empties the ring and the score (only_score: the score only).
    virtual void reset(bool only_score) = 0;
    virtual int64_t distmap_width() const = 0;
    virtual int64_t distmap_height() const = 0;
    virtual int bands() const = 0;
    virtual int ring_frames() const = 0;
    virtual KernelTimer& timer() = 0;
};

// Resolves a CVVDP display model (built-in name, then the JSON file's entry); throws Error.
void cvvdp_display_model(const std::string& model_key, const std::string& model_config_json, VshipExt_CVVDPDisplay* out);

Ssimu2Api* make_ssimu2_engine();
CvvdpApi* make_cvvdp_engine();
SurrogateApi* make_surrogate_engine();
Ssimu2BatchApi* make_ssimu2_batch_engine();
void record_global_error(const Error& e);
ButterApi* make_butter_engine();

}  // namespace vship

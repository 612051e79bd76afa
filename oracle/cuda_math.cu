// cuda_math.cu -- CUDA's own float powf, cbrtf and expf over host arrays.
//
// TEST INFRASTRUCTURE ONLY.  The FP32 restatement of the reference's SSIMULACRA2 arithmetic
// (ssimu2_f32.c) takes its transcendental values through one array hook.  On a machine with a
// GPU the tests point that hook here, so the restatement uses the very functions the reference
// library calls on the device (compiled by the same nvcc with the same default flags: no fast
// math), not correctly rounded substitutes that may differ from them in the last bit.
// Built by oracle.build_cuda_math() into oracle/libcudamath.so; the product never loads it.
#include <cuda_runtime.h>
#include <cstdint>

namespace {

__global__ void eval_kernel(int op, const float* x, float y, float* out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = x[i];
    if (op == 0) out[i] = powf(v, y);
    else if (op == 1) out[i] = cbrtf(v);
    else out[i] = expf(v);
}

}  // namespace

// op 0: out[i] = powf(x[i], y); op 1: cbrtf(x[i]); op 2: expf(x[i]).  Host pointers in and
// out.  Returns 0, or the CUDA error code.
extern "C" __attribute__((visibility("default"))) int cm_eval(int op, const float* x, float y, float* out, int64_t n) {
    if (n <= 0) return 0;
    float *dx = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&dx, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(float) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int threads = 256;
        const int64_t blocks = (n + threads - 1) / threads;
        eval_kernel<<<(unsigned)blocks, threads>>>(op, dx, y, dout, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    return (int)e;
}

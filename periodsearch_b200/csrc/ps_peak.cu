// FP64 tensor-core throughput probe: the denominator of the roofline that the
// fast form's shape contraction (m8n8k4 FP64 MMA) and its FP64 arithmetic are
// measured against, taken on the GPU that runs the fits.  B200 has no FP64
// kind of tcgen05.mma; the FP64 tensor path is mma.sync m8n8k4.f64.
#include <cuda_runtime.h>

#include "../../include/period_search_b200.h"
#include "ps_ctx.hpp"

namespace {

constexpr int kTiles = 28;   // independent accumulator tiles per warp
constexpr int kSteps = 4096; // MMA steps per tile

__global__ void __launch_bounds__(256, 1) fp64_mma_peak_kernel(double* out, double seed) {
    double c[kTiles][2];
#pragma unroll
    for (int t = 0; t < kTiles; t++) c[t][0] = c[t][1] = 0;
    double b[8];
#pragma unroll
    for (int k = 0; k < 8; k++) b[k] = seed * (k + 1 + threadIdx.x);
    double a = seed * threadIdx.x;
    for (int it = 0; it < kSteps; it++) {
        a = a * 0.999 + 1e-3;
#pragma unroll
        for (int t = 0; t < kTiles; t++)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(c[t][0]), "+d"(c[t][1])
                         : "d"(a), "d"(b[t & 7]));
    }
    double s = 0;
#pragma unroll
    for (int t = 0; t < kTiles; t++) s += c[t][0] + c[t][1];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int ps_fp64_tensor_peak(int device, double* tflops) {
    if (!tflops) return psb::set_error(PS_ERR_ARG, "tflops is NULL");
    if (cudaSetDevice(device) != cudaSuccess) return psb::set_error(PS_ERR_CUDA, "cudaSetDevice failed");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double* out = nullptr;
    if (cudaMalloc(&out, (size_t)sms * 256 * sizeof(double)) != cudaSuccess)
        return psb::set_error(PS_ERR_CUDA, "cudaMalloc failed");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        fp64_mma_peak_kernel<<<sms, 256>>>(out, 1e-3);
        psb::count_launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return psb::set_error(PS_ERR_CUDA, cudaGetErrorString(err));
    // per warp and step: kTiles MMAs of 8 x 8 x 4 multiply-adds
    const double flop = 2.0 * 8 * 8 * 4 * kTiles * (double)kSteps * (sms * 256 / 32);
    *tflops = flop / (best * 1e-3) / 1e12;
    return PS_OK;
}

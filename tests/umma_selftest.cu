// Test-only library: a 128 x 64 x K GEMM D = A B^T on the tcgen05 tensor
// core with split-BF16 operands (hi*hi + hi*lo + lo*hi, FP32 accumulation in
// TMEM), built from the same helpers (periodsearch_b200/csrc/ps_umma.cuh) as
// the mixed-precision fit kernel.  tests/test_umma.py checks it against an
// FP64 product: it validates the swizzled operand layout, the descriptors,
// the instruction descriptor and the TMEM lane/column mapping on the device.
#include <cuda_runtime.h>

#include "../periodsearch_b200/csrc/ps_umma.cuh"

using namespace psb::umma;

__global__ void __launch_bounds__(128, 1)
    umma_gemm_selftest(const float* __restrict__ A, const float* __restrict__ B, int K, float* __restrict__ D,
                       int* __restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_u32 = smem_u32(smem_raw);
    const uint32_t pad = ((base_u32 + 1023u) & ~1023u) - base_u32;
    uint8_t* sm = smem_raw + pad;                  // 1024-byte aligned
    uint8_t* Ahi = sm;                             // 128 rows x 128 B
    uint8_t* Alo = sm + 16384;
    uint8_t* Bhi = sm + 32768;                     // 64 rows x 128 B
    uint8_t* Blo = sm + 40960;
    uint64_t* mbar = (uint64_t*)(sm + 49152);
    uint32_t* slot = (uint32_t*)(sm + 49152 + 16);
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) tmem_alloc(slot, 64);
    if (tid == 0) mbar_init(mbar, 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t idesc = idesc_bf16_f32(128, 64);
    bool ok = true;
    for (int c = 0; c < K / 64; c++) {
        for (int idx = tid; idx < 128 * 64; idx += 128) {
            const int r = idx >> 6, k = idx & 63;
            __nv_bfloat16 hi, lo;
            split_bf16(A[(size_t)r * K + c * 64 + k], hi, lo);
            *(__nv_bfloat16*)(Ahi + sw128_off(r, k)) = hi;
            *(__nv_bfloat16*)(Alo + sw128_off(r, k)) = lo;
        }
        for (int idx = tid; idx < 64 * 64; idx += 128) {
            const int r = idx >> 6, k = idx & 63;
            __nv_bfloat16 hi, lo;
            split_bf16(B[(size_t)r * K + c * 64 + k], hi, lo);
            *(__nv_bfloat16*)(Bhi + sw128_off(r, k)) = hi;
            *(__nv_bfloat16*)(Blo + sw128_off(r, k)) = lo;
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const uint32_t o = kk * 32;
                mma_bf16(tmem, desc_kmajor_sw128(smem_u32(Ahi) + o), desc_kmajor_sw128(smem_u32(Bhi) + o), idesc,
                         (c > 0 || kk > 0) ? 1u : 0u);
                mma_bf16(tmem, desc_kmajor_sw128(smem_u32(Ahi) + o), desc_kmajor_sw128(smem_u32(Blo) + o), idesc, 1u);
                mma_bf16(tmem, desc_kmajor_sw128(smem_u32(Alo) + o), desc_kmajor_sw128(smem_u32(Bhi) + o), idesc, 1u);
            }
            commit(mbar);
        }
        if (!mbar_wait(mbar, (uint32_t)(c & 1), 1u << 22)) ok = false;
        fence_after_sync();
    }
    if (!ok) atomicExch(status, 1);
    float v[16];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + q * 16, v);
        const int row = warp * 32 + (tid & 31);
#pragma unroll
        for (int i = 0; i < 16; i++) D[row * 64 + q * 16 + i] = v[i];
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

// The same GEMM with split-TF32 operands on kind::tf32 (32 K elements per
// 128-byte row).
__global__ void __launch_bounds__(128, 1)
    umma_gemm_selftest_tf32(const float* __restrict__ A, const float* __restrict__ B, int K, float* __restrict__ D,
                            int* __restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t base_u32 = smem_u32(smem_raw);
    const uint32_t pad = ((base_u32 + 1023u) & ~1023u) - base_u32;
    uint8_t* sm = smem_raw + pad;
    uint8_t* Ahi = sm;
    uint8_t* Alo = sm + 16384;
    uint8_t* Bhi = sm + 32768;
    uint8_t* Blo = sm + 40960;
    uint64_t* mbar = (uint64_t*)(sm + 49152);
    uint32_t* slot = (uint32_t*)(sm + 49152 + 16);
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) tmem_alloc(slot, 64);
    if (tid == 0) mbar_init(mbar, 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t idesc = idesc_tf32_f32(128, 64);
    bool ok = true;
    for (int c = 0; c < K / 32; c++) {
        for (int idx = tid; idx < 128 * 32; idx += 128) {
            const int r = idx >> 5, k = idx & 31;
            uint32_t hi, lo;
            split_tf32(A[(size_t)r * K + c * 32 + k], hi, lo);
            *(uint32_t*)(Ahi + sw128_off32(r, k)) = hi;
            *(uint32_t*)(Alo + sw128_off32(r, k)) = lo;
        }
        for (int idx = tid; idx < 64 * 32; idx += 128) {
            const int r = idx >> 5, k = idx & 31;
            uint32_t hi, lo;
            split_tf32(B[(size_t)r * K + c * 32 + k], hi, lo);
            *(uint32_t*)(Bhi + sw128_off32(r, k)) = hi;
            *(uint32_t*)(Blo + sw128_off32(r, k)) = lo;
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const uint32_t o = kk * 32;
                mma_tf32(tmem, desc_kmajor_sw128(smem_u32(Ahi) + o), desc_kmajor_sw128(smem_u32(Bhi) + o), idesc,
                         (c > 0 || kk > 0) ? 1u : 0u);
                mma_tf32(tmem, desc_kmajor_sw128(smem_u32(Ahi) + o), desc_kmajor_sw128(smem_u32(Blo) + o), idesc, 1u);
                mma_tf32(tmem, desc_kmajor_sw128(smem_u32(Alo) + o), desc_kmajor_sw128(smem_u32(Bhi) + o), idesc, 1u);
            }
            commit(mbar);
        }
        if (!mbar_wait(mbar, (uint32_t)(c & 1), 1u << 22)) ok = false;
        fence_after_sync();
    }
    if (!ok) atomicExch(status, 1);
    float v[16];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + q * 16, v);
        const int row = warp * 32 + (tid & 31);
#pragma unroll
        for (int i = 0; i < 16; i++) D[row * 64 + q * 16 + i] = v[i];
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 64);
}

extern "C" int umma_selftest_tf32(const float* hA, const float* hB, int K, float* hD) {
    if (K <= 0 || K % 32) return -1;
    float *A, *B, *D;
    int* st;
    if (cudaMalloc(&A, sizeof(float) * 128 * K) || cudaMalloc(&B, sizeof(float) * 64 * K) ||
        cudaMalloc(&D, sizeof(float) * 128 * 64) || cudaMalloc(&st, sizeof(int)))
        return -2;
    cudaMemcpy(A, hA, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
    cudaMemcpy(B, hB, sizeof(float) * 64 * K, cudaMemcpyHostToDevice);
    cudaMemset(st, 0, sizeof(int));
    const int smem = 49152 + 64 + 1024;
    cudaFuncSetAttribute(umma_gemm_selftest_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    umma_gemm_selftest_tf32<<<1, 128, smem>>>(A, B, K, D, st);
    cudaError_t e = cudaDeviceSynchronize();
    int status = 0;
    cudaMemcpy(&status, st, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(hD, D, sizeof(float) * 128 * 64, cudaMemcpyDeviceToHost);
    cudaFree(A);
    cudaFree(B);
    cudaFree(D);
    cudaFree(st);
    if (e != cudaSuccess) return -3;
    return status;
}

extern "C" int umma_selftest(const float* hA, const float* hB, int K, float* hD) {
    if (K <= 0 || K % 64) return -1;
    float *A, *B, *D;
    int* st;
    if (cudaMalloc(&A, sizeof(float) * 128 * K) || cudaMalloc(&B, sizeof(float) * 64 * K) ||
        cudaMalloc(&D, sizeof(float) * 128 * 64) || cudaMalloc(&st, sizeof(int)))
        return -2;
    cudaMemcpy(A, hA, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
    cudaMemcpy(B, hB, sizeof(float) * 64 * K, cudaMemcpyHostToDevice);
    cudaMemset(st, 0, sizeof(int));
    const int smem = 49152 + 64 + 1024;
    cudaFuncSetAttribute(umma_gemm_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    umma_gemm_selftest<<<1, 128, smem>>>(A, B, K, D, st);
    cudaError_t e = cudaDeviceSynchronize();
    int status = 0;
    cudaMemcpy(&status, st, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(hD, D, sizeof(float) * 128 * 64, cudaMemcpyDeviceToHost);
    cudaFree(A);
    cudaFree(B);
    cudaFree(D);
    cudaFree(st);
    if (e != cudaSuccess) return -3;
    return status;
}

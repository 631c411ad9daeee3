// Private definition of the C ABI's context (ps_ctx) and its device
// buffers, shared by the translation units that implement the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/period_search_b200.h"
#include "ps_device.hpp"
#include "ps_host.hpp"

namespace psb {

// Records the message returned by ps_last_error() for the calling thread.
int set_error(int code, const std::string& msg);
// After a launch on stream s: if s is not the context's own stream, record
// the context's caller_done event on it (no allocation).
cudaError_t note_caller_stream(ps_ctx* c, cudaStream_t s);
// Counts one kernel launch for ps_kernel_launches().
void count_launch();

// Process-wide cache of device buffers per device.  Buffers released by a
// context or batch (ps_close, ps_batch_close) go back to the cache and are
// handed to the next request they fit (at most twice its size, or 1 MiB
// more), so that opening and closing a context per asteroid does not pay a
// cudaMalloc and a device-synchronising cudaFree for each of its tables and
// its ~100 MB Jacobian scratch every time.  A buffer belongs to one owner at
// a time.  The cache keeps at most kPoolMaxBuffers buffers and kPoolMaxBytes
// per device, until ps_release_cached_memory or process exit.
cudaError_t pool_take(int device, size_t bytes, void** p, size_t* cap);
void pool_give(int device, void* p, size_t cap);

// Grow-only device buffer on the device that is current when it first
// allocates, drawn from and returned to the per-device cache.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    int device = -1;
    cudaError_t ensure(size_t count) {
        if (count <= n) return cudaSuccess;
        release();
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        void* q = nullptr;
        size_t cap = 0;
        e = pool_take(dev, count * sizeof(T), &q, &cap);
        if (e == cudaSuccess) {
            p = (T*)q;
            n = cap / sizeof(T);
            device = dev;
        }
        return e;
    }
    cudaError_t upload(const std::vector<T>& v, cudaStream_t s) {
        cudaError_t e = ensure(v.size() ? v.size() : 1);
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    }
    void release() {
        if (p) pool_give(device, p, n * sizeof(T));
        p = nullptr;
        n = 0;
    }
};

}  // namespace psb

struct ps_ctx {
    psb::Problem prob;
    int device = 0;
    int form = PS_FORM_FP64;
    bool host_only = true;
    bool rows_ready = false;
    cudaStream_t stream = nullptr;
    // recorded after each scan launched on a caller's stream: ps_close waits
    // for it before the context's buffers go back to the cache
    cudaEvent_t caller_done = nullptr;
    bool caller_pending = false;
    int sms = 0, blocks_per_sm = 0;
    int prepass_fits = 0;  // fits run by the last ps_precalc
    psb::DevProblem dp{};
    // device tables
    psb::DevBuf<double> d_pts, d_rows, d_fac, d_dsph, d_cpl, d_cfc, d_cfs, d_cgf, d_pole;
    psb::DevBuf<int> d_lc, d_free, d_queue;
    psb::DevBuf<double> d_scratch;
    psb::DevBuf<psb::FitOut> d_fits;
    psb::DevBuf<ps_record> d_rec;
    psb::DevBuf<double> d_eval;
    psb::DevBuf<double> d_adj;  // matrix-free work arrays
    psb::DevBuf<psb::DevProblem> d_dp;
    psb::DevBuf<float> d_fac32;
    psb::DevBuf<uint16_t> d_bsw;
    psb::DevBuf<int> d_err;
    // speculative convexity pre-pass rounds: rows and problem copies per round
    psb::DevBuf<double> d_pre_rows;
    psb::DevBuf<psb::DevProblem> d_pre_dp;
    psb::DevBuf<int> d_pre_ctl;
    std::vector<int> free_idx;
};


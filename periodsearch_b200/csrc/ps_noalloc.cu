// ps_scan_device_noalloc: the period scan (the FP64 fit kernel and the
// best-of-poles reduction) with every piece of scratch memory taken from one
// file-scope device array instead of from cudaMalloc.
//
// Who needs this: callers that must not allocate device memory while they
// run -- a host that runs under a fixed, pre-sized device-memory budget, a
// plugin loaded into a process whose allocator it does not own, or a
// latency-sensitive service that cannot take cudaMalloc/cudaFree on its scan
// path (cudaFree waits for all work on the device).  Such a caller sets
// the context up once (ps_open*, ps_precalc / ps_set_conw_r allocate the
// per-asteroid tables there) and afterwards scans with this entry point,
// which calls no cudaMalloc, cudaFree or other allocating routine.
//
// The array is kNoAllocScratchBytes (64 MiB) of device memory that every GPU
// loading this library holds until the process exits.  It carries the work
// counter, the per-fit results (72 bytes per fit) and the per-CTA Jacobian
// scratch ((ma + 1) x npad doubles per resident CTA); the launch uses as many
// CTAs as fit in what is left after the per-fit results, and a request whose
// per-fit results plus one CTA's scratch exceed the array is rejected with
// PS_ERR_LIMIT.  All calls share the array and it keeps the last call's
// contents: the work counter is cleared on the stream before every launch,
// and calls whose launches overlap on the GPU (different streams, or
// different host threads) race on it -- serialise them.
//
// The device address of the array is looked up once per device
// (cudaGetSymbolAddress, with that device current) by the first call made on
// that device; make that first call before any stream capture begins.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/period_search_b200.h"
#include "ps_ctx.hpp"
#include "ps_device.hpp"

namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the array on `device` (which must be current).
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return psb::set_error(PS_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return psb::set_error(PS_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                                   cudaGetErrorString(e));
        g_scratch_ptr[device] = p;
    }
    *out = (unsigned char*)g_scratch_ptr[device];
    return PS_OK;
}

}  // namespace

extern "C" int ps_scan_device_noalloc(ps_ctx* c, int n_from, int n_to, ps_record* d_out, void* stream) {
    if (!c) return psb::set_error(PS_ERR_ARG, "null context");
    if (c->host_only) return psb::set_error(PS_ERR_ARG, "context was opened without a device");
    if (c->form != PS_FORM_FP64) return psb::set_error(PS_ERR_ARG, "the no-allocation scan runs the FP64 form");
    if (!c->rows_ready) return psb::set_error(PS_ERR_ARG, "call ps_precalc or ps_set_conw_r first");
    if (n_from < 1 || n_to < n_from || n_to > c->prob.n_periods() || !d_out)
        return psb::set_error(PS_ERR_ARG, "period range out of bounds");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return psb::set_error(PS_ERR_CUDA, cudaGetErrorString(e));
    unsigned char* base = nullptr;
    int rc = scratch_address(c->device, &base);
    if (rc) return rc;
    const psb::DevProblem& d = c->dp;
    const int np = n_to - n_from + 1;
    const size_t n_fits = (size_t)np * 10;
    // layout: [work counter, 256 B][per-fit results][per-CTA J scratch]
    const size_t fits_off = 256;
    const size_t fits_bytes = (n_fits * sizeof(psb::FitOut) + 255) & ~(size_t)255;
    const size_t stride = (size_t)(d.ma + 1) * d.npad;  // doubles per CTA
    const size_t cta_bytes = stride * sizeof(double);
    if (fits_off + fits_bytes + cta_bytes > kNoAllocScratchBytes)
        return psb::set_error(PS_ERR_LIMIT, "scan too large for the 64 MiB no-allocation scratch: " +
                                                std::to_string(n_fits) + " fits need " +
                                                std::to_string(fits_off + fits_bytes + cta_bytes) +
                                                " bytes; scan fewer periods per call");
    const size_t fit_slots = (kNoAllocScratchBytes - fits_off - fits_bytes) / cta_bytes;
    long long grid = (long long)c->sms * c->blocks_per_sm;
    if (grid > (long long)n_fits) grid = (long long)n_fits;
    if (grid > (long long)fit_slots) grid = (long long)fit_slots;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    int* queue = (int*)base;
    psb::FitOut* fits = (psb::FitOut*)(base + fits_off);
    double* scratch = (double*)(base + fits_off + fits_bytes);
    e = cudaMemsetAsync(queue, 0, sizeof(int), s);
    if (e != cudaSuccess) return psb::set_error(PS_ERR_CUDA, cudaGetErrorString(e));
    psb::FitBatch b{};
    b.n_from = n_from;
    b.n_fits = (int)n_fits;
    b.queue = queue;
    b.out = fits;
    b.scratch = scratch;
    b.scratch_stride = (long long)stride;
    e = psb::launch_fp64_fits(d, c->d_dp.p, b, (int)grid, s);
    if (e != cudaSuccess) return psb::set_error(PS_ERR_CUDA, cudaGetErrorString(e));
    psb::count_launch();
    e = psb::launch_period_reduce(fits, np, d.ndata_m3, 0, d_out, s);
    if (e != cudaSuccess) return psb::set_error(PS_ERR_CUDA, cudaGetErrorString(e));
    psb::count_launch();
    e = psb::note_caller_stream(c, s);  // records an event created at open: no allocation
    if (e != cudaSuccess) return psb::set_error(PS_ERR_CUDA, cudaGetErrorString(e));
    return PS_OK;
}

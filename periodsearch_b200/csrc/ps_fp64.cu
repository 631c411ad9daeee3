// Plain FP64 form of the convex-inversion fit (the drop-in form).
//
// One CTA runs one complete Levenberg-Marquardt fit (one trial period, one
// initial pole): every model evaluation (the reference's mrqcof), every
// damped normal-equation solve (mrqmin + gauss_errc) and the stop rule of
// the driver loop (period_search_BOINC.cpp:846-893) happen on the device,
// with no host round trip per iteration.  CTAs are persistent and pull fits
// from a device work counter, so fits with different iteration counts do
// not wait for one another.
//
// Arithmetic follows the reference's FP64 operation order (this file is
// compiled with -fmad=false): sums over facets and over data rows are
// sequential in the reference's loop order, products and quotients are
// evaluated left to right as the C source writes them.  The remaining
// differences to the CPU reference are the libm routines (exp, sin, cos and
// pow(x, 2), computed as x*x here), each within an ulp.
//
// Work split inside a CTA (256 threads):
//   curv        thread per facet (facet areas, curv.c:10-38)
//   bright      two threads per data point, each holding half of the
//               point's sums (every sum in one thread, in facet order),
//               facets streamed through shared memory in chunks of kFch
//               (bright.c:14-126); Dg = g * Dsph built per chunk; two CTAs
//               (fits) per SM
//   conv        thread per (row, coefficient), sequential over facets
//               (conv.c:12-29)
//   normalise   per relative lightcurve: thread per column for the sums,
//               thread per row for the rank-1 update (mrqcof.c:53-104)
//   alpha/beta  thread per output entry, sequential over rows through
//               shared-memory row tiles (mrqcof.c:106-147)
//   solve       Gauss-Jordan with full pivoting, block-parallel
//               eliminations, the reference's pivot tie rule
//               (gauss_errc.c:9-73)
// Every loop is bounded by the problem sizes and by the LM iteration limit;
// nothing waits on a flag.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ps_device.hpp"
#include "ps_fit_common.cuh"
#include "ps_fit_impl.cuh"

namespace psb {

namespace {

// Best-of-poles record per trial period (period_search_BOINC.cpp:811-931).
struct RecordOut {
    double period_h, rms, chi2, dark_pct, lambda_deg, beta_deg;
};

__global__ void period_reduce_kernel(const FitOut* fits, int n_periods, double ndata_m3, int prepass, RecordOut* rec) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_periods) return;
    double per_best = 0, dark_best = 0, la_best = 0, be_best = 0, dev_best = 1e40;
    for (int m = 0; m < 10; m++) {
        const FitOut& f = fits[(size_t)n * 10 + m];
        if (f.dev < dev_best) {
            dev_best = f.dev;
            per_best = f.prd;
            dark_best = f.dark / f.totarea * 100;
            la_best = f.la;
            be_best = f.be;
        }
    }
    if (la_best < 0) la_best += 360;
    if (prepass && isnan(dark_best)) dark_best = 1.0;
    RecordOut r;
    r.period_h = 24 * per_best;
    r.rms = dev_best;
    r.chi2 = dev_best * dev_best * ndata_m3;
    r.dark_pct = dark_best;
    r.lambda_deg = la_best;
    r.beta_deg = be_best;
    rec[n] = r;
}

// Batched variant: global period g belongs to the asteroid a with
// per_off[a] <= g < per_off[a+1].
__global__ void period_reduce_batch_kernel(const FitOut* fits, const int* n_periods_dev, int n_ast, const int* per_off,
                                           const double* ndata_m3, RecordOut* rec) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= *n_periods_dev) return;
    int lo = 0, hi = n_ast - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (per_off[mid] <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    double per_best = 0, dark_best = 0, la_best = 0, be_best = 0, dev_best = 1e40;
    for (int m = 0; m < 10; m++) {
        const FitOut& f = fits[(size_t)g * 10 + m];
        if (f.dev < dev_best) {
            dev_best = f.dev;
            per_best = f.prd;
            dark_best = f.dark / f.totarea * 100;
            la_best = f.la;
            be_best = f.be;
        }
    }
    if (la_best < 0) la_best += 360;
    RecordOut r;
    r.period_h = 24 * per_best;
    r.rms = dev_best;
    r.chi2 = dev_best * dev_best * ndata_m3[lo];
    r.dark_pct = dark_best;
    r.lambda_deg = la_best;
    r.beta_deg = be_best;
    rec[g] = r;
}

}  // namespace

cudaError_t launch_period_reduce_batch(const FitOut* fits, const int* n_periods_dev, int max_periods, int n_ast,
                                       const int* per_off, const double* ndata_m3, void* records, cudaStream_t s) {
    if (max_periods <= 0) return cudaSuccess;
    const int tb = 128;
    period_reduce_batch_kernel<<<(max_periods + tb - 1) / tb, tb, 0, s>>>(fits, n_periods_dev, n_ast, per_off, ndata_m3,
                                                                          (RecordOut*)records);
    return cudaGetLastError();
}

size_t fp64_smem_bytes(const DevProblem& P) { return fitimpl::make_layout(P).bytes; }

int fp64_max_blocks_per_sm(const DevProblem& P, int* threads) {
    if (threads) *threads = fitcommon::kThreads;
    switch (P.NCB) {
        case 8: return fitimpl::max_blocks_t<8, false>(P);
        case 16: return fitimpl::max_blocks_t<16, false>(P);
        case 24: return fitimpl::max_blocks_t<24, false>(P);
        case 32: return fitimpl::max_blocks_t<32, false>(P);
        case 40: return fitimpl::max_blocks_t<40, false>(P);
        case 48: return fitimpl::max_blocks_t<48, false>(P);
        case 56: return fitimpl::max_blocks_t<56, false>(P);
        case 64: return fitimpl::max_blocks_t<64, false>(P);
        case 72: return fitimpl::max_blocks_t<72, false>(P);
        case 80: return fitimpl::max_blocks_t<80, false>(P);
        case 88: return fitimpl::max_blocks_t<88, false>(P);
        default: return 0;
    }
}

cudaError_t launch_fp64_fits(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s) {
    if (P.nq <= 0 || P.mfit > P.NCB + 8) return cudaErrorInvalidValue;
    switch (P.NCB) {
        case 8: return fitimpl::launch_fits_t<8, false>(P, dP, B, grid, s);
        case 16: return fitimpl::launch_fits_t<16, false>(P, dP, B, grid, s);
        case 24: return fitimpl::launch_fits_t<24, false>(P, dP, B, grid, s);
        case 32: return fitimpl::launch_fits_t<32, false>(P, dP, B, grid, s);
        case 40: return fitimpl::launch_fits_t<40, false>(P, dP, B, grid, s);
        case 48: return fitimpl::launch_fits_t<48, false>(P, dP, B, grid, s);
        case 56: return fitimpl::launch_fits_t<56, false>(P, dP, B, grid, s);
        case 64: return fitimpl::launch_fits_t<64, false>(P, dP, B, grid, s);
        case 72: return fitimpl::launch_fits_t<72, false>(P, dP, B, grid, s);
        case 80: return fitimpl::launch_fits_t<80, false>(P, dP, B, grid, s);
        case 88: return fitimpl::launch_fits_t<88, false>(P, dP, B, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fp64_eval(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s) {
    if (P.nq <= 0 || P.mfit > P.NCB + 8) return cudaErrorInvalidValue;
    switch (P.NCB) {
        case 8: return fitimpl::launch_eval_t<8, false>(P, dP, E, s);
        case 16: return fitimpl::launch_eval_t<16, false>(P, dP, E, s);
        case 24: return fitimpl::launch_eval_t<24, false>(P, dP, E, s);
        case 32: return fitimpl::launch_eval_t<32, false>(P, dP, E, s);
        case 40: return fitimpl::launch_eval_t<40, false>(P, dP, E, s);
        case 48: return fitimpl::launch_eval_t<48, false>(P, dP, E, s);
        case 56: return fitimpl::launch_eval_t<56, false>(P, dP, E, s);
        case 64: return fitimpl::launch_eval_t<64, false>(P, dP, E, s);
        case 72: return fitimpl::launch_eval_t<72, false>(P, dP, E, s);
        case 80: return fitimpl::launch_eval_t<80, false>(P, dP, E, s);
        case 88: return fitimpl::launch_eval_t<88, false>(P, dP, E, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_period_reduce(const FitOut* fits, int n_periods, double ndata_m3, int prepass, void* records,
                                 cudaStream_t s) {
    if (n_periods <= 0) return cudaSuccess;
    const int tb = 128;
    period_reduce_kernel<<<(n_periods + tb - 1) / tb, tb, 0, s>>>(fits, n_periods, ndata_m3, prepass,
                                                                  (RecordOut*)records);
    return cudaGetLastError();
}

}  // namespace psb

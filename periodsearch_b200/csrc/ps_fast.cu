// Fast FP64 form of the convex-inversion fit (PS_FORM_FAST): the FP64 fit
// kernels of ps_fit_impl.cuh with kFast = true, compiled with fused
// multiply-add contraction.  Every quantity stays FP64; the per-(point,
// facet) derivative work is rearranged (one reciprocal, facet-summed rotation
// vectors) and fused, so results differ from the reference-order form by
// rounding only -- the same order of difference as the reference rebuilt with
// FMA contraction.
#include <cuda_runtime.h>

#include "ps_device.hpp"
#include "ps_fit_common.cuh"
#include "ps_fit_impl.cuh"

namespace psb {

size_t fast_smem_bytes(const DevProblem& P) { return fitimpl::make_layout(P).bytes; }

int fast_max_blocks_per_sm(const DevProblem& P, int* threads) {
    if (threads) *threads = fitcommon::kThreads;
    switch (P.NCB) {
        case 8: return fitimpl::max_blocks_t<8, true>(P);
        case 16: return fitimpl::max_blocks_t<16, true>(P);
        case 24: return fitimpl::max_blocks_t<24, true>(P);
        case 32: return fitimpl::max_blocks_t<32, true>(P);
        case 40: return fitimpl::max_blocks_t<40, true>(P);
        case 48: return fitimpl::max_blocks_t<48, true>(P);
        case 56: return fitimpl::max_blocks_t<56, true>(P);
        case 64: return fitimpl::max_blocks_t<64, true>(P);
        case 72: return fitimpl::max_blocks_t<72, true>(P);
        case 80: return fitimpl::max_blocks_t<80, true>(P);
        case 88: return fitimpl::max_blocks_t<88, true>(P);
        default: return 0;
    }
}

cudaError_t launch_fast_fits(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s) {
    if (P.nq <= 0 || P.mfit > P.NCB + 8) return cudaErrorInvalidValue;
    switch (P.NCB) {
        case 8: return fitimpl::launch_fits_t<8, true>(P, dP, B, grid, s);
        case 16: return fitimpl::launch_fits_t<16, true>(P, dP, B, grid, s);
        case 24: return fitimpl::launch_fits_t<24, true>(P, dP, B, grid, s);
        case 32: return fitimpl::launch_fits_t<32, true>(P, dP, B, grid, s);
        case 40: return fitimpl::launch_fits_t<40, true>(P, dP, B, grid, s);
        case 48: return fitimpl::launch_fits_t<48, true>(P, dP, B, grid, s);
        case 56: return fitimpl::launch_fits_t<56, true>(P, dP, B, grid, s);
        case 64: return fitimpl::launch_fits_t<64, true>(P, dP, B, grid, s);
        case 72: return fitimpl::launch_fits_t<72, true>(P, dP, B, grid, s);
        case 80: return fitimpl::launch_fits_t<80, true>(P, dP, B, grid, s);
        case 88: return fitimpl::launch_fits_t<88, true>(P, dP, B, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fast_eval(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s) {
    if (P.nq <= 0 || P.mfit > P.NCB + 8) return cudaErrorInvalidValue;
    switch (P.NCB) {
        case 8: return fitimpl::launch_eval_t<8, true>(P, dP, E, s);
        case 16: return fitimpl::launch_eval_t<16, true>(P, dP, E, s);
        case 24: return fitimpl::launch_eval_t<24, true>(P, dP, E, s);
        case 32: return fitimpl::launch_eval_t<32, true>(P, dP, E, s);
        case 40: return fitimpl::launch_eval_t<40, true>(P, dP, E, s);
        case 48: return fitimpl::launch_eval_t<48, true>(P, dP, E, s);
        case 56: return fitimpl::launch_eval_t<56, true>(P, dP, E, s);
        case 64: return fitimpl::launch_eval_t<64, true>(P, dP, E, s);
        case 72: return fitimpl::launch_eval_t<72, true>(P, dP, E, s);
        case 80: return fitimpl::launch_eval_t<80, true>(P, dP, E, s);
        case 88: return fitimpl::launch_eval_t<88, true>(P, dP, E, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace psb

// Device-side data of the B200 period scan: the per-asteroid tables in HBM,
// the per-fit result record and the launch interface of the fit kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace psb {

// Per-asteroid tables, all device pointers, 0-based.
//  rows: n_points data rows (lightcurve order) followed by 3 convexity rows.
struct DevProblem {
    int n_points, n_rows, n_lc;      // n_lc counts the convexity pseudo-curve
    int F, C, NCB, nq, lmax, mmax, ma, mfit;
    int npad;                        // leading dimension of the J scratch
    // points [n_points]
    const double *t, *ex, *ey, *ez, *e0x, *e0y, *e0z, *alpha;
    // rows [n_rows]
    const double *yobs, *sig, *sig2i, *wght;
    // lightcurves [n_lc] (+1 for lc_start)
    const int *lc_start, *lc_rel, *lc_npts;
    // facets
    const double* fac;   // [F][4]: nx, ny, nz, darea
    const double* dsph;  // [F][NCB], zero padded beyond C
    const double* cpl;   // [F][nq]: Pleg in curv's (m, l) order
    const double* cfc;   // [F][mmax+1]
    const double* cfs;   // [F][mmax+1]
    const int* free_idx; // [mfit] parameter index of each free parameter
    const double* cg_first;  // [C]
    const double* pole0;     // [10][2]: initial beta' and lambda [rad]
    // tile shapes (ps_set_tiles / ps_autotune): the fast form's facets per
    // staged chunk and alpha rows per tile, and the points sorted together
    int fch, rt, sortseg;
    const float* fac32;          // [F][4]: nx, ny, nz, 0 (FP32 copies, mixed form)
    // mixed-precision form only
    const uint16_t* bsw;         // [nchunk][2][64 x 64] BF16 hi/lo of Dsph, swizzled K-major tiles
    int nchunk;                  // facet chunks of 64 (F padded up)
    int* err;                    // device error word (bounded waits that gave up)
    unsigned int max_polls;      // polls of an ordinary bounded wait before it gives up
    // scalars
    double phi0, conw_r, alamda_start, alamda_incr, log_cl, par1, par2, par3, ndata_m3;
    double freq_start, freq_step;
    int n_iter_max, n_iter_min;
    double iter_diff_max;
};

// One fit's outcome (the quantities period_search_BOINC.cpp:900-920 reads).
struct FitOut {
    double dev, dark, totarea, prd, la, be, chisq;
    int niter, status;
    unsigned int dur_us;  // the fit's duration [us] by the GPU's global timer
    unsigned int end_us;  // the global timer at the fit's end [us], low 32 bits
};
static_assert(sizeof(FitOut) == 72, "the C ABI documents 72 bytes per fit");

// A batch of fits: fit w is trial period n_from + w / 10, pole w % 10 + 1,
// unless `freq_override` > 0 (single-fit API), then the only fit uses it.
struct FitBatch {
    int n_from;
    int n_fits;
    int pole_override;       // 1..10 for the single-fit API, else 0
    double freq_override;
    int* queue;              // work counter, zeroed before launch
    FitOut* out;             // [n_fits]
    double* scratch;         // per resident CTA: J^T (ma x npad) + y (npad)
    long long scratch_stride;
    // Several asteroids in one launch (the problem pointer is then an array):
    // fits [ast_fit_off[a], ast_fit_off[a+1]) belong to asteroid a, ten per
    // trial period from period ast_n_from[a].  n_ast == 0: one asteroid.
    // n_fits_dev, if set, holds the fit count (kept in device memory so that a
    // captured CUDA graph can be replayed for batches of any size).
    int n_ast;
    const int* ast_fit_off;
    const int* ast_n_from;
    const int* n_fits_dev;
    // Optional order of the work queue over the asteroids (n_ast > 1): the
    // queue hands out the fits of ast_order[0] first, then ast_order[1], ...;
    // ast_ord_off[k] = queue position of the first fit of ast_order[k].
    const int* ast_order;
    const int* ast_ord_off;
};

// Diagnostics of one evaluation (ps_mrqcof / ps_model): J, y, alpha, beta.
struct EvalOut {
    const double* a;   // [ma] parameters
    double* alpha;     // [mfit*mfit]
    double* beta;      // [mfit]
    double* chisq;     // [1]
    double* y;         // [n_rows] normalised model
    double* J;         // [n_rows*ma] normalised Jacobian, row-major
    double* scratch;
};

size_t fp64_smem_bytes(const DevProblem& P);
int fp64_max_blocks_per_sm(const DevProblem& P, int* threads);
// P is the host copy (sizes, launch shape); dP the same struct in device memory.
cudaError_t launch_fp64_fits(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s);
cudaError_t launch_fp64_eval(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s);
// Fast FP64 form (ps_fast.cu): same launch interface as the FP64 form.
size_t fast_smem_bytes(const DevProblem& P);
int fast_max_blocks_per_sm(const DevProblem& P, int* threads);
cudaError_t launch_fast_fits(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s);
cudaError_t launch_fast_eval(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s);

// Mixed-precision form (ps_mixed.cu).  The J scratch holds FP32 columns
// (ma x npad floats) followed by the FP64 model values (npad doubles).
size_t mixed_smem_bytes(const DevProblem& P);
int mixed_max_blocks_per_sm(const DevProblem& P, int* threads);
cudaError_t launch_mixed_fits(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s);
cudaError_t launch_mixed_eval(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s);
inline long long mixed_scratch_doubles(const DevProblem& P) { return ((long long)P.ma * P.npad + 1) / 2 + P.npad; }

// Best-of-poles records for a batch: periods [per_off[a], per_off[a+1]) of
// the concatenated records belong to asteroid a (ndata_m3[a]); the period
// count is read from *n_periods_dev.
cudaError_t launch_period_reduce_batch(const FitOut* fits, const int* n_periods_dev, int max_periods, int n_ast,
                                       const int* per_off, const double* ndata_m3, void* records, cudaStream_t s);

cudaError_t launch_period_reduce(const FitOut* fits, int n_periods, double ndata_m3, int prepass,
                                 void* records /* ps_record[n_periods] */, cudaStream_t s);

}  // namespace psb

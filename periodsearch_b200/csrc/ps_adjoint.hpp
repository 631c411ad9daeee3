// Matrix-free chi2 gradient and Gauss-Newton product (ps_adjoint.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "ps_device.hpp"

namespace psb {

// Device work arrays of one matrix-free evaluation (all carved from one
// buffer of adjoint_work_doubles(P) doubles).
struct AdjWork {
    const double* a;  // [ma] parameters
    const double* v;  // [ma] direction (zero on fixed parameters); null: gradient mode
    double *g, *area, *z, *z0, *qs, *qs0;  // [F]
    double* dres;                          // [3][C] convexity-row derivatives
    double* misc;                          // scalars (blmatrix, scattering, phase, chck, conv J v)
    double *y, *scale, *jv, *jv0, *lam, *ls, *ls0;  // [N] per point
    double* jns;                           // [8][N] non-shape columns of J
    double* e6;                            // [6][N] e, e0 of every point
    double* u;                             // [n_rows] W (y_obs - y') or W J' v
    double* lcw;                           // [4][n_lc] per-lightcurve sums
    double *q, *q0;                        // [npb][F] per point block
    double* full;                          // [ma + 8] result over all parameters
    double* out;                           // [mfit] result over the free parameters
    double* chi2;                          // [1]
    double* x2part;                        // [nrb] chi2 per row block
    double* pp;                            // [11][nfs][N] per-slice partial sums of the point pass
    int npb, nrb, nfs;
};

size_t adjoint_work_doubles(const DevProblem& P);
// Scalars of the last evaluation at work + adjoint_misc_offset(P): the
// convexity residuals chck (3) at kAdjMiscChk, the facet-area sum at
// kAdjMiscSarea.
size_t adjoint_misc_offset(const DevProblem& P);
constexpr int kAdjMiscChk = 33;
constexpr int kAdjMiscSarea = 36;
// Kernel launches of one launch_adjoint call.
constexpr int kAdjointLaunches = 12;
// chi2 into d_chi2; d_v == nullptr: beta = J^T W (y_obs - y) into d_out,
// else J^T W (J v) (v over all ma parameters, zero on the fixed ones).
cudaError_t launch_adjoint(const DevProblem& P, const DevProblem* dP, double* work, const double* d_a,
                           const double* d_v, double* d_out, double* d_chi2, cudaStream_t s);

}  // namespace psb

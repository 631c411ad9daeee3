// Device building blocks shared by the FP64 and mixed-precision fit
// kernels: pole and spin rotation matrices, per-point geometry, the
// Gauss-Jordan solve and the alpha/beta/chi2 entry map.  Compiled into each
// kernel file under that file's flags (the FP64 form uses -fmad=false).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "ps_device.hpp"

namespace psb {
namespace fitcommon {
// internal linkage: each kernel file gets its own copy
namespace {

constexpr int kThreads = 256;
constexpr double kPiD = 3.14159265358979323846;
constexpr double kTinyD = 1e-8;  // constants.h:10

// blmatrix.c:9-46.  B[i*3+j] = Blmat[i+1][j+1]; D[(d*3+i)*3+j] = Dblm[d+1][i+1][j+1].
__device__ void blmatrix(double bet, double lam, double* B, double* D) {
    double cb = cos(bet), sb = sin(bet), cl = cos(lam), sl = sin(lam);
    B[0] = cb * cl;
    B[1] = cb * sl;
    B[2] = -sb;
    B[3] = -sl;
    B[4] = cl;
    B[5] = 0;
    B[6] = sb * cl;
    B[7] = sb * sl;
    B[8] = cb;
    D[0] = -sb * cl;
    D[1] = -sb * sl;
    D[2] = -cb;
    D[3] = 0;
    D[4] = 0;
    D[5] = 0;
    D[6] = cb * cl;
    D[7] = cb * sl;
    D[8] = -sb;
    D[9] = -cb * sl;
    D[10] = cb * cl;
    D[11] = 0;
    D[12] = -cl;
    D[13] = -sl;
    D[14] = 0;
    D[15] = -sb * sl;
    D[16] = sb * cl;
    D[17] = 0;
}

struct PointGeom {
    double e[3], e0[3];
    double de[3][3], de0[3][3];  // [component][derivative], bright.c:41-53
    double scale, dphp[3];
};

// phasec.c:11-24, matrix.c:11-58 and bright.c:28-53 for data point p.
__device__ __forceinline__ void point_geometry(const DevProblem& P, int p, const double* B, const double* D,
                                               double omg, double p1, double p2, double p3, PointGeom& G) {
    const double alpha = P.alpha[p];
    const double ex_ = exp(-alpha / p2);
    G.scale = 1 + p1 * ex_ + p3 * alpha;
    G.dphp[0] = ex_;
    G.dphp[1] = p1 * ex_ * alpha / (p2 * p2);
    G.dphp[2] = alpha;
    const double t = P.t[p];
    double f = omg * t + P.phi0;
    f = fmod(f, 2 * kPiD);
    const double cf = cos(f), sf = sin(f);
    const double fm[3][3] = {{cf, sf, 0}, {-sf, cf, 0}, {0, 0, 1}};
    const double dfm[3][3] = {{-t * sf, t * cf, 0}, {-t * cf, -t * sf, 0}, {0, 0, 0}};
    double tm[3][3], dtm[3][3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double a = 0, b1 = 0, b2 = 0, b3 = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                a = a + fm[i][k] * B[k * 3 + j];
                b1 = b1 + fm[i][k] * D[k * 3 + j];
                b2 = b2 + fm[i][k] * D[9 + k * 3 + j];
                b3 = b3 + dfm[i][k] * B[k * 3 + j];
            }
            tm[i][j] = a;
            dtm[0][i][j] = b1;
            dtm[1][i][j] = b2;
            dtm[2][i][j] = b3;
        }
    const double ee[3] = {P.ex[p], P.ey[p], P.ez[p]};
    const double ee0[3] = {P.e0x[p], P.e0y[p], P.e0z[p]};
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double a = 0, b = 0;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            a = a + tm[i][j] * ee[j];
            b = b + tm[i][j] * ee0[j];
            double c = 0, d = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                c = c + dtm[j][i][k] * ee[k];
                d = d + dtm[j][i][k] * ee0[k];
            }
            G.de[i][j] = c;
            G.de0[i][j] = d;
        }
        G.e[i] = a;
        G.e0[i] = b;
    }
}

// Block-wide argmax of |a| candidates with the reference's tie rule: the
// largest value wins, among equal values the largest linear index (the last
// one met in row-major scan order, gauss_errc.c:21-28).  idx < 0 = none.
__device__ void block_argmax(double& v, int& idx, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_down_sync(0xffffffffu, v, o);
        int oi = __shfl_down_sync(0xffffffffu, idx, o);
        if (oi >= 0 && (idx < 0 || ov > v || (ov == v && oi > idx))) {
            v = ov;
            idx = oi;
        }
    }
    int* redi = (int*)(red + kThreads / 32);
    if (lane == 0) {
        red[warp] = v;
        redi[warp] = idx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bv = red[0];
        int bi = redi[0];
        for (int w = 1; w < kThreads / 32; w++) {
            if (redi[w] >= 0 && (bi < 0 || red[w] > bv || (red[w] == bv && redi[w] > bi))) {
                bv = red[w];
                bi = redi[w];
            }
        }
        red[kThreads / 16] = bv;
        ((int*)(red + kThreads / 16 + 1))[0] = bi;
    }
    __syncthreads();
    v = red[kThreads / 16];
    idx = ((int*)(red + kThreads / 16 + 1))[0];
}

// gauss_errc.c:9-73 on the n x n row-major matrix a (shared memory) with
// right-hand side b; the solution replaces b.  Returns 0, 1 or 2, the same
// value in every thread.  The final column unscrambling of the inverse is
// omitted: mrqmin (mrqmin.c:59-76) only uses b.
__device__ int gauss_jordan(double* a, double* b, int n, int* ipiv, double* dum, double* red) {
    const int tid = threadIdx.x;
    for (int j = tid; j < n; j += kThreads) ipiv[j] = 0;
    __syncthreads();
    for (int i = 0; i < n; i++) {
        double bv = -1.0;
        int bi = -1;
        for (int idx = tid; idx < n * n; idx += kThreads) {
            const int j = idx / n, k = idx - j * n;
            if (ipiv[j] != 1 && ipiv[k] == 0) {
                const double v = fabs(a[idx]);
                if (v >= bv) {
                    bv = v;
                    bi = idx;
                }
            }
        }
        block_argmax(bv, bi, red);
        if (bi < 0) return 1;  // only NaNs left: the reference ends in error 1
        const int irow = bi / n, icol = bi - irow * n;
        __syncthreads();
        if (tid == 0) ++ipiv[icol];
        if (irow != icol) {
            for (int l = tid; l < n; l += kThreads) {
                const double tmp = a[irow * n + l];
                a[irow * n + l] = a[icol * n + l];
                a[icol * n + l] = tmp;
            }
            if (tid == 0) {
                const double tmp = b[irow];
                b[irow] = b[icol];
                b[icol] = tmp;
            }
        }
        __syncthreads();
        const double piv = a[icol * n + icol];
        if (piv == 0.0) return 2;
        const double pivinv = 1.0 / piv;
        __syncthreads();
        if (tid == 0) a[icol * n + icol] = 1.0;
        __syncthreads();
        for (int l = tid; l < n; l += kThreads) a[icol * n + l] *= pivinv;
        if (tid == 0) b[icol] *= pivinv;
        __syncthreads();
        for (int ll = tid; ll < n; ll += kThreads) dum[ll] = a[ll * n + icol];
        __syncthreads();
        for (int ll = tid; ll < n; ll += kThreads)
            if (ll != icol) a[ll * n + icol] = 0.0;
        __syncthreads();
        for (int idx = tid; idx < n * n; idx += kThreads) {
            const int ll = idx / n, l = idx - ll * n;
            if (ll != icol) a[idx] -= a[icol * n + l] * dum[ll];
        }
        for (int ll = tid; ll < n; ll += kThreads)
            if (ll != icol) b[ll] -= b[icol] * dum[ll];
        __syncthreads();
    }
    return 0;
}

// Output-entry map of the alpha/beta/chi2 accumulation: entry e < tri is
// alpha[j][k] (k <= j, row-major lower triangle), then beta[j] as (j, mfit),
// then chi2 as (mfit, mfit + 1); packed as j | k << 16 in shared memory.
// See the tile layout in evaluate().
__device__ void entry_map(int mfit, int* ent) {
    const int tri = mfit * (mfit + 1) / 2;
    for (int j = threadIdx.x; j < mfit; j += kThreads)
        for (int k = 0; k <= j; k++) ent[j * (j + 1) / 2 + k] = j | (k << 16);
    for (int j = threadIdx.x; j < mfit; j += kThreads) ent[tri + j] = j | (mfit << 16);
    if (threadIdx.x == 0) ent[tri + mfit] = mfit | ((mfit + 1) << 16);
    __syncthreads();
}


}  // namespace
}  // namespace fitcommon
}  // namespace psb

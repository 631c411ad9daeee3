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

// Words of shared memory gauss_jordan (and solve_spd) need in buf for an
// n x n system.
__host__ __device__ constexpr int gj_buf_doubles(int n) { return 4 * n + 4 + 4 * (kThreads / 32); }

// Register tile of gauss_jordan for systems of at most nmax unknowns: rows
// warp + 8 r (r < kR), columns lane + 32 c (c < kC), column n standing for b.
template <int nmax>
struct GjTile {
    static constexpr int kW = kThreads / 32;
    static constexpr int kR = (nmax + kW - 1) / kW;
    static constexpr int kC = (nmax + 1 + 31) / 32;
};

// gauss_errc.c:9-73 on the n x n row-major matrix a (shared memory,
// n <= nmax <= 96) with right-hand side b; the solution replaces b, a is left
// undefined.  Returns 0, 1 or 2, the same value in every thread.  The final
// column unscrambling of the inverse is omitted: mrqmin (mrqmin.c:59-76) only
// uses b.
//
// Full pivoting as in the reference: the pivot is the last element of largest
// magnitude, in row-major order, among rows and columns not yet pivoted; a
// NaN never wins.  Magnitudes are compared as unsigned integers (the bit
// patterns of non-negative doubles are ordered like their values).  Thread
// (warp, lane) holds the elements (warp + 8 r, lane + 32 c) in registers and
// looks for the next pivot while it updates them; per pivot the owners
// publish the pivot row, the row it is swapped with and the pivot column to
// buf, so a step costs two block barriers.  Every element receives the
// reference's operations in the reference's order: the swap,
// a[icol][l] * pivinv, then a[ll][l] - a[icol][l] * dum.
template <int nmax>
__device__ int gauss_jordan(double* a, double* b, int n, double* buf) {
    using T = GjTile<nmax>;
    constexpr int kW = T::kW, kR = T::kR, kC = T::kC;
    static_assert(nmax <= 96 && kR <= 32 && kC <= 32, "tile");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* prow = buf;              // pivot row before the step, [n] = b
    double* orow = buf + n + 1;      // row icol before the step, [n] = b
    double* colv = buf + 2 * n + 2;  // column icol before the step
    unsigned long long* pk = (unsigned long long*)(buf + 3 * n + 4);  // per-warp keys, two generations
    int* pidx = (int*)(pk + 2 * kW);
    double x[kR][kC];
    unsigned rlive = 0, clive = 0;  // owned rows / matrix columns not yet pivoted
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int j = warp + kW * r;
        if (j < n) rlive |= 1u << r;
#pragma unroll
        for (int c = 0; c < kC; c++) {
            const int l = lane + 32 * c;
            x[r][c] = (j < n && l <= n) ? (l < n ? a[j * n + l] : b[j]) : 0.0;
        }
    }
#pragma unroll
    for (int c = 0; c < kC; c++)
        if (lane + 32 * c < n) clive |= 1u << c;
    // candidate over the rows not yet pivoted: the last maximum of |x| in the
    // owned row-major order (>= as in the reference; a NaN never compares),
    // returned as key = |x| bits + 1 (0: none) and its element index
    auto candidate = [&](unsigned long long& bk, int& bi) {
        double bv = -1.0;
        int bs = -1;
        bool cl[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) cl[c] = (clive >> c) & 1u;
#pragma unroll
        for (int r = 0; r < kR; r++) {
            if (!((rlive >> r) & 1u)) continue;
#pragma unroll
            for (int c = 0; c < kC; c++) {
                const double v = fabs(x[r][c]);
                const bool take = cl[c] && v >= bv;
                bv = take ? v : bv;
                bs = take ? r * kC + c : bs;
            }
        }
        bk = bs >= 0 ? (unsigned long long)__double_as_longlong(bv) + 1 : 0ull;
        bi = bs >= 0 ? (warp + kW * (bs / kC)) * n + lane + 32 * (bs % kC) : -1;
    };
    auto warp_max = [&](unsigned long long& bk, int& bi) {
        const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)(bk >> 32));
        const unsigned lo = __reduce_max_sync(0xffffffffu, (unsigned)(bk >> 32) == hi ? (unsigned)bk : 0u);
        const bool top = (unsigned)(bk >> 32) == hi && (unsigned)bk == lo;
        bi = (int)__reduce_max_sync(0xffffffffu, top ? (unsigned)(bi + 1) : 0u) - 1;
        bk = ((unsigned long long)hi << 32) | lo;
    };
    unsigned long long bk;
    int bi;
    candidate(bk, bi);
    for (int i = 0; i < n; i++) {
        warp_max(bk, bi);
        const int gen = (i & 1) * kW;
        if (lane == 0) {
            pk[gen + warp] = bk;
            pidx[gen + warp] = bi;
        }
        __syncthreads();
        bk = lane < kW ? pk[gen + lane] : 0ull;
        bi = lane < kW ? pidx[gen + lane] : -1;
        warp_max(bk, bi);
        if (bk == 0) return 1;  // only NaNs left: the reference ends in error 1
        const int irow = bi / n, icol = bi - irow * n;
        // owners publish rows irow, icol and column icol
        if ((irow & (kW - 1)) == warp) {
            const int rr = irow / kW;
#pragma unroll
            for (int r = 0; r < kR; r++)
                if (r == rr) {
#pragma unroll
                    for (int c = 0; c < kC; c++)
                        if (lane + 32 * c <= n) prow[lane + 32 * c] = x[r][c];
                }
        }
        if ((icol & (kW - 1)) == warp) {
            const int rr = icol / kW;
#pragma unroll
            for (int r = 0; r < kR; r++)
                if (r == rr) {
#pragma unroll
                    for (int c = 0; c < kC; c++)
                        if (lane + 32 * c <= n) orow[lane + 32 * c] = x[r][c];
                }
        }
        if ((icol & 31) == lane) {
            const int cc = icol >> 5;
#pragma unroll
            for (int c = 0; c < kC; c++)
                if (c == cc) {
#pragma unroll
                    for (int r = 0; r < kR; r++)
                        if (warp + kW * r < n) colv[warp + kW * r] = x[r][c];
                }
        }
        __syncthreads();
        const double piv = prow[icol];
        if (piv == 0.0) return 2;
        const double pivinv = 1.0 / piv;
        double pr[kC], orv[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) {
            const int l = lane + 32 * c;
            pr[c] = l <= n ? (l == icol ? 1.0 : prow[l]) * pivinv : 0.0;
            orv[c] = l <= n ? (l == icol ? 0.0 : orow[l]) : 0.0;
        }
        const double odum = orow[icol];
        // the pivot leaves the live set before the next search
        if ((icol & (kW - 1)) == warp) rlive &= ~(1u << (icol / kW));
        if ((icol & 31) == lane) {
            const int cc = icol >> 5;
            clive &= ~(1u << cc);
            // a[ll][icol] = 0 before the reduction (its old value is in colv)
#pragma unroll
            for (int c = 0; c < kC; c++)
                if (c == cc) {
#pragma unroll
                    for (int r = 0; r < kR; r++) x[r][c] = 0.0;
                }
        }
#pragma unroll
        for (int r = 0; r < kR; r++) {
            const int j = warp + kW * r;
            if (j >= n) continue;
            if (j == icol) {
#pragma unroll
                for (int c = 0; c < kC; c++) x[r][c] = pr[c];
            } else if (j == irow) {
#pragma unroll
                for (int c = 0; c < kC; c++) x[r][c] = orv[c] - pr[c] * odum;
            } else {
                const double dum = colv[j];
#pragma unroll
                for (int c = 0; c < kC; c++) x[r][c] = x[r][c] - pr[c] * dum;
            }
        }
        candidate(bk, bi);
    }
#pragma unroll
    for (int r = 0; r < kR; r++)
#pragma unroll
        for (int c = 0; c < kC; c++) {
            const int j = warp + kW * r, l = lane + 32 * c;
            if (j < n && l == n) b[j] = x[r][c];
        }
    __syncthreads();
    return 0;
}

// Solve a x = b for a symmetric positive definite n x n row-major matrix a
// (shared memory, n <= nmax <= 96; the damped alpha of an LM step, alpha with
// its diagonal times 1 + lambda) by Gauss-Jordan elimination with the
// diagonal as pivots, in order: no pivot search, one block barrier per step.
// The solution replaces b.  Returns 0, or -1 as soon as a pivot is not
// above kSpdPivot times its original diagonal entry (a singular, nearly
// singular or indefinite system, or NaN), leaving a and b untouched, so that
// the caller runs gauss_jordan, the reference's full-pivot solve, for those:
// there the pivot order decides the solution's ill-determined directions
// and the singular verdict.  Same register tile as gauss_jordan; per step the owners publish
// the pivot row and the pivot column to alternating halves of buf.
constexpr double kSpdPivot = 1e-3;
template <int nmax>
__device__ int solve_spd(const double* a, double* b, int n, double* buf) {
    using T = GjTile<nmax>;
    constexpr int kW = T::kW, kR = T::kR, kC = T::kC;
    static_assert(nmax <= 96 && kR <= 32 && kC <= 32, "tile");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double x[kR][kC];
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int j = warp + kW * r;
#pragma unroll
        for (int c = 0; c < kC; c++) {
            const int l = lane + 32 * c;
            x[r][c] = (j < n && l <= n) ? (l < n ? a[j * n + l] : b[j]) : 0.0;
        }
    }
    for (int i = 0; i < n; i++) {
        double* prow = buf + (i & 1) * (2 * n + 2);  // row i, [n] = b_i
        double* colv = prow + n + 1;                 // column i
        if ((i & (kW - 1)) == warp) {
            const int ri = i / kW;
#pragma unroll
            for (int r = 0; r < kR; r++)
                if (r == ri) {
#pragma unroll
                    for (int c = 0; c < kC; c++)
                        if (lane + 32 * c <= n) prow[lane + 32 * c] = x[r][c];
                }
        }
        if ((i & 31) == lane) {
            const int ci = i >> 5;
#pragma unroll
            for (int c = 0; c < kC; c++)
                if (c == ci) {
#pragma unroll
                    for (int r = 0; r < kR; r++)
                        if (warp + kW * r < n) colv[warp + kW * r] = x[r][c];
                }
        }
        __syncthreads();
        const double piv = prow[i];
        if (!(piv > kSpdPivot * a[i * n + i])) {  // the same value in every thread
            __syncthreads();  // nobody reads buf any more when the caller reuses it
            return -1;
        }
        const double pivinv = 1.0 / piv;
        double pr[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) {
            const int l = lane + 32 * c;
            pr[c] = l <= n ? prow[l] * pivinv : 0.0;
        }
#pragma unroll
        for (int r = 0; r < kR; r++) {
            const int j = warp + kW * r;
            if (j >= n) continue;
            if (j == i) {
#pragma unroll
                for (int c = 0; c < kC; c++) x[r][c] = pr[c];
            } else {
                const double dum = colv[j];
#pragma unroll
                for (int c = 0; c < kC; c++) x[r][c] = x[r][c] - pr[c] * dum;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kR; r++)
#pragma unroll
        for (int c = 0; c < kC; c++) {
            const int j = warp + kW * r, l = lane + 32 * c;
            if (j < n && l == n) b[j] = x[r][c];
        }
    __syncthreads();
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

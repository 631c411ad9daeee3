// Matrix-free derivatives of the convex-inversion model (PS_FORM_FAST
// arithmetic, FP64): chi2 and beta = J^T W (y_obs - y) -- the chi2 gradient is
// -2 beta -- and the Gauss-Newton product J^T W (J v), without forming J.
//
// The shape block of J is J_pk = Scale_p sum_f Darea_f s_pf g_f Dsph_fk
// (bright.c:78-85 with Dg = g Dsph, curv.c:31-35).  Its products with a vector
// and its transpose need no p x k array:
//   (J v)_p   = Scale_p sum_f Area_f s_pf z_f,      z = Dsph v        (forward)
//   (J^T l)_k = sum_f (sum_p l_p Scale_p s_pf) Area_f Dsph_fk       (adjoint)
// so one product costs two passes over the (point, facet) pairs plus two
// F x C contractions instead of the N F C of the explicit Jacobian.  The eight
// non-shape columns are formed per point.  The relative-lightcurve
// normalisation (mrqcof.c:92-104), J'_r = coef (J_r - y_r dave / ave) with
// dave = sum_r J_r and J'_r1 = 0, becomes per-lightcurve scalars:
//   (J' v)_r  = coef ((J v)_r - y_r sum_{r'} (J v)_{r'} / ave)   (v_1 left out)
//   J'^T u    = J^T l,  l_r = coef (u_r - sum_{r'} y_{r'} u_{r'} / ave).
// The convexity rows (conv.c:12-29) are added explicitly.  Every reduction
// runs in a fixed order, so results are deterministic.
//
// Kernels, in stream order, each spread over the GPU: adj_curv (thread per
// facet: blmatrix, curv, z), adj_conv (warp per convexity-row sum),
// adj_points (thread per point and facet slice), adj_points_fin (thread per
// point: the slices' sums in order, the per-point results), adj_lc (CTA per lightcurve: model and J v
// sums), adj_rowsum (rows: normalised model, residual, u, per-CTA chi2),
// adj_lck (CTA per lightcurve: the adjoint's y.u sum), adj_weights (thread
// per point), adj_facets (thread per facet, blocks of points), adj_qs
// (thread per facet), adj_cols (CTA per output column: the F x C
// contraction and the non-shape columns), adj_out (the free parameters).
#include <cuda_runtime.h>
#include <math.h>

#include "ps_adjoint.hpp"
#include "ps_device.hpp"
#include "ps_fit_common.cuh"

namespace psb {
namespace {

using namespace fitcommon;

constexpr int kPtThreads = 128;  // adj_points: points per CTA
constexpr int kFacetChunk = 256; // adj_points: facets staged per chunk
constexpr int kFcThreads = 128;  // adj_facets: facets per CTA
constexpr int kPtBlock = 512;    // adj_facets: points per CTA (staged)
constexpr int kRowThreads = 256; // adj_rowsum: rows per CTA
constexpr int kPart = 11;        // adj_points: partial sums per point and facet slice
constexpr int kMaxSlices = 8;    // adj_points: facet slices at most

// Facet slices of the (point, facet) pass: enough CTAs to fill the GPU,
// slices of at least 256 facets.
inline int facet_slices(const DevProblem& P) {
    const int pb = (P.n_points + kPtThreads - 1) / kPtThreads;
    int s = 1;
    while (s < kMaxSlices && pb * s < 4 * 148 && P.F / (2 * s) >= 256) s *= 2;
    return s;
}

// misc slots (X_CHK and X_SAREA are read by the host: kAdjMiscChk, kAdjMiscSarea)
enum { X_B = 0, X_D = 9, X_CL = 27, X_CLS = 28, X_OMG = 29, X_P1 = 30, X_P2 = 31, X_P3 = 32, X_CHK = kAdjMiscChk,
       X_SAREA = kAdjMiscSarea, X_N = 40 };

__device__ double block_sum(double v, double* red) {
    // fixed-order tree: warp shuffles, then warp 0 over the warp partials
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0;
    if (warp == 0) {
        s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[0] = s;
    }
    __syncthreads();
    s = red[0];
    __syncthreads();
    return s;
}

// blmatrix and the scattering/phase scalars (block 0), curv (curv.c:15-37)
// and z = Dsph v, z0 = z without the first coefficient; thread per facet.
__global__ void adj_curv(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    const double* a = W.a;
    const int C = P.C, NCB = P.NCB;
    double* x = W.misc;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        blmatrix(a[C], a[C + 1], x + X_B, x + X_D);
        x[X_CL] = exp(a[C + 6]);
        x[X_CLS] = a[C + 7];
        x[X_OMG] = a[C + 2];
        x[X_P1] = a[C + 3];
        x[X_P2] = a[C + 4];
        x[X_P3] = a[C + 5];
    }
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= P.F) return;
    const double* pl = P.cpl + (size_t)f * P.nq;
    const double* fc = P.cfc + (size_t)f * (P.mmax + 1);
    const double* fs = P.cfs + (size_t)f * (P.mmax + 1);
    double gi = 0;
    int n = 0, q = 0;
    for (int m = 0; m <= P.mmax; m++) {
        for (int l = m; l <= P.lmax; l++) {
            double fsum = a[n] * fc[m];
            n++;
            if (m != 0) {
                fsum = fma(a[n], fs[m], fsum);
                n++;
            }
            gi = fma(pl[q], fsum, gi);
            q++;
        }
    }
    gi = exp(gi);
    W.g[f] = gi;
    W.area[f] = P.fac[(size_t)f * 4 + 3] * gi;
    double z = 0;
    const double* ds = P.dsph + (size_t)f * NCB;
    if (W.v)
        for (int k = 1; k < C; k++) z = fma(ds[k], W.v[k], z);
    W.z0[f] = z;
    W.z[f] = W.v ? fma(ds[0], W.v[0], z) : 0.0;
}

// Convexity rows: chck_nc = sum Area n_nc and dres_nc,k = sum Darea g Dsph_k
// n_nc, and the facet-area sum; one warp per sum (lanes stride the facets,
// fixed-order shuffle tree).
__global__ void adj_conv(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    const int F = P.F, C = P.C, NCB = P.NCB;
    const int job = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (job >= 4 + 3 * C) return;
    double s = 0;
    if (job < 3) {
        for (int f = lane; f < F; f += 32) s = fma(W.area[f], P.fac[(size_t)f * 4 + job], s);
    } else if (job == 3) {
        for (int f = lane; f < F; f += 32) s += W.area[f];
    } else {
        const int nc = (job - 4) / C, k = (job - 4) - nc * C;
        for (int f = lane; f < F; f += 32) s = fma(W.area[f] * P.dsph[(size_t)f * NCB + k], P.fac[(size_t)f * 4 + nc], s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
        if (job < 3)
            W.misc[X_CHK + job] = s;
        else if (job == 3)
            W.misc[X_SAREA] = s;
        else
            W.dres[job - 4] = s;
    }
}

// Per point and facet slice: partial sums over the slice's facets of the
// model brightness and of what the eight non-shape columns and the shape
// part of J v need (br, Area s z, Area s z0, the Lambert / Lommel-Seeliger
// sums, T = sum Area dsmu n, S = sum Area dsmu0 n); grid (point blocks,
// facet slices), so that the (point, facet) pass fills the GPU.
__global__ void __launch_bounds__(kPtThreads) adj_points(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    __shared__ double sf[6][kFacetChunk];  // nx, ny, nz, Area, z, z0
    const int tid = threadIdx.x, F = P.F, N = P.n_points;
    const int p = blockIdx.x * kPtThreads + tid;
    const bool act = p < N;
    const int per = (F + W.nfs - 1) / W.nfs;
    const int fa0 = blockIdx.y * per, fa1 = min(F, fa0 + per);
    const double* x = W.misc;
    const double cl = x[X_CL], cls = x[X_CLS];
    PointGeom G;
    if (act) point_geometry(P, p, x + X_B, x + X_D, x[X_OMG], x[X_P1], x[X_P2], x[X_P3], G);
    double acc[kPart] = {};
    for (int f0 = fa0; f0 < fa1; f0 += kFacetChunk) {
        const int nf = min(kFacetChunk, fa1 - f0);
        __syncthreads();
        for (int i = tid; i < nf; i += kPtThreads) {
            const double* fa = P.fac + (size_t)(f0 + i) * 4;
            sf[0][i] = fa[0];
            sf[1][i] = fa[1];
            sf[2][i] = fa[2];
            sf[3][i] = W.area[f0 + i];
            sf[4][i] = W.z[f0 + i];
            sf[5][i] = W.z0[f0 + i];
        }
        __syncthreads();
        if (!act) continue;
        for (int i = 0; i < nf; i++) {
            const double nx = sf[0][i], ny = sf[1][i], nz = sf[2][i];
            const double mu = G.e[0] * nx + G.e[1] * ny + G.e[2] * nz;
            const double mu0 = G.e0[0] * nx + G.e0[1] * ny + G.e0[2] * nz;
            if (mu > kTinyD && mu0 > kTinyD) {
                const double ar = sf[3][i];
                const double r = 1.0 / (mu + mu0);
                const double s = mu * mu0 * fma(cls, r, cl);
                const double t = ar * s;
                acc[0] += t;                      // br
                acc[1] = fma(t, sf[4][i], acc[1]);  // sum Area s z
                acc[2] = fma(t, sf[5][i], acc[2]);  // sum Area s z0
                const double q0 = mu0 * r, q1 = mu * r;
                const double w = ar * fma(cls * q0, q0, cl * mu0);
                const double w0 = ar * fma(cls * q1, q1, cl * mu);
                acc[3] = fma(w, nx, acc[3]);
                acc[4] = fma(w, ny, acc[4]);
                acc[5] = fma(w, nz, acc[5]);
                acc[6] = fma(w0, nx, acc[6]);
                acc[7] = fma(w0, ny, acc[7]);
                acc[8] = fma(w0, nz, acc[8]);
                const double mm = mu * mu0 * ar;
                acc[9] += mm;                     // sum mu mu0 Area
                acc[10] = fma(mm, r, acc[10]);    // sum mu mu0 Area / (mu + mu0)
            }
        }
    }
    if (!act) return;
    for (int j = 0; j < kPart; j++) W.pp[((size_t)j * W.nfs + blockIdx.y) * N + p] = acc[j];
}

// Per point: the slices' partial sums in slice order, then the model, the
// eight non-shape columns of J, the shape part of J v (with and without the
// first coefficient), Scale, and e, e0 for the adjoint pass.
__global__ void adj_points_fin(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    const int N = P.n_points, C = P.C;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const double* x = W.misc;
    const double cl = x[X_CL];
    PointGeom G;
    point_geometry(P, p, x + X_B, x + X_D, x[X_OMG], x[X_P1], x[X_P2], x[X_P3], G);
    double acc[kPart];
    for (int j = 0; j < kPart; j++) {
        double v = 0;
        for (int k = 0; k < W.nfs; k++) v += W.pp[((size_t)j * W.nfs + k) * N + p];
        acc[j] = v;
    }
    const double br = acc[0], sz = acc[1], sz0 = acc[2], s_cl = acc[9], s_cls = acc[10];
    const double sc = G.scale;
    double jn[8];
    const double T[3] = {acc[3], acc[4], acc[5]}, S[3] = {acc[6], acc[7], acc[8]};
    for (int k = 0; k < 3; k++) {
        double v = 0;
        for (int j = 0; j < 3; j++) v = fma(T[j], G.de[j][k], fma(S[j], G.de0[j][k], v));
        jn[k] = sc * v;
    }
    jn[3] = br * G.dphp[0];
    jn[4] = br * G.dphp[1];
    jn[5] = br * G.dphp[2];
    jn[6] = sc * s_cl * cl;
    jn[7] = sc * s_cls;
    double ns = 0;
    for (int j = 0; j < 8; j++) {
        W.jns[(size_t)j * N + p] = jn[j];
        if (W.v) ns = fma(jn[j], W.v[C + j], ns);
    }
    W.y[p] = br * sc;
    W.scale[p] = sc;
    W.jv[p] = fma(sc, sz, ns);
    W.jv0[p] = fma(sc, sz0, ns);
    for (int c = 0; c < 3; c++) {
        W.e6[(size_t)c * N + p] = G.e[c];
        W.e6[(size_t)(3 + c) * N + p] = G.e0[c];
    }
}

// Lightcurve of data row r (binary search over the lightcurve starts).
__device__ __forceinline__ int lc_of(const DevProblem& P, int r) {
    int lo = 0, hi = P.n_lc - 2;  // the last lightcurve is the convexity pseudo-curve
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.lc_start[mid] <= r)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Per relative lightcurve (one CTA each): ave = sum y, S = sum (J v without
// v_1), coef = sig L / ave (mrqcof.c:53-58, 92-104).
__global__ void adj_lc(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    __shared__ double red[32];
    const int lc = blockIdx.x, nlc = P.n_lc - 1;
    if (!P.lc_rel[lc]) return;
    const int r0 = P.lc_start[lc], r1 = P.lc_start[lc + 1];
    double sy = 0, sj = 0;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        sy += W.y[r];
        sj += W.jv0[r];
    }
    sy = block_sum(sy, red);
    sj = block_sum(sj, red);
    if (threadIdx.x == 0) {
        W.lcw[lc] = sy;
        W.lcw[nlc + lc] = sj;
        W.lcw[3 * nlc + lc] = P.sig[r0] * (double)P.lc_npts[lc] / sy;
    }
}

// Rows: the normalised model and J v, the residual, u = W (y_obs - y') or
// W J' v, and each CTA's share of chi2 (summed in block order by adj_cols).
__global__ void adj_rowsum(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    __shared__ double red[32];
    const int nlc = P.n_lc - 1;
    const double* lc_ave = W.lcw;
    const double* lc_s = W.lcw + nlc;
    const double* lc_coef = W.lcw + 3 * nlc;
    double x2 = 0;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < P.n_rows) {
        double yy, jv;
        if (r < P.n_points) {
            const int lc = lc_of(P, r);
            if (P.lc_rel[lc]) {
                const double coef = lc_coef[lc];
                yy = coef * W.y[r];
                jv = coef * (W.jv0[r] - W.y[r] * lc_s[lc] / lc_ave[lc]);
            } else {
                yy = W.y[r];
                jv = W.jv[r];
            }
        } else {
            // the convexity rows; their J v needs the C-term dot products
            const int nc = r - P.n_points;
            yy = W.misc[X_CHK + nc];
            jv = 0;
            if (W.v)
                for (int k = 0; k < P.C; k++) jv = fma(W.dres[nc * P.C + k], W.v[k], jv);
        }
        const double w = P.sig2i[r] * P.wght[r];
        const double dy = P.yobs[r] - yy;
        x2 = dy * dy * w;
        W.u[r] = W.v ? w * jv : w * dy;
    }
    x2 = block_sum(x2, red);
    if (threadIdx.x == 0) W.x2part[blockIdx.x] = x2;
}

// Per relative lightcurve (one CTA each): kappa = sum y u / ave.
__global__ void adj_lck(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    __shared__ double red[32];
    const int lc = blockIdx.x, nlc = P.n_lc - 1;
    if (!P.lc_rel[lc]) return;
    const int r0 = P.lc_start[lc], r1 = P.lc_start[lc + 1];
    double s = 0;
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) s = fma(W.y[r], W.u[r], s);
    s = block_sum(s, red);
    if (threadIdx.x == 0) W.lcw[2 * nlc + lc] = s / W.lcw[lc];
}

// Adjoint weights per point: l (all columns), l0 (the first shape
// coefficient, zero on relative rows); ls = l Scale for the facet pass.
__global__ void adj_weights(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= P.n_points) return;
    const int nlc = P.n_lc - 1;
    const int lc = lc_of(P, r);
    double l = W.u[r], l0 = l;
    if (P.lc_rel[lc]) {
        l = W.lcw[3 * nlc + lc] * (W.u[r] - W.lcw[2 * nlc + lc]);
        l0 = 0.0;
    }
    W.lam[r] = l;
    W.ls[r] = l * W.scale[r];
    W.ls0[r] = l0 * W.scale[r];
}

// q_f = sum_p ls_p s_pf and q0_f = sum_p ls0_p s_pf over a block of points;
// thread per facet, points staged in shared memory.
__global__ void __launch_bounds__(kFcThreads) adj_facets(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    __shared__ double sp[8][kPtBlock];  // e (3), e0 (3), ls, ls0
    const int f = blockIdx.x * kFcThreads + threadIdx.x;
    const int p0 = blockIdx.y * kPtBlock;
    const int np = min(kPtBlock, P.n_points - p0);
    for (int i = threadIdx.x; i < np; i += kFcThreads) {
        for (int c = 0; c < 6; c++) sp[c][i] = W.e6[(size_t)c * P.n_points + p0 + i];
        sp[6][i] = W.ls[p0 + i];
        sp[7][i] = W.ls0[p0 + i];
    }
    __syncthreads();
    if (f >= P.F) return;
    const double cl = W.misc[X_CL], cls = W.misc[X_CLS];
    const double nx = P.fac[(size_t)f * 4 + 0], ny = P.fac[(size_t)f * 4 + 1], nz = P.fac[(size_t)f * 4 + 2];
    double q = 0, q0 = 0;
    for (int i = 0; i < np; i++) {
        const double mu = sp[0][i] * nx + sp[1][i] * ny + sp[2][i] * nz;
        const double mu0 = sp[3][i] * nx + sp[4][i] * ny + sp[5][i] * nz;
        if (mu > kTinyD && mu0 > kTinyD) {
            const double r = 1.0 / (mu + mu0);
            const double s = mu * mu0 * fma(cls, r, cl);
            q = fma(sp[6][i], s, q);
            q0 = fma(sp[7][i], s, q0);
        }
    }
    W.q[(size_t)blockIdx.y * P.F + f] = q;
    W.q0[(size_t)blockIdx.y * P.F + f] = q0;
}

// Q_f = Area_f sum over the point blocks of q (q0); thread per facet.
__global__ void adj_qs(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= P.F) return;
    double s = 0, s0 = 0;
    for (int b = 0; b < W.npb; b++) {
        s += W.q[(size_t)b * P.F + f];
        s0 += W.q0[(size_t)b * P.F + f];
    }
    W.qs[f] = s * W.area[f];
    W.qs0[f] = s0 * W.area[f];
}

// One CTA per output column k < C + 8: out_k = sum_f Q_f Dsph_fk (Q0 for the
// first coefficient) + the convexity rows, out_{C+j} = sum_p l_p J_p,C+j;
// block C + 8 sums the per-CTA chi2 shares in block order.
__global__ void adj_cols(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    __shared__ double red[32];
    const int k = blockIdx.x, C = P.C, F = P.F;
    double s = 0;
    if (k < C) {
        const double* q = k == 0 ? W.qs0 : W.qs;
        for (int f = threadIdx.x; f < F; f += blockDim.x) s = fma(q[f], P.dsph[(size_t)f * P.NCB + k], s);
    } else if (k < C + 8) {
        const double* col = W.jns + (size_t)(k - C) * P.n_points;
        for (int p = threadIdx.x; p < P.n_points; p += blockDim.x) s = fma(W.lam[p], col[p], s);
    } else {
        for (int b = threadIdx.x; b < W.nrb; b += blockDim.x) s += W.x2part[b];
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) {
        if (k < C) {
            for (int nc = 0; nc < 3; nc++) s = fma(W.dres[nc * C + k], W.u[P.n_points + nc], s);
            W.full[k] = s;
        } else if (k < C + 8) {
            W.full[k] = s;
        } else {
            *W.chi2 = s;
        }
    }
}

// The free parameters' entries.
__global__ void adj_out(const DevProblem* __restrict__ Pp, AdjWork W) {
    const DevProblem& P = *Pp;
    for (int i = threadIdx.x; i < P.mfit; i += blockDim.x) W.out[i] = W.full[P.free_idx[i]];
}

}  // namespace

size_t adjoint_misc_offset(const DevProblem& P) { return (size_t)P.F * 7 + 3 * (size_t)P.C; }

size_t adjoint_work_doubles(const DevProblem& P) {
    const size_t N = P.n_points, F = P.F;
    const size_t npb = (N + kPtBlock - 1) / kPtBlock;
    const size_t nrb = ((size_t)P.n_rows + kRowThreads - 1) / kRowThreads;
    return 2 * (size_t)P.ma + F * 7 + 3 * (size_t)P.C + X_N + N * (8 + 6 + 7) + P.n_rows + 4 * (size_t)P.n_lc +
           2 * npb * F + 2 * (size_t)P.ma + 8 + nrb + (size_t)kPart * kMaxSlices * N;
}

cudaError_t launch_adjoint(const DevProblem& P, const DevProblem* dP, double* work, const double* d_a,
                           const double* d_v, double* d_out, double* d_chi2, cudaStream_t s) {
    AdjWork W{};
    const size_t N = P.n_points, F = P.F;
    W.npb = (int)((N + kPtBlock - 1) / kPtBlock);
    double* o = work;
    auto take = [&](size_t n) {
        double* r = o;
        o += n;
        return r;
    };
    W.a = d_a;
    W.v = d_v;
    W.g = take(F);
    W.area = take(F);
    W.z = take(F);
    W.z0 = take(F);
    W.qs = take(F);
    W.qs0 = take(F);
    take(F);
    W.dres = take(3 * (size_t)P.C);
    W.misc = take(X_N);
    W.y = take(N);
    W.scale = take(N);
    W.jv = take(N);
    W.jv0 = take(N);
    W.lam = take(N);
    W.ls = take(N);
    W.ls0 = take(N);
    W.jns = take(8 * N);
    W.e6 = take(6 * N);
    W.u = take(P.n_rows);
    W.lcw = take(4 * (size_t)P.n_lc);
    W.q = take((size_t)W.npb * F);
    W.q0 = take((size_t)W.npb * F);
    W.full = take(P.ma + 8);
    W.nrb = (int)(((size_t)P.n_rows + kRowThreads - 1) / kRowThreads);
    W.x2part = take((size_t)W.nrb);
    W.nfs = facet_slices(P);
    W.pp = take((size_t)kPart * W.nfs * N);
    W.out = d_out;
    W.chi2 = d_chi2;
    const int nlc = P.n_lc - 1;
    const unsigned fb = (unsigned)((F + 255) / 256);
    adj_curv<<<fb, 256, 0, s>>>(dP, W);
    adj_conv<<<(unsigned)((4 + 3 * P.C + 7) / 8), 256, 0, s>>>(dP, W);
    adj_points<<<dim3((unsigned)((N + kPtThreads - 1) / kPtThreads), (unsigned)W.nfs), kPtThreads, 0, s>>>(dP, W);
    adj_points_fin<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(dP, W);
    if (nlc > 0) adj_lc<<<(unsigned)nlc, 256, 0, s>>>(dP, W);
    adj_rowsum<<<(unsigned)W.nrb, kRowThreads, 0, s>>>(dP, W);
    if (nlc > 0) adj_lck<<<(unsigned)nlc, 256, 0, s>>>(dP, W);
    adj_weights<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(dP, W);
    adj_facets<<<dim3((unsigned)((F + kFcThreads - 1) / kFcThreads), (unsigned)W.npb), kFcThreads, 0, s>>>(dP, W);
    adj_qs<<<fb, 256, 0, s>>>(dP, W);
    adj_cols<<<(unsigned)(P.C + 9), 256, 0, s>>>(dP, W);
    adj_out<<<1, 128, 0, s>>>(dP, W);
    return cudaGetLastError();
}

}  // namespace psb

// FP64 fit kernels, shared by the reference-order form (ps_fp64.cu, built
// with -fmad=false, kFast = false) and the fast FP64 form (ps_fast.cu, FMA
// contraction, kFast = true).  kFast changes only how the per-(point, facet)
// brightness derivatives and the facet/row sums are evaluated: one
// reciprocal instead of four divisions, rotation derivatives through the
// facet-summed vectors sum(Area dsmu n) and sum(Area dsmu0 n) (bright.c:88-104
// rearranged), fused multiply-adds; the model, every sum and the solve stay
// FP64.  The structure is described in ps_fp64.cu.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ps_device.hpp"
#include "ps_fit_common.cuh"

namespace psb {
namespace fitimpl {
namespace {

using namespace fitcommon;

constexpr int kFch = 64;     // facets per shared-memory chunk (reference-order form)
constexpr int kRt = 32;      // rows per alpha tile (reference-order form)
constexpr int kMf = 128;     // facets per staged chunk of the model-only pass

constexpr int kMp = 4;       // points per thread at most in the model-only pass

// 1/x for x in (2e-8, 2] (mu + mu0 of a visible pair), fast form only: the
// hardware's approximate FP64 reciprocal refined by two Newton-Raphson steps
// r <- r + r (1 - x r), each of which squares the relative error, so the
// result is within rounding of the IEEE quotient.
__device__ __forceinline__ double rcp_newton(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}
// The fast form takes its facet-chunk and alpha row-tile sizes and both forms
// the point-sort segment from the problem (DevProblem::fch, rt, sortseg):
// runtime tile shapes, chosen by ps_autotune; no choice changes any result.

// Blocks of the alpha/beta/chi2 accumulation for mfit free parameters: for
// each even j0 <= mfit - 1, the 4-column blocks k0 = 4 kb of the lower
// triangle (k0 <= j0 + 1) and the beta block k0 = kB; then the chi2 block
// (jC, kB), kB = jC = mfit rounded up to even.  Packed as j0 | k0 << 16.
__host__ __device__ constexpr int alpha_job_count(int mfit) {
    int n = 1;
    for (int j0 = 0; j0 < mfit; j0 += 2) {
        const int kmax = (j0 + 1) / 4 < (mfit - 1) / 4 ? (j0 + 1) / 4 : (mfit - 1) / 4;
        n += kmax + 2;
    }
    return n;
}

// Offset (doubles) in the work area of the damped matrix the Gauss-Jordan
// solve starts from, after the solve's own buffers.
__host__ __device__ constexpr int gj_covar_off(int mfit) { return (gj_buf_doubles(mfit) + 1) & ~1; }

// Shared-memory layout, offsets in doubles.
struct Layout {
    int cg, atry, alpha, beta, da, g, area, dres, dave, blm, misc, red, perm, work, ipiv, ent;
    int wlen;  // doubles of the work area
    size_t bytes;
};

__host__ __device__ inline Layout make_layout(const DevProblem& P) {
    Layout L;
    int o = 2;  // doubles 0-1: the fit kernel's work-queue slots (fit index, asteroid)
#define PSB_TAKE(field, n) \
    L.field = o;           \
    o += ((n) + 1) & ~1;
    PSB_TAKE(cg, P.ma)
    PSB_TAKE(atry, P.ma)
    PSB_TAKE(alpha, P.mfit * P.mfit)
    PSB_TAKE(beta, P.mfit)
    PSB_TAKE(da, P.mfit)
    PSB_TAKE(g, P.F)
    PSB_TAKE(area, P.F + 128)  // zeros past F: the fast point loop reads whole chunks
    PSB_TAKE(dres, 3 * P.C)
    PSB_TAKE(dave, P.ma + 2)
    PSB_TAKE(blm, 28)
    PSB_TAKE(misc, 32)
    PSB_TAKE(red, 2 * (kThreads / 32) + 2)
    // reference-order form: staged facets and g Dsph, then the rotation
    // derivative vectors of the 128 points of a pass (18 doubles each)
    int chunk = ((kFch * 5 + kFch * P.NCB + 1) & ~1) + 18 * (kThreads / 2);
    // fast form: two staged chunks, dsph rows padded to NCB + 4 doubles
    if (2 * P.fch * (8 + P.NCB) > chunk) chunk = 2 * P.fch * (8 + P.NCB);
    const int kB = (P.mfit + 1) & ~1;
    int tile = kRt * (kB + 2) + kRt * (kB + 4);  // alpha tiles Ws, Js
    const int st8 = (kB + 2 + 7) / 8 * 8 + 4;     // fast form: 8-column tiles, two buffers
    if (2 * P.rt * (st8 + 1) > tile) tile = 2 * P.rt * (st8 + 1);
    int w = chunk > tile ? chunk : tile;
    if (P.mfit + 2 > w) w = P.mfit + 2;
    if (P.sortseg > w) w = P.sortseg;  // sort keys (uint64) before the point loop
    if (4 * kMf > w) w = 4 * kMf;      // model-only pass: staged facet normals and areas
    // Gauss-Jordan: its buffers, then the damped matrix it starts from (covar),
    // which it reads into registers -- covar needs no region of its own
    if (gj_covar_off(P.mfit) + P.mfit * P.mfit > w) w = gj_covar_off(P.mfit) + P.mfit * P.mfit;
    PSB_TAKE(perm, P.sortseg / 2)
    PSB_TAKE(work, w)
    L.wlen = w;
#undef PSB_TAKE
    L.ipiv = o;
    L.ent = o + (P.mfit + 2 + 1) / 2;  // int offset counted in doubles
    L.bytes = (size_t)L.ent * sizeof(double) + (size_t)alpha_job_count(P.mfit) * sizeof(int);
    return L;
}

// alpha/beta/chi2 blocks per thread for mfit <= NCB + 8
template <int NCB>
constexpr int kJobsFor = (alpha_job_count(NCB + 8) + kThreads - 1) / kThreads;

__device__ void alpha_jobs(int mfit, int* jobs) {
    if (threadIdx.x == 0) {
        const int kB = (mfit + 1) & ~1;
        int n = 0;
        for (int j0 = 0; j0 < mfit; j0 += 2) {
            const int kmax = min((j0 + 1) / 4, (mfit - 1) / 4);
            for (int kb = 0; kb <= kmax; kb++) jobs[n++] = j0 | ((4 * kb) << 16);
            jobs[n++] = j0 | (kB << 16);
        }
        jobs[n++] = kB | (kB << 16);
    }
    __syncthreads();
}

// slots of the misc area
enum {
    M_CHISQ = 0,  // chi2 of the evaluation just done
    M_CHK0 = 1,   // its convexity residuals (3)
    M_SAREA = 4,  // its facet-area sum
    M_CL = 5,
    M_CLS = 6,
    M_OMG = 7,
    M_P1 = 8,
    M_P2 = 9,
    M_P3 = 10,
    M_WORK = 11
};

// Order the points [s0, s0 + len) by the direction of the Sun-Earth bisector
// in the body frame (equal-area latitude bands, longitude in alternating
// direction), so that the 32 points of a warp see nearly the same facets and
// a warp skips a facet whenever none of its points sees it.  Only the
// assignment of points to threads changes: every point's sums, and so every
// result, are the same in any order.  perm[i] receives the i-th point.
__device__ void sort_points(const DevProblem& P, int s0, int len, const double* B, double omg,
                            unsigned long long* keys, int* perm) {
    int n2 = 1;
    while (n2 < len) n2 <<= 1;
    const int nw = (len + 31) / 32;
    int nb = (int)(sqrt((double)nw / 1.5) + 0.5);
    if (nb < 1) nb = 1;
    for (int i = threadIdx.x; i < n2; i += kThreads) {
        unsigned long long key = ~0ull;
        if (i < len) {
            const int p = s0 + i;
            const double f = fmod(omg * P.t[p] + P.phi0, 2 * kPiD);
            const double cf = cos(f), sf = sin(f);
            const double bx = P.ex[p] + P.e0x[p], by = P.ey[p] + P.e0y[p], bz = P.ez[p] + P.e0z[p];
            const double w0 = B[0] * bx + B[1] * by + B[2] * bz;
            const double w1 = B[3] * bx + B[4] * by + B[5] * bz;
            const double z = B[6] * bx + B[7] * by + B[8] * bz;
            const double x = cf * w0 + sf * w1, y = cf * w1 - sf * w0;
            const double r = sqrt(x * x + y * y + z * z);
            const double c = r > 0 ? z / r : 1.0;
            int band = (int)((1.0 - c) * 0.5 * nb);
            band = band < 0 ? 0 : (band >= nb ? nb - 1 : band);
            const double ax = fabs(x) + fabs(y);
            double pa = ax > 0 ? (y >= 0 ? 1.0 - x / ax : 3.0 + x / ax) : 0.0;  // pseudo-angle in [0, 4]
            if (band & 1) pa = 4.0 - pa;
            const float kf = (float)(band * 8 + pa + 0.5);
            key = ((unsigned long long)__float_as_uint(kf) << 32) | (unsigned)p;
        }
        keys[i] = key;
    }
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n2; i += kThreads) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = keys[i], b = keys[ixj];
                    if ((a > b) == ((i & k) == 0)) {
                        keys[i] = b;
                        keys[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < len; i += kThreads) perm[i] = (int)(keys[i] & 0xffffffffu);
    __syncthreads();
}

// One FP64 tensor-core step, D = A B + D with A 8x4 (row), B 4x8 (col):
// lane l holds A[l/4][l%4], B[l%4][l/4] and D[l/4][2(l%4)], D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// The GPU's global nanosecond timer (the same clock on every SM).
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Stage facets [f0, f0 + fch) of the facet table (nx, ny, nz, Darea) and of
// dsph into one chunk buffer: asynchronous 16-byte copies, zeros past F.
// Row stride (doubles) of a staged dsph chunk.  The m8n8k4 B fragment has
// lane (g, q) read row q, column g + 8t: with a stride of 4 or 12 mod 16
// doubles the 16 lanes of each half-warp fall on distinct bank pairs (an
// unpadded stride of NCB = 0 or 8 mod 16 puts two lanes on each pair).
template <int NCB>
constexpr int kDs = NCB + 4;

template <int NCB>
__device__ __forceinline__ void stage_chunk_async(const DevProblem& P, int f0, double* fb, double* db) {
    const int fch = P.fch;
    const int nf = min(fch, P.F - f0);
    const double* fs = P.fac + (size_t)f0 * 4;
    const double* ds = P.dsph + (size_t)f0 * NCB;
    for (int i = threadIdx.x; i < fch * 2; i += kThreads) {
        if (i < nf * 2)
            cp_async16(fb + 2 * i, fs + 2 * i);
        else
            reinterpret_cast<double2*>(fb)[i] = make_double2(0.0, 0.0);
    }
    for (int i = threadIdx.x; i < fch * (NCB / 2); i += kThreads) {
        const int ff = i / (NCB / 2), c = 2 * (i - ff * (NCB / 2));
        if (i < nf * (NCB / 2))
            cp_async16(db + ff * kDs<NCB> + c, ds + 2 * i);
        else
            *reinterpret_cast<double2*>(db + ff * kDs<NCB> + c) = make_double2(0.0, 0.0);
    }
    cp_async_commit();
}

// bright.c:54-125 for every data point, fast form, with the shape sums on the
// FP64 tensor cores.  The shape derivatives are a matrix product,
//   dyda[p][k] = sum_f (Darea_f s_pf) (g_f dsph[f][k]) = sum_f A[p][f] dsph[f][k]
// with A[p][f] = Area_f s_pf for the facets p sees (0 otherwise).  A warp owns
// kMT tiles of 8 points; per step of 4 facets lane (g, q) forms A for point g
// and facet q of each tile -- visibility, s, and the brightness, rotation and
// scattering sums over its facets -- and the warp multiplies the 8x4 A tile
// into the 8 x NCB accumulator tiles with m8n8k4 FP64 MMAs (B = dsph rows from
// shared memory).  A tile with no visible (point, facet) pair in the step
// skips its MMAs.  Facet chunks are staged with asynchronous copies, one chunk
// ahead.  Sums split by facet (lane q takes facets q mod 4) are combined at
// the end: the form differs from the reference order by rounding only.
// kX1 (C = NCB - 7, i.e. C = 1 mod 8 as for every even lmax = mmax): the last
// 8-column tile would carry a single coefficient, so coefficient C - 1 is
// summed per lane on the FP64 pipe (one FMA per visible pair) and the MMA
// sequence covers the first NCB - 8 columns.
template <int NCB, bool kX1>
__device__ __forceinline__ void point_loop_fast(const DevProblem& P, double* sm, const Layout& L, const double* B,
                                                const double* D, double* misc, const double* g_f,
                                                const double* area, double* dres, double* work, double* Jt,
                                                double* yt) {
    constexpr int NT = kX1 ? NCB / 8 - 1 : NCB / 8;  // MMA accumulator tiles per 8 points
    static_assert(NT > 0, "kX1 needs NCB >= 16");
    constexpr int kMT = 1;                       // point tiles per warp
    constexpr int kPts = (kThreads / 32) * 8 * kMT;  // points per pass
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int F = P.F, C = P.C, npad = P.npad;
    const int fch = P.fch, sseg = P.sortseg;
    // chunk buffer b at work + b * cstride: fch facet rows, then fch dsph rows.
    // Buffers are selected by arithmetic on `work`, not from an array of
    // pointers: a dynamically indexed pointer array would live in local memory
    // and every load through its elements become a generic load.
    const int cstride = fch * (4 + kDs<NCB>);
    int* perm = (int*)(sm + L.perm);
    const double cl = misc[M_CL], cls = misc[M_CLS];
    const unsigned full = 0xffffffffu;
    const int nch = (F + fch - 1) / fch;
    constexpr int kSumJobs = (4 + 3 * NCB + kThreads - 1) / kThreads;
    double fsum[kSumJobs];
#pragma unroll
    for (int u = 0; u < kSumJobs; u++) fsum[u] = 0;
    for (int s0 = 0; s0 < P.n_points; s0 += sseg) {
        const int seg = min(sseg, P.n_points - s0);
        __syncthreads();
        sort_points(P, s0, seg, B, misc[M_OMG], (unsigned long long*)work, perm);
        for (int base = 0; base < seg; base += kPts) {
            int p[kMT];
            bool act[kMT];
            double e[kMT][3], e0[kMT][3];
#pragma unroll
            for (int i = 0; i < kMT; i++) {
                const int ps = base + warp * 8 * kMT + i * 8 + g;
                act[i] = ps < seg;
                p[i] = act[i] ? perm[ps] : 0;
#pragma unroll
                for (int c = 0; c < 3; c++) e[i][c] = e0[i][c] = 0;
                if (act[i]) {
                    PointGeom G;
                    point_geometry(P, p[i], B, D, misc[M_OMG], misc[M_P1], misc[M_P2], misc[M_P3], G);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        e[i][c] = G.e[c];
                        e0[i][c] = G.e0[c];
                    }
                }
            }
            double acc[kMT][NT][2];
            double br[kMT], T[kMT][3], S[kMT][3], s_cl[kMT], s_cls[kMT], x1[kMT];
#pragma unroll
            for (int i = 0; i < kMT; i++) {
#pragma unroll
                for (int t = 0; t < NT; t++) acc[i][t][0] = acc[i][t][1] = 0;
                br[i] = s_cl[i] = s_cls[i] = x1[i] = 0;
#pragma unroll
                for (int c = 0; c < 3; c++) T[i][c] = S[i][c] = 0;
            }
            __syncthreads();
            stage_chunk_async<NCB>(P, 0, work, work + fch * 4);
            cp_async_wait_all();
            __syncthreads();
            for (int ch = 0; ch < nch; ch++) {
                const int f0 = ch * fch;
                double* nb = work + ((ch + 1) & 1) * cstride;
                if (ch + 1 < nch) stage_chunk_async<NCB>(P, f0 + fch, nb, nb + fch * 4);
                const double* fb = work + (ch & 1) * cstride;
                const double* db = fb + fch * 4;
                const int nf = min(fch, F - f0);
                if (s0 == 0 && base == 0) {
                    // the facet sums (convexity residuals and derivatives, facet-area
                    // sum) from the staged chunk, facets in order, one thread per sum
#pragma unroll
                    for (int u = 0; u < kSumJobs; u++) {
                        const int job = tid + u * kThreads;
                        if (job >= 4 + 3 * C) continue;
                        double sacc = fsum[u];
                        if (job < 4) {
                            for (int ff = 0; ff < nf; ff++)
                                sacc = sacc + (job < 3 ? area[f0 + ff] * fb[ff * 4 + job] : area[f0 + ff]);
                        } else {
                            const int nc = (job - 4) / C, jj = (job - 4) - nc * C;
                            for (int ff = 0; ff < nf; ff++) {
                                const double dg = g_f[f0 + ff] * db[ff * kDs<NCB> + jj];
                                sacc += fb[ff * 4 + 3] * dg * fb[ff * 4 + nc];
                            }
                        }
                        fsum[u] = sacc;
                    }
                }
                // Facets past F (zero rows in the staged chunk, zero area) and
                // inactive lanes (e = e0 = 0) have mu = mu0 = 0: not visible.
                for (int j = 0; j < nf; j += 4) {
                    const int ff = j + q;
                    const double nx = fb[ff * 4 + 0], ny = fb[ff * 4 + 1], nz = fb[ff * 4 + 2];
                    const double ar = area[f0 + ff];
                    double av[kMT];
                    bool any[kMT];
#pragma unroll
                    for (int i = 0; i < kMT; i++) {
                        const double mu = e[i][0] * nx + e[i][1] * ny + e[i][2] * nz;
                        const double mu0 = e0[i][0] * nx + e0[i][1] * ny + e0[i][2] * nz;
                        const bool vis = (mu > kTinyD) && (mu0 > kTinyD);
                        any[i] = __any_sync(full, vis);
                        av[i] = 0;
                        if (vis) {
                            const double r = 1.0 / (mu + mu0);
                            const double sv = mu * mu0 * fma(cls, r, cl);
                            av[i] = ar * sv;
                            br[i] += av[i];
                            const double q0 = mu0 * r, q1 = mu * r;
                            const double w = ar * fma(cls * q0, q0, cl * mu0);
                            const double w0 = ar * fma(cls * q1, q1, cl * mu);
                            T[i][0] = fma(w, nx, T[i][0]);
                            T[i][1] = fma(w, ny, T[i][1]);
                            T[i][2] = fma(w, nz, T[i][2]);
                            S[i][0] = fma(w0, nx, S[i][0]);
                            S[i][1] = fma(w0, ny, S[i][1]);
                            S[i][2] = fma(w0, nz, S[i][2]);
                            const double mm = mu * mu0 * ar;
                            s_cl[i] += mm;
                            s_cls[i] = fma(mm, r, s_cls[i]);
                            if (kX1) x1[i] = fma(av[i], db[ff * kDs<NCB> + 8 * NT], x1[i]);
                        }
                    }
                    bool some = false;
#pragma unroll
                    for (int i = 0; i < kMT; i++) some = some || any[i];
                    if (!some) continue;
                    const double* brow = db + ff * kDs<NCB> + g;
#pragma unroll
                    for (int t = 0; t < NT; t++) {
                        const double bv = brow[t * 8];
#pragma unroll
                        for (int i = 0; i < kMT; i++)
                            if (any[i]) dmma_8x8x4(acc[i][t][0], acc[i][t][1], av[i], bv);
                    }
                }
                cp_async_wait_all();
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < kMT; i++) {
                // the four lanes of a point hold the sums over facets q mod 4
#pragma unroll
                for (int o = 1; o <= 2; o <<= 1) {
                    br[i] += __shfl_xor_sync(full, br[i], o);
                    s_cl[i] += __shfl_xor_sync(full, s_cl[i], o);
                    s_cls[i] += __shfl_xor_sync(full, s_cls[i], o);
                    if (kX1) x1[i] += __shfl_xor_sync(full, x1[i], o);
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        T[i][c] += __shfl_xor_sync(full, T[i][c], o);
                        S[i][c] += __shfl_xor_sync(full, S[i][c], o);
                    }
                }
                if (!act[i]) continue;
                PointGeom G;
                point_geometry(P, p[i], B, D, misc[M_OMG], misc[M_P1], misc[M_P2], misc[M_P3], G);
                const double sc = G.scale;
#pragma unroll
                for (int t = 0; t < NT; t++)
#pragma unroll
                    for (int jj = 0; jj < 2; jj++) {
                        const int k = t * 8 + 2 * q + jj;
                        if (k < C) Jt[(size_t)k * npad + p[i]] = sc * acc[i][t][jj];
                    }
                if (kX1 && q == 0) Jt[(size_t)(8 * NT) * npad + p[i]] = sc * x1[i];
                if (q == 0) {
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        double v = 0;
#pragma unroll
                        for (int c = 0; c < 3; c++) v = fma(T[i][c], G.de[c][k], fma(S[i][c], G.de0[c][k], v));
                        Jt[(size_t)(C + k) * npad + p[i]] = sc * v;
                    }
                    Jt[(size_t)(C + 3) * npad + p[i]] = br[i] * G.dphp[0];
                    Jt[(size_t)(C + 4) * npad + p[i]] = br[i] * G.dphp[1];
                    Jt[(size_t)(C + 5) * npad + p[i]] = br[i] * G.dphp[2];
                    Jt[(size_t)(C + 6) * npad + p[i]] = sc * s_cl[i] * cl;
                    Jt[(size_t)(C + 7) * npad + p[i]] = sc * s_cls[i];
                    yt[p[i]] = br[i] * sc;
                }
            }
        }
    }
#pragma unroll
    for (int u = 0; u < kSumJobs; u++) {
        const int job = tid + u * kThreads;
        if (job < 3)
            misc[M_CHK0 + job] = fsum[u];
        else if (job == 3)
            misc[M_SAREA] = fsum[u];
        else if (job < 4 + 3 * C)
            dres[job - 4] = fsum[u];
    }
}

// alpha = J^T W J, beta = J^T W dy, chi2 (mrqcof.c:106-147) on the FP64
// tensor cores (fast form).  Tiles of kRt rows, two buffers: Js[r][k] =
// J[r][l_k] (k < mfit), Js[r][kB] = dy, zero elsewhere, and the row weight
// w[r] = sig2i wght; the next tile's J values arrive by asynchronous copies
// and its dy and w through registers while the current tile is multiplied.
// With A = (Js w)^T and B = Js, entry (j, k) is alpha (k <= j < mfit), beta
// (k = kB) or chi2 (j = k = kB).  Output tiles of 8 x 8 entries: the lower
// triangle (kt <= jt) and the tiles above it in the beta column; a warp
// accumulates its tiles over all rows with m8n8k4 MMAs.
template <int NCB>
__device__ __forceinline__ void alpha_tensor(const DevProblem& P, const double* Jt, const double* yt, double* work,
                                             double* alpha_out, double* beta_out, double* misc) {
    constexpr int kBmax = (NCB + 8 + 1) & ~1;
    constexpr int Tmax = (kBmax + 2 + 7) / 8;
    constexpr int kTiles = (Tmax * (Tmax + 1) / 2 + Tmax + kThreads / 32 - 1) / (kThreads / 32);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, q = lane & 3;
    const int mfit = P.mfit, npad = P.npad, nrows = P.n_rows;
    const int kB = (mfit + 1) & ~1;
    const int T = (kB + 2 + 7) / 8, st = T * 8 + 4, ktB = kB / 8;
    const int ntri = T * (T + 1) / 2, ntile = ntri + ktB;
    const int rt = P.rt;
    // buffer b: Js at work + b * bstride (rt rows of st), then the rt weights
    // (arithmetic on `work`, not a pointer array: see point_loop_fast)
    const int bstride = rt * (st + 1);
    int tj[kTiles], tk[kTiles];
    double acc[kTiles][2];
#pragma unroll
    for (int i = 0; i < kTiles; i++) {
        const int t = warp + i * (kThreads / 32);
        int jt = 0, kt = 0;
        if (t < ntri) {
            while ((jt + 1) * (jt + 2) / 2 <= t) jt++;
            kt = t - jt * (jt + 1) / 2;
        } else {
            jt = t - ntri;
            kt = ktB;
        }
        tj[i] = t < ntile ? jt * 8 : -1;
        tk[i] = kt * 8;
        acc[i][0] = acc[i][1] = 0;
    }
    // warp w copies parameter columns w, w + 8, ...; lane r rows r, r + 32, ...
    auto issue = [&](int r0, int b) {
        const int nr = min(rt, nrows - r0);
        for (int j = warp; j < mfit; j += kThreads / 32) {
            const double* src = Jt + (size_t)P.free_idx[j] * npad + r0;
            double* dst = work + b * bstride + j;
            for (int r = lane; r < nr; r += 32) cp_async8(dst + r * st, src + r);
        }
        cp_async_commit();
    };
    __syncthreads();
    for (int i = tid; i < 2 * rt * (st + 1); i += kThreads) work[i] = 0.0;
    __syncthreads();
    const int ntl = (nrows + rt - 1) / rt;
    issue(0, 0);
    if (tid < rt) {
        const double dy = tid < nrows ? P.yobs[tid] - yt[tid] : 0.0;
        work[tid * st + kB] = dy;
        work[rt * st + tid] = tid < nrows ? P.sig2i[tid] * P.wght[tid] : 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    for (int t = 0; t < ntl; t++) {
        const int b = t & 1, r0 = t * rt;
        const int nr4 = (min(rt, nrows - r0) + 3) & ~3;
        double ndy = 0.0, nw = 0.0;
        if (t + 1 < ntl) {
            const int r1 = r0 + rt;
            issue(r1, b ^ 1);
            if (tid < rt && r1 + tid < nrows) {
                ndy = P.yobs[r1 + tid] - yt[r1 + tid];
                nw = P.sig2i[r1 + tid] * P.wght[r1 + tid];
            }
        }
        const double* jb = work + b * bstride;
        const double* wb = jb + rt * st;
        for (int rr = 0; rr < nr4; rr += 4) {
            const double* row = jb + (rr + q) * st + g;
            const double w = wb[rr + q];
#pragma unroll
            for (int i = 0; i < kTiles; i++)
                if (tj[i] >= 0) dmma_8x8x4(acc[i][0], acc[i][1], row[tj[i]] * w, row[tk[i]]);
        }
        if (t + 1 < ntl && tid < rt) {
            double* jn = work + (b ^ 1) * bstride;
            jn[tid * st + kB] = ndy;
            jn[rt * st + tid] = nw;  // zero past the last row
        }
        cp_async_wait_all();
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < kTiles; i++) {
        if (tj[i] < 0) continue;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int j = tj[i] + g, k = tk[i] + 2 * q + e;
            const double v = acc[i][e];
            if (j < mfit && k < mfit) {
                if (k <= j) {
                    alpha_out[j * mfit + k] = v;
                    alpha_out[k * mfit + j] = v;
                }
            } else if (j < mfit && k == kB) {
                beta_out[j] = v;
            } else if (j == kB && k == kB) {
                misc[M_CHISQ] = v;
            }
        }
    }
}

// One model evaluation, the reference's mrqcof (mrqcof.c:16-148) at
// parameters a (shared memory, at offset a_off).  Writes the symmetrised
// alpha and beta into alpha_out / beta_out (shared memory, offsets alpha_off
// and beta_off) and chi2, the convexity residuals (= the driver's chck,
// period_search_BOINC.cpp:876-880) and the facet-area sum into misc.  J^T (ma
// columns of npad rows) and y go to the CTA's scratch.  All threads enter and
// leave together.  The shared-memory operands are passed as offsets from the
// dynamic shared-memory base declared here, not as pointers: a pointer
// argument of this out-of-line function would be a generic address, and every
// access through it a generic load or store instead of a shared-memory one.
// blmatrix (mrqcof.c:34) and the per-evaluation scalars of bright.c:26-33.
__device__ __forceinline__ void eval_scalars(const double* a, int C, double* B, double* D, double* misc) {
    if (threadIdx.x == 0) {
        blmatrix(a[C], a[C + 1], B, D);
        misc[M_CL] = exp(a[C + 6]);
        misc[M_CLS] = a[C + 7];
        misc[M_OMG] = a[C + 2];
        misc[M_P1] = a[C + 3];
        misc[M_P2] = a[C + 4];
        misc[M_P3] = a[C + 5];
    }
}

// curv.c:15-37: g = exp(sum over (m, l) of Pleg * (c*Fc + s*Fs)), thread per
// facet; area = Darea g, zero for the 128 slots past F.
__device__ __forceinline__ void curv_phase(const DevProblem& P, const double* a, double* g, double* area,
                                           bool pad = true) {
    const int F = P.F;
    for (int f = threadIdx.x; f < F; f += kThreads) {
        const double* pl = P.cpl + (size_t)f * P.nq;
        const double* fc = P.cfc + (size_t)f * (P.mmax + 1);
        const double* fs = P.cfs + (size_t)f * (P.mmax + 1);
        double gi = 0;
        int n = 0, q = 0;
        for (int m = 0; m <= P.mmax; m++) {
            const double fcm = fc[m], fsm = fs[m];
            for (int l = m; l <= P.lmax; l++) {
                double fsum = a[n] * fcm;
                n++;
                if (m != 0) {
                    fsum = fsum + a[n] * fsm;
                    n++;
                }
                gi = gi + pl[q] * fsum;
                q++;
            }
        }
        gi = exp(gi);
        g[f] = gi;
        area[f] = P.fac[(size_t)f * 4 + 3] * gi;
    }
    if (pad)
        for (int f = F + threadIdx.x; f < F + 128; f += kThreads) area[f] = 0.0;
}

// chi2 over all rows (mrqcof.c:119-135) from the normalised model yt.  The
// reference-order form sums the rows in order on one thread, with the
// operations of its alpha/beta/chi2 phase (whose chi2 entry is the same
// sum), so both give the same bits; the fast form sums on one warp in a
// fixed order.  The result lands in misc[M_CHISQ].
template <bool kFast>
__device__ __forceinline__ void chi2_rows(const DevProblem& P, const double* yt, double* misc) {
    if constexpr (!kFast) {
        if (threadIdx.x == 0) {
            double acc = 0;
            for (int r = 0; r < P.n_rows; r++) {
                const double dy = P.yobs[r] - yt[r];
                acc = acc + dy * dy * P.sig2i[r] * P.wght[r];
            }
            misc[M_CHISQ] = acc;
        }
    } else {
        if (threadIdx.x < 32) {
            double acc = 0;
            for (int r = threadIdx.x; r < P.n_rows; r += 32) {
                const double dy = P.yobs[r] - yt[r];
                acc = fma(dy * P.sig2i[r] * P.wght[r], dy, acc);
            }
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (threadIdx.x == 0) misc[M_CHISQ] = acc;
        }
    }
}

// The model alone at parameters a: what the LM step's accept/reject test and
// the stop rule read from mrqcof at a trial point -- chi2, the convexity
// residuals chck (conv.c:22-27) and the facet-area sum -- without the
// Jacobian or alpha/beta.  curv, the brightness of every point
// (bright.c:54-76, 106-125 without the derivative terms), the convexity
// rows, the relative-lightcurve normalisation of the model (mrqcof.c:53-58,
// 92-104) and chi2, with the operations and sum orders of evaluate(), so
// that in the reference-order form every value is bit-identical to the one
// evaluate() gives at the same point.  The model goes to yt; Jt is not
// touched.  Thread per data point, facet normals staged in chunks of kMf.
// Buffers (shared memory): g, area [F] (area is not padded past F here);
// misc and B/D (blmatrix) as in evaluate(); work >= max(sortseg, 4 kMf,
// kThreads) doubles, 16-byte aligned; perm sortseg ints.  Used by the FP64
// fit kernels (evaluate_model) and the mixed-precision one.
template <bool kFast>
__device__ void model_pass(const DevProblem& P, const double* a, double* g, double* area, double* misc, double* B,
                           double* D, double* work, int* perm, double* yt) {
    const int tid = threadIdx.x;
    const int F = P.F, C = P.C;
    eval_scalars(a, C, B, D, misc);
    curv_phase(P, a, g, area, false);
    __syncthreads();
    // chck and the facet-area sum, facets in order (as evaluate() and the
    // fast point loop form them); four threads, loads ahead of the sums
    if (tid < 4) {
        double s = 0;
        if (tid < 3) {
#pragma unroll 8
            for (int f = 0; f < F; f++) s = s + area[f] * __ldg(P.fac + (size_t)f * 4 + tid);
            misc[M_CHK0 + tid] = s;
        } else {
#pragma unroll 8
            for (int f = 0; f < F; f++) s = s + area[f];
            misc[M_SAREA] = s;
        }
    }
    const double cl = misc[M_CL], cls = misc[M_CLS];
    // points in segments sorted by viewing direction (as in evaluate()), so
    // that the points of a warp see nearly the same facets
    for (int s0 = 0; s0 < P.n_points; s0 += P.sortseg) {
    const int seg = min(P.sortseg, P.n_points - s0);
    __syncthreads();
    sort_points(P, s0, seg, B, misc[M_OMG], (unsigned long long*)work, perm);
    // kMp points per thread at most (slot j of thread t: point base + j kThreads
    // + t, so each slot's warp holds consecutive sorted points): independent
    // chains per facet and one load of each facet for all of them
    const int k = min(kMp, (seg + kThreads - 1) / kThreads);
    for (int base = 0; base < seg; base += k * kThreads) {
        int pj[kMp];
        bool aj[kMp];
        double ej[kMp][3], fj[kMp][3], sc[kMp], br[kMp];
#pragma unroll
        for (int j = 0; j < kMp; j++) {
            const int i = base + j * kThreads + tid;
            aj[j] = j < k && i < seg;
            pj[j] = aj[j] ? perm[i] : 0;
            br[j] = 0;
            sc[j] = 0;
#pragma unroll
            for (int c = 0; c < 3; c++) ej[j][c] = fj[j][c] = 0;
            if (aj[j]) {
                PointGeom G;
                point_geometry(P, pj[j], B, D, misc[M_OMG], misc[M_P1], misc[M_P2], misc[M_P3], G);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    ej[j][c] = G.e[c];
                    fj[j][c] = G.e0[c];
                }
                sc[j] = G.scale;
            }
        }
        double4* nrm = reinterpret_cast<double4*>(work);  // [kMf] nx, ny, nz, Area
        for (int c0 = 0; c0 < F; c0 += kMf) {
            const int nf = min(kMf, F - c0);
            __syncthreads();
            for (int ff = tid; ff < nf; ff += kThreads) {
                const double* fa = P.fac + (size_t)(c0 + ff) * 4;
                nrm[ff] = make_double4(fa[0], fa[1], fa[2], area[c0 + ff]);
            }
            __syncthreads();
#pragma unroll 2
            for (int ff = 0; ff < nf; ff++) {
                const double4 n = nrm[ff];
#pragma unroll
                for (int j = 0; j < kMp; j++) {
                    if (!aj[j]) continue;
                    const double mu = ej[j][0] * n.x + ej[j][1] * n.y + ej[j][2] * n.z;
                    const double mu0 = fj[j][0] * n.x + fj[j][1] * n.y + fj[j][2] * n.z;
                    if ((mu > kTinyD) && (mu0 > kTinyD)) {
                        if constexpr (kFast) {
                            const double r = rcp_newton(mu + mu0);
                            br[j] = fma(n.w, mu * mu0 * fma(cls, r, cl), br[j]);
                        } else {
                            const double dnom = mu + mu0;
                            const double s = mu * mu0 * (cl + cls / dnom);
                            br[j] = br[j] + n.w * s;
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kMp; j++)
            if (aj[j]) yt[pj[j]] = br[j] * sc[j];
    }
    }
    __syncthreads();
    if (tid < 3) yt[P.n_points + tid] = misc[M_CHK0 + tid];
    // relative-lightcurve normalisation of the model, mrqcof.c:53-58, 92-104
    for (int lc0 = 0; lc0 < P.n_lc; lc0 += kThreads) {
        __syncthreads();
        const int lc = lc0 + tid;
        if (lc < P.n_lc && P.lc_rel[lc]) {
            double s = 0;
            for (int r = P.lc_start[lc]; r < P.lc_start[lc + 1]; r++) s = s + yt[r];
            work[tid] = s;
        }
        __syncthreads();
        for (int k = 0; k < kThreads && lc0 + k < P.n_lc; k++) {
            const int l2 = lc0 + k;
            if (!P.lc_rel[l2]) continue;
            const double ave = work[k];
            const double lpts = (double)P.lc_npts[l2];
            for (int r = P.lc_start[l2] + tid; r < P.lc_start[l2 + 1]; r += kThreads) {
                const double coef = P.sig[r] * lpts / ave;
                yt[r] = coef * yt[r];
            }
        }
    }
    __syncthreads();
    chi2_rows<kFast>(P, yt, misc);
    __syncthreads();
}

// The model rows go to the work area past the sort keys and the staged
// normals when they fit there (nothing reads them after the pass but its own
// normalisation and chi2), else to yt in global memory.
template <int NCB, bool kFast>
__device__ __noinline__ void evaluate_model(const DevProblem* __restrict__ Pp, int a_off, double* yt) {
    extern __shared__ __align__(16) double sm[];
    const DevProblem& P = *Pp;
    const Layout L = make_layout(P);
    const int yoff = P.sortseg > 4 * kMf ? P.sortseg : 4 * kMf;
    double* ym = yoff + P.npad <= L.wlen ? sm + L.work + yoff : yt;
    model_pass<kFast>(P, sm + a_off, sm + L.g, sm + L.area, sm + L.misc, sm + L.blm, sm + L.blm + 9, sm + L.work,
                      (int*)(sm + L.perm), ym);
}

// bright.c:54-125 for every data point in the reference's operation order
// (PS_FORM_FP64), in segments of points sorted by viewing direction.  Two
// threads per point: thread t works on point slot t mod 128 of a pass of 128
// points, and its half h = t / 128 (warps 0-3, warps 4-7) keeps the shape
// sums of coefficients [h NCB/2, (h + 1) NCB/2) and half of the other
// per-point sums (h = 0: the brightness and the rotation derivatives 0 and 1;
// h = 1: rotation derivative 2 and the two scattering sums).  Every sum runs
// over the facets in order with the reference's operations, each in one
// thread, so the results are the bits of one thread per point; both halves
// form the per-pair terms (visibility, s, the derivative factors).  Each half
// runs its own instantiation of the pass (H), so that a thread holds only its
// half's state and its accumulators fit in 128 registers (two fits per SM);
// both execute the same block barriers, warp by warp.
template <int NCB, int H>
__device__ __forceinline__ void ref_pass(const DevProblem& P, const double* B, const double* D, double* misc,
                                         const double* g, const double* area, double* s_fac, double* s_dg,
                                         double* sdv, int pl, bool act, int p, double* Jt, double* yt) {
    constexpr int KH = NCB / 2;
    constexpr int kPts = kThreads / 2;
    const int tid = threadIdx.x;
    const int F = P.F, C = P.C, npad = P.npad;
    const double cl = misc[M_CL], cls = misc[M_CLS];
    constexpr int c0 = H == 0 ? 0 : 2;  // the rotation derivative both halves keep
    // this point's derivative vectors in shared memory ([vector][slot]: the
    // loads of a warp are consecutive): H = 0 columns 0 and 1 of de, de0
    // (12 doubles), H = 1 column 2 (6 doubles, after the 12 x 128 of H = 0)
    double* dv = sdv + (H == 0 ? 0 : 12 * kPts) + pl;
    double e[3] = {0, 0, 0}, e0[3] = {0, 0, 0};
    if (act) {
        PointGeom G;
        point_geometry(P, p, B, D, misc[M_OMG], misc[M_P1], misc[M_P2], misc[M_P3], G);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            e[i] = G.e[i];
            e0[i] = G.e0[i];
            dv[(0 + i) * kPts] = G.de[i][c0];
            dv[(3 + i) * kPts] = G.de0[i][c0];
            if constexpr (H == 0) {
                dv[(6 + i) * kPts] = G.de[i][1];
                dv[(9 + i) * kPts] = G.de0[i][1];
            }
        }
    }
    double acc[KH];
#pragma unroll
    for (int k = 0; k < KH; k++) acc[k] = 0;
    double a0 = 0, a1 = 0, a2 = 0;  // H = 0: br, rot0, rot1; H = 1: s_cl, rot2, s_cls
    for (int f0 = 0; f0 < F; f0 += kFch) {
        const int nf = min(kFch, F - f0);
        __syncthreads();
        for (int idx = tid; idx < nf * NCB; idx += kThreads) {
            const int ff = idx / NCB, k = idx - ff * NCB;
            s_dg[idx] = g[f0 + ff] * P.dsph[(size_t)(f0 + ff) * NCB + k];
        }
        for (int ff = tid; ff < nf; ff += kThreads) {
            const double* fa = P.fac + (size_t)(f0 + ff) * 4;
            s_fac[ff * 5 + 0] = fa[0];
            s_fac[ff * 5 + 1] = fa[1];
            s_fac[ff * 5 + 2] = fa[2];
            s_fac[ff * 5 + 3] = area[f0 + ff];
            s_fac[ff * 5 + 4] = fa[3];
        }
        __syncthreads();
        if (act) {
#pragma unroll 2  // two facets in flight (1.9 % on c2; same operations per sum)
            for (int ff = 0; ff < nf; ff++) {
                const double nx = s_fac[ff * 5 + 0], ny = s_fac[ff * 5 + 1], nz = s_fac[ff * 5 + 2];
                const double mu = e[0] * nx + e[1] * ny + e[2] * nz;
                const double mu0 = e0[0] * nx + e0[1] * ny + e0[2] * nz;
                if ((mu > kTinyD) && (mu0 > kTinyD)) {
                    const double ar = s_fac[ff * 5 + 3], darea = s_fac[ff * 5 + 4];
                    const double dnom = mu + mu0;
                    const double s = mu * mu0 * (cl + cls / dnom);
                    const double q0 = mu0 / dnom, q1 = mu / dnom;
                    const double dsmu = cls * (q0 * q0) + cl * mu0;
                    const double dsmu0 = cls * (q1 * q1) + cl * mu;
                    const double dbr = darea * s;
                    const double* dg = s_dg + ff * NCB + H * KH;
#pragma unroll
                    for (int k = 0; k < KH; k++) acc[k] = acc[k] + dbr * dg[k];
                    {
                        const double sum = nx * dv[0] + ny * dv[kPts] + nz * dv[2 * kPts];
                        const double sum0 = nx * dv[3 * kPts] + ny * dv[4 * kPts] + nz * dv[5 * kPts];
                        a1 = a1 + ar * (dsmu * sum + dsmu0 * sum0);
                    }
                    if constexpr (H == 0) {
                        a0 = a0 + ar * s;
                        const double sum = nx * dv[6 * kPts] + ny * dv[7 * kPts] + nz * dv[8 * kPts];
                        const double sum0 = nx * dv[9 * kPts] + ny * dv[10 * kPts] + nz * dv[11 * kPts];
                        a2 = a2 + ar * (dsmu * sum + dsmu0 * sum0);
                    } else {
                        a0 = a0 + mu * mu0 * ar;
                        a2 = a2 + ar * mu * mu0 / (mu + mu0);
                    }
                }
            }
        }
    }
    if (act) {
        PointGeom G;  // recomputed (the same values): no registers across the facet loop
        point_geometry(P, p, B, D, misc[M_OMG], misc[M_P1], misc[M_P2], misc[M_P3], G);
        const double sc = G.scale;
#pragma unroll
        for (int k = 0; k < KH; k++)
            if (H * KH + k < C) Jt[(size_t)(H * KH + k) * npad + p] = sc * acc[k];
        if constexpr (H == 0) {
            Jt[(size_t)(C + 0) * npad + p] = sc * a1;
            Jt[(size_t)(C + 1) * npad + p] = sc * a2;
            Jt[(size_t)(C + 3) * npad + p] = a0 * G.dphp[0];
            Jt[(size_t)(C + 4) * npad + p] = a0 * G.dphp[1];
            Jt[(size_t)(C + 5) * npad + p] = a0 * G.dphp[2];
            yt[p] = a0 * sc;
        } else {
            Jt[(size_t)(C + 2) * npad + p] = sc * a1;
            Jt[(size_t)(C + 6) * npad + p] = sc * a0 * cl;
            Jt[(size_t)(C + 7) * npad + p] = sc * a2;
        }
    }
}

template <int NCB>
__device__ __forceinline__ void point_loop_ref(const DevProblem& P, double* sm, const Layout& L, const double* B,
                                               const double* D, double* misc, const double* g, const double* area,
                                               double* work, double* Jt, double* yt) {
    constexpr int kPts = kThreads / 2;
    const int tid = threadIdx.x, h = tid / kPts, pl = tid - h * kPts;
    double* s_fac = work;
    double* s_dg = work + kFch * 5;
    double* sdv = work + ((kFch * 5 + kFch * NCB + 1) & ~1);
    int* perm = (int*)(sm + L.perm);
    for (int s0 = 0; s0 < P.n_points; s0 += P.sortseg) {
        const int seg = min(P.sortseg, P.n_points - s0);
        __syncthreads();
        sort_points(P, s0, seg, B, misc[M_OMG], (unsigned long long*)work, perm);
        for (int base = 0; base < seg; base += kPts) {
            const bool act = base + pl < seg;
            const int p = act ? perm[base + pl] : 0;
            if (h == 0)
                ref_pass<NCB, 0>(P, B, D, misc, g, area, s_fac, s_dg, sdv, pl, act, p, Jt, yt);
            else
                ref_pass<NCB, 1>(P, B, D, misc, g, area, s_fac, s_dg, sdv, pl, act, p, Jt, yt);
        }
    }
}

template <int NCB, bool kFast>
__device__ __noinline__ void evaluate(const DevProblem* __restrict__ Pp, int a_off, int alpha_off, int beta_off,
                                      double* Jt, double* yt) {
    extern __shared__ __align__(16) double sm[];
    const double* a = sm + a_off;
    double* alpha_out = sm + alpha_off;
    double* beta_out = sm + beta_off;
    const DevProblem& P = *Pp;
    const Layout L = make_layout(P);
    const int tid = threadIdx.x;
    const int F = P.F, C = P.C, ma = P.ma, npad = P.npad, mfit = P.mfit;
    double* g = sm + L.g;
    double* area = sm + L.area;
    double* misc = sm + L.misc;
    double* B = sm + L.blm;
    double* D = sm + L.blm + 9;
    double* dres = sm + L.dres;
    double* work = sm + L.work;

    eval_scalars(a, C, B, D, misc);
    curv_phase(P, a, g, area);
    __syncthreads();
    // Sequential facet sums: chck / conv residuals (conv.c:22-27), the
    // facet-area sum (period_search_BOINC.cpp:900-902) and the conv-row shape
    // derivatives, one thread per sum, facets in order (the fast form forms
    // them from the facet chunks its point loop stages).
    if constexpr (!kFast)
    for (int job = tid; job < 4 + 3 * C; job += kThreads) {
        double s = 0;
        if (job < 3) {
#pragma unroll 8
            for (int f = 0; f < F; f++) s = s + area[f] * P.fac[(size_t)f * 4 + job];
            misc[M_CHK0 + job] = s;
        } else if (job == 3) {
#pragma unroll 8
            for (int f = 0; f < F; f++) s = s + area[f];
            misc[M_SAREA] = s;
        } else {
            const int nc = (job - 4) / C, j = (job - 4) - nc * C;
#pragma unroll 8
            for (int f = 0; f < F; f++) {
                const double dg = g[f] * P.dsph[(size_t)f * NCB + j];
                s += P.fac[(size_t)f * 4 + 3] * dg * P.fac[(size_t)f * 4 + nc];
            }
            dres[nc * C + j] = s;
        }
    }
    if constexpr (kFast) {
        if constexpr (NCB >= 16) {
            if (C == NCB - 7)
                point_loop_fast<NCB, true>(P, sm, L, B, D, misc, g, area, dres, work, Jt, yt);
            else
                point_loop_fast<NCB, false>(P, sm, L, B, D, misc, g, area, dres, work, Jt, yt);
        } else {
            point_loop_fast<NCB, false>(P, sm, L, B, D, misc, g, area, dres, work, Jt, yt);
        }
    } else {
        point_loop_ref<NCB>(P, sm, L, B, D, misc, g, area, work, Jt, yt);
    }
    __syncthreads();
    // convexity rows (conv.c:12-29): y = residual, J = dres for the shape
    // coefficients and 0 elsewhere
    for (int job = tid; job < 3 * ma; job += kThreads) {
        const int nc = job / ma, l = job - nc * ma;
        const int row = P.n_points + nc;
        Jt[(size_t)l * npad + row] = l < C ? dres[nc * C + l] : 0.0;
        if (l == 0) yt[row] = misc[M_CHK0 + nc];
    }
    __syncthreads();
    // relative-lightcurve normalisation (mrqcof.c:53-58, 75-83, 92-104)
    double* dave = sm + L.dave;
    for (int lc = 0; lc < P.n_lc; lc++) {
        if (!P.lc_rel[lc]) continue;
        const int r0 = P.lc_start[lc], r1 = P.lc_start[lc + 1];
        for (int job = tid; job <= ma; job += kThreads) {
            const double* col = job < ma ? Jt + (size_t)job * npad : yt;
            double s = 0;
            for (int r = r0; r < r1; r++) s = s + col[r];
            dave[job] = s;
        }
        __syncthreads();
        const double ave = dave[ma];
        const double lpts = (double)P.lc_npts[lc];
        for (int r = r0 + tid; r < r1; r += kThreads) {
            const double coef = P.sig[r] * lpts / ave;
            const double y = yt[r];
            for (int l = 0; l < ma; l++) {
                double* d = Jt + (size_t)l * npad + r;
                *d = coef * (*d - y * dave[l] / ave);
            }
            yt[r] = coef * y;
            Jt[r] = 0;
        }
        __syncthreads();
    }
    if constexpr (kFast) {
        alpha_tensor<NCB>(P, Jt, yt, work, alpha_out, beta_out, misc);
        // chi2 as the model-only pass sums it, so that the LM test compares
        // values of one rounding
        __syncthreads();
        chi2_rows<true>(P, yt, misc);
    } else {
        // alpha = J^T W J, beta = J^T W dy, chi2 (mrqcof.c:106-147), every entry
        // summing the rows in order.  Tile of kRt rows: Ws[r][j] = (J[r][l_j]
        // sig2i) wght (j < mfit), Ws[r][jC] = dy dy sig2i wght; Js[r][k] =
        // J[r][l_k] (k < mfit), Js[r][kB] = dy, Js[r][kB+1] = 1; other columns 0.
        // Each job is a 2 x 4 block of entries (Ws columns j0, j0+1 against Js
        // columns k0..k0+3), held in registers across the tiles.
        const int kB = (mfit + 1) & ~1, jC = kB;
        const int wst = jC + 2, jst = kB + 4;
        double* Ws = work;
        double* Js = work + kRt * wst;
        const int* jobs = (const int*)(sm + L.ent);
        const int njob = alpha_job_count(mfit);
        constexpr int kJobs = kJobsFor<NCB>;
        double acc2[kJobs][2][4];
    #pragma unroll
        for (int q = 0; q < kJobs; q++)
    #pragma unroll
            for (int a2 = 0; a2 < 2; a2++)
    #pragma unroll
                for (int b4 = 0; b4 < 4; b4++) acc2[q][a2][b4] = 0;
        for (int r0 = 0; r0 < P.n_rows; r0 += kRt) {
            const int nr = min(kRt, P.n_rows - r0);
            __syncthreads();
            for (int idx = tid; idx < nr * mfit; idx += kThreads) {
                const int j = idx / nr, r = idx - j * nr;
                const int row = r0 + r;
                const double d = Jt[(size_t)P.free_idx[j] * npad + row];
                Js[r * jst + j] = d;
                Ws[r * wst + j] = d * P.sig2i[row] * P.wght[row];
            }
            for (int r = tid; r < nr; r += kThreads) {
                const int row = r0 + r;
                const double dy = P.yobs[row] - yt[row];
                for (int k = mfit; k < jst; k++) Js[r * jst + k] = k == kB ? dy : (k == kB + 1 ? 1.0 : 0.0);
                for (int j = mfit; j < wst; j++) Ws[r * wst + j] = j == jC ? dy * dy * P.sig2i[row] * P.wght[row] : 0.0;
            }
            __syncthreads();
    #pragma unroll
            for (int q = 0; q < kJobs; q++) {
                const int e = tid + q * kThreads;
                if (e < njob) {
                    const int j0 = jobs[e] & 0xffff, k0 = jobs[e] >> 16;
                    const double* wp = Ws + j0;
                    const double* jp = Js + k0;
                    for (int r = 0; r < nr; r++) {
                        const double2 w = *reinterpret_cast<const double2*>(wp + r * wst);
                        const double2 ja = *reinterpret_cast<const double2*>(jp + r * jst);
                        const double2 jb = *reinterpret_cast<const double2*>(jp + r * jst + 2);
                        const double wv[2] = {w.x, w.y}, jv[4] = {ja.x, ja.y, jb.x, jb.y};
    #pragma unroll
                        for (int a2 = 0; a2 < 2; a2++)
    #pragma unroll
                            for (int b4 = 0; b4 < 4; b4++) acc2[q][a2][b4] = acc2[q][a2][b4] + wv[a2] * jv[b4];
                    }
                }
            }
        }
    #pragma unroll
        for (int q = 0; q < kJobs; q++) {
            const int e = tid + q * kThreads;
            if (e < njob) {
                const int j0 = jobs[e] & 0xffff, k0 = jobs[e] >> 16;
    #pragma unroll
                for (int a2 = 0; a2 < 2; a2++)
    #pragma unroll
                    for (int b4 = 0; b4 < 4; b4++) {
                        const int j = j0 + a2, k = k0 + b4;
                        const double v = acc2[q][a2][b4];
                        if (j < mfit && k < mfit) {
                            if (k <= j) {
                                alpha_out[j * mfit + k] = v;
                                alpha_out[k * mfit + j] = v;
                            }
                        } else if (j < mfit && k == kB) {
                            beta_out[j] = v;
                        } else if (j == jC && k == kB + 1) {
                            misc[M_CHISQ] = v;
                        }
                    }
            }
        }
    }
    __syncthreads();
}

template <int NCB, bool kFast>
__global__ void __launch_bounds__(kThreads, NCB <= 64 ? 2 : 1) fit_kernel(const DevProblem* __restrict__ Parr, FitBatch Bt) {
    // No static __shared__ variable may be declared in these kernels: with
    // one, the dynamic region would start after it here but not in the
    // out-of-line evaluate(), which addresses it through its own extern
    // declaration.  The queue slots live in the first 16 bytes instead.
    extern __shared__ __align__(16) double sm[];
    int& s_work = reinterpret_cast<int*>(sm)[0];
    int& s_ast = reinterpret_cast<int*>(sm)[1];
    const int tid = threadIdx.x;
    int cur_mfit = -1, cur_ent = -1;
    for (;;) {
        __syncthreads();
        if (tid == 0) {
            const int nf = Bt.n_fits_dev ? *Bt.n_fits_dev : Bt.n_fits;
            int w = atomicAdd(Bt.queue, 1);
            int a = 0;
            if (w >= nf) {
                w = -1;
            } else if (Bt.n_ast > 1) {
                // queue position -> asteroid; with an order, the queue runs over
                // the asteroids in that order (largest first) and w becomes the
                // fit's index in the asteroid-ordered result array
                const int* off = Bt.ast_order ? Bt.ast_ord_off : Bt.ast_fit_off;
                int lo = 0, hi = Bt.n_ast - 1;  // last k with off[k] <= w
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (off[mid] <= w)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                a = lo;
                if (Bt.ast_order) {
                    a = Bt.ast_order[lo];
                    w = Bt.ast_fit_off[a] + (w - off[lo]);
                }
            }
            s_work = w;
            s_ast = a;
        }
        __syncthreads();
        const int w = s_work;
        if (w < 0) break;
        const DevProblem* Pp = Parr + s_ast;
        const DevProblem& P = *Pp;
        const Layout L = make_layout(P);
        const int C = P.C, ma = P.ma, mfit = P.mfit;
        double* cg = sm + L.cg;
        double* atry = sm + L.atry;
        double* misc = sm + L.misc;
        double* Jt = Bt.scratch + (size_t)blockIdx.x * Bt.scratch_stride;
        double* yt = Jt + (size_t)ma * P.npad;
        if (mfit != cur_mfit || L.ent != cur_ent) {
            alpha_jobs(mfit, (int*)(sm + L.ent));
            cur_mfit = mfit;
            cur_ent = L.ent;
        }
        const unsigned long long t_start = global_ns();
        double freq;
        int pole;
        if (Bt.pole_override) {
            freq = Bt.freq_override;
            pole = Bt.pole_override;
        } else {
            const int local = Bt.n_ast > 1 ? w - Bt.ast_fit_off[s_ast] : w;
            const int n = (Bt.n_ast > 1 ? Bt.ast_n_from[s_ast] : Bt.n_from) + local / 10;
            pole = local % 10 + 1;
            freq = P.freq_start - (n - 1) * P.freq_step;
        }
        // initial parameters, period_search_BOINC.cpp:819-844
        for (int i = tid; i < ma; i += kThreads) {
            double v;
            if (i < C)
                v = P.cg_first[i];
            else if (i == C)
                v = P.pole0[(pole - 1) * 2];
            else if (i == C + 1)
                v = P.pole0[(pole - 1) * 2 + 1];
            else if (i == C + 2) {
                const double prd = 1 / freq;
                v = 24 * 2 * kPiD / prd;
            } else if (i == C + 3)
                v = P.par1;
            else if (i == C + 4)
                v = P.par2;
            else if (i == C + 5)
                v = P.par3;
            else if (i == C + 6)
                v = P.log_cl;
            else
                v = 1;
            cg[i] = v;
        }
        __syncthreads();
        // Levenberg-Marquardt loop, period_search_BOINC.cpp:846-893, with
        // mrqmin (mrqmin.c:11-110) inlined.  Scalars are kept identically in
        // every thread.
        //
        // mrqmin evaluates mrqcof in full at every trial point, but alpha and
        // beta from a trial point are only used when the step is accepted
        // (mrqmin.c:91-101); about half the steps of these fits are rejected.
        // So a trial point gets the model alone (evaluate_model: chi2, chck,
        // facet-area sum -- all the accept/reject test and the stop rule
        // read), and the Jacobian with alpha and beta is evaluated at the new
        // point only when the next step needs it (j_stale), which also skips
        // it after the last step.  Every value, and so every result, is the
        // same as with a full evaluation per step.
        double* alpha = sm + L.alpha;
        double* covar = sm + L.work + gj_covar_off(mfit);  // free while no evaluation runs
        double* beta = sm + L.beta;
        double* da = sm + L.da;
        double alamda = -1, ochisq = 0, chisq = 0, iter_diff = 1e40, dev_old = 1e30, dev_new = 0, rchisq = -1;
        double chk0 = 0, chk1 = 0, chk2 = 0, cur0 = 0, cur1 = 0, cur2 = 0, s_cur = 0, s_last = 0;
        int niter = 0, status = 0;
        bool j_stale = false;
        while (((niter < P.n_iter_max) && (iter_diff > P.iter_diff_max)) || (niter < P.n_iter_min)) {
            if (alamda < 0) {
                alamda = P.alamda_start;
                evaluate<NCB, kFast>(Pp, (int)(cg - sm), (int)(alpha - sm), (int)(beta - sm), Jt, yt);
                ochisq = misc[M_CHISQ];
                cur0 = misc[M_CHK0];
                cur1 = misc[M_CHK0 + 1];
                cur2 = misc[M_CHK0 + 2];
                s_cur = s_last = misc[M_SAREA];
                for (int i = tid; i < ma; i += kThreads) atry[i] = cg[i];
            } else if (j_stale) {
                // alpha and beta at the point accepted last (its chi2, chck and
                // area sum came from the model-only evaluation and are kept)
                evaluate<NCB, kFast>(Pp, (int)(cg - sm), (int)(alpha - sm), (int)(beta - sm), Jt, yt);
                j_stale = false;
            }
            for (int idx = tid; idx < mfit * mfit; idx += kThreads) {
                const int j = idx / mfit, k = idx - j * mfit;
                covar[idx] = (j == k) ? alpha[idx] * (1 + alamda) : alpha[idx];
            }
            for (int j = tid; j < mfit; j += kThreads) da[j] = beta[j];
            __syncthreads();
            // the fast form solves the damped system (symmetric positive
            // definite unless singular) without pivot search; the full-pivot
            // solve decides the cases that fails on, as in the reference
            int err = kFast ? solve_spd<NCB + 8>(covar, da, mfit, sm + L.work) : -1;
            if (err < 0) err = gauss_jordan<NCB + 8>(covar, da, mfit, sm + L.work);
            __syncthreads();
            if (err == 0) {
                for (int j = tid; j < mfit; j += kThreads) {
                    const int l = P.free_idx[j];
                    atry[l] = cg[l] + da[j];
                }
                __syncthreads();
                evaluate_model<NCB, kFast>(Pp, (int)(atry - sm), yt);
                const double temp = misc[M_CHISQ];
                chisq = temp;
                s_last = misc[M_SAREA];
                if (temp < ochisq) {
                    alamda = alamda / P.alamda_incr;
                    j_stale = true;
                    for (int i = tid; i < ma; i += kThreads) cg[i] = atry[i];
                    cur0 = misc[M_CHK0];
                    cur1 = misc[M_CHK0 + 1];
                    cur2 = misc[M_CHK0 + 2];
                    s_cur = misc[M_SAREA];
                } else {
                    alamda = P.alamda_incr * alamda;
                    chisq = ochisq;
                }
            } else {
                if (status == 0) status = err;
                // The reference leaves its global Chisq untouched here; at the
                // first step that is the previous fit's value.  A fit on its own
                // uses its first chi2 instead.
                if (niter == 0) chisq = ochisq;
            }
            niter++;
            if ((niter == 1) || (chisq < ochisq)) {
                ochisq = chisq;
                chk0 = cur0;
                chk1 = cur1;
                chk2 = cur2;
                s_last = s_cur;
                rchisq = chisq - (chk0 * chk0 + chk1 * chk1 + chk2 * chk2) * (P.conw_r * P.conw_r);
            }
            dev_new = sqrt(rchisq / P.ndata_m3);
            if (dev_old - dev_new > 1e-10) {
                iter_diff = dev_old - dev_new;
                dev_old = dev_new;
            }
            __syncthreads();
        }
        if (tid == 0) {
            FitOut o;
            o.dev = dev_new;
            o.dark = sqrt(chk0 * chk0 + chk1 * chk1 + chk2 * chk2);
            o.totarea = s_last;
            o.prd = 2 * kPiD / cg[C + 2];
            o.la = (180 / kPiD) * cg[C + 1];
            o.be = 90 - (180 / kPiD) * cg[C];
            o.chisq = chisq;
            o.niter = niter;
            o.status = status;
            const unsigned long long t_end = global_ns();
            o.dur_us = (unsigned int)((t_end - t_start) / 1000ull);
            o.end_us = (unsigned int)(t_end / 1000ull);
            Bt.out[w] = o;
        }
        // a single fit (ps_fit) leaves its final parameters at the start of
        // the CTA's scratch, which no thread reads any more
        if (Bt.pole_override)
            for (int i = tid; i < ma; i += kThreads) Jt[i] = cg[i];
    }
}

// Single evaluation for the diagnostic API (ps_mrqcof / ps_model).
template <int NCB, bool kFast>
__global__ void __launch_bounds__(kThreads, 1) eval_kernel(const DevProblem* __restrict__ Pp, EvalOut E) {
    extern __shared__ __align__(16) double sm[];
    const DevProblem& P = *Pp;
    const Layout L = make_layout(P);
    const int tid = threadIdx.x;
    double* cg = sm + L.cg;
    double* Jt = E.scratch;
    double* yt = Jt + (size_t)P.ma * P.npad;
    alpha_jobs(P.mfit, (int*)(sm + L.ent));
    for (int i = tid; i < P.ma; i += kThreads) cg[i] = E.a[i];
    __syncthreads();
    evaluate<NCB, kFast>(Pp, L.cg, L.alpha, L.beta, Jt, yt);
    for (int i = tid; i < P.mfit * P.mfit; i += kThreads) E.alpha[i] = sm[L.alpha + i];
    for (int i = tid; i < P.mfit; i += kThreads) E.beta[i] = sm[L.beta + i];
    if (tid == 0) E.chisq[0] = sm[L.misc + M_CHISQ];
    for (int idx = tid; idx < P.n_rows * P.ma; idx += kThreads) {
        const int r = idx / P.ma, l = idx - r * P.ma;
        E.J[idx] = Jt[(size_t)l * P.npad + r];
    }
    for (int r = tid; r < P.n_rows; r += kThreads) E.y[r] = yt[r];
}

template <int NCB, bool kFast>
cudaError_t launch_fits_t(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s) {
    const Layout L = make_layout(P);
    cudaError_t e = cudaFuncSetAttribute(fit_kernel<NCB, kFast>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes);
    if (e != cudaSuccess) return e;
    fit_kernel<NCB, kFast><<<grid, kThreads, L.bytes, s>>>(dP, B);
    return cudaGetLastError();
}

template <int NCB, bool kFast>
cudaError_t launch_eval_t(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s) {
    const Layout L = make_layout(P);
    cudaError_t e = cudaFuncSetAttribute(eval_kernel<NCB, kFast>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes);
    if (e != cudaSuccess) return e;
    eval_kernel<NCB, kFast><<<1, kThreads, L.bytes, s>>>(dP, E);
    return cudaGetLastError();
}

template <int NCB, bool kFast>
int max_blocks_t(const DevProblem& P) {
    const Layout L = make_layout(P);
    if (cudaFuncSetAttribute(fit_kernel<NCB, kFast>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes) != cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fit_kernel<NCB, kFast>, kThreads, L.bytes) != cudaSuccess) return 0;
    return nb;
}


}  // namespace
}  // namespace fitimpl
}  // namespace psb

// Mixed-precision form of the convex-inversion fit (PS_FORM_MIXED).
//
// Same persistent one-CTA-per-fit structure as the FP64 form (ps_fp64.cu),
// with the arithmetic split by what each quantity needs:
//
//   FP64  the model brightness y (mu, mu0, visibility, Lambert + Lommel-
//         Seeliger sum per point), chi2 and the accept/reject comparison,
//         beta = J^T W dy, the rotation angle phi0 + omega t (mod 2 pi) and
//         its sin/cos, the facet areas (curv) and the damped Gauss-Jordan
//         solve -- everything that decides where a fit converges to;
//   FP32  the per-(point, facet) derivative work (dmu terms of the rotation
//         derivatives, the Lambert/Lommel-Seeliger derivatives) and the
//         Jacobian storage -- it only steers the LM steps;
//   tcgen05 the shape block of the Jacobian, J_shape = diag(Scale) U Y with
//         U[p][f] = Darea_f g_f s_pf vis_pf (points x facets) and Y = Dsph
//         (facets x coefficients), on the 5th-generation tensor cores in
//         split BF16 (hi*hi + hi*lo + lo*hi, ~2^-16 relative per product)
//         with FP32 accumulation in TMEM.
//
// Per point tile (128 points = the MMA M): the 256 threads compute U for a
// chunk of 64 facets (2 threads per point, 32 facets each, packed 8 BF16 per
// 16-byte store into the 128-byte-swizzled K-major A tile), thread 0 issues
// 4 x 3 MMAs (M=128, N=64, K=16) into the TMEM accumulator and commits to an
// mbarrier; operand tiles are double-buffered so the next chunk's SIMT work
// overlaps the tensor core.  Y chunks are stored pre-split and pre-swizzled
// in HBM (built once per asteroid) and copied to shared memory per chunk.
// alpha = J^T W J runs on the tensor cores too (kind::tf32, split TF32,
// FP32 accumulation: it only shapes the step, not the fixed point); beta and
// chi2 in FP64 on the SIMT pipes.  Every mbarrier wait is bounded; a
// wait that gives up sets the device error word, which the host reports.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ps_device.hpp"
#include "ps_fit_common.cuh"
#include "ps_fit_impl.cuh"
#include "ps_umma.cuh"

namespace psb {

namespace {

using namespace fitcommon;

constexpr int kTileP = 128;     // points per tile (MMA M)
constexpr int kKc = 64;         // facets per chunk (one swizzled 128-byte row)
constexpr int kNc = 64;         // MMA N (shape coefficients, C <= 64)
constexpr int kRtM = 32;        // rows per alpha chunk (one 128-byte FP32 K row)
// Bounded waits: the ordinary waits on the tensor core take P.max_polls
// polls at most (ps_open sets it, by default kMaxPolls); a wait that gives up
// ends the fit: the CTA stops taking work, waits for its own MMAs in flight
// with the fixed kDrainPolls limit, frees its TMEM and returns, and the host
// reports PS_ERR_DEVICE_LOOP.
constexpr uint32_t kDrainPolls = 1u << 26;
constexpr uint32_t kTmemCols = 64;

// Shared memory: a 1024-byte aligned block of MMA operand tiles followed by
// the doubles/floats/ints of the fit.
struct MLayout {
    uint32_t a_hi[2], a_lo[2], b_hi[2], b_lo[2];  // byte offsets
    uint32_t mbar, tslot, exch;                   // byte offsets
    uint32_t dbl;                                 // byte offset of the double region
    int cg, atry, alpha, covar, beta, da, area, dres, dave, blm, misc, red, gwork;  // double offsets
    uint32_t flt;                                 // byte offset of the float region
    int area32, dga32;                            // float offsets
    uint32_t ints;                                // byte offset of the int region
    int ipiv;                                     // int offsets
    size_t bytes;                                 // total incl. 1024 B alignment slack
};

// Doubles of the model pass's work buffer (staged normals, sort keys,
// lightcurve sums).
__host__ __device__ inline int model_work_doubles(const DevProblem& P) {
    int w = 4 * fitimpl::kMf;
    if (P.sortseg > w) w = P.sortseg;
    if (kThreads > w) w = kThreads;
    return w;
}

__host__ __device__ inline MLayout make_mlayout(const DevProblem& P) {
    MLayout L;
    uint32_t o = 0;
    for (int b = 0; b < 2; b++) {
        L.a_hi[b] = o;
        o += kTileP * 128;
        L.a_lo[b] = o;
        o += kTileP * 128;
    }
    for (int b = 0; b < 2; b++) {
        L.b_hi[b] = o;
        o += kNc * 128;
        L.b_lo[b] = o;
        o += kNc * 128;
    }
    // the alpha chunks (split TF32) reuse the operand buffers after the point loop
    L.mbar = o;
    o += 32;
    // TMEM base address, then the work item and asteroid of the current fit
    // (broadcast before the fit's own layout is known)
    L.tslot = o;
    o += 16;
    // per-tile exchange of the second thread's partial sums: 128 x (double + 8 floats)
    L.exch = o;
    o += kTileP * 48;
    o = (o + 15) & ~15u;
    L.dbl = o;
    int d = 0;
#define PSB_TAKE(field, n) \
    L.field = d;           \
    d += ((n) + 1) & ~1;
    PSB_TAKE(cg, P.ma)
    PSB_TAKE(atry, P.ma)
    PSB_TAKE(alpha, P.mfit * P.mfit)
    PSB_TAKE(covar, P.mfit * P.mfit)
    PSB_TAKE(beta, P.mfit)
    PSB_TAKE(da, P.mfit)
    PSB_TAKE(area, P.F)
    PSB_TAKE(dres, 3 * P.C)
    PSB_TAKE(dave, P.ma + 2)
    PSB_TAKE(blm, 28)
    PSB_TAKE(misc, 32)
    PSB_TAKE(red, 2 * (kThreads / 32) + 2)
    PSB_TAKE(gwork, gj_buf_doubles(P.mfit) > 3 * kRtM ? gj_buf_doubles(P.mfit) : 3 * kRtM)  // solve; alpha rows
#undef PSB_TAKE
    o += (uint32_t)d * 8;
    L.flt = o;
    int f = 0;
    L.area32 = f;
    f += (P.F + 3) & ~3;
    L.dga32 = f;
    f += (P.F + 3) & ~3;
    o += (uint32_t)f * 4;
    L.ints = o;
    L.ipiv = 0;
    o += (uint32_t)((P.mfit + 3) & ~3) * 4;
    L.bytes = (size_t)o + 1024;
    return L;
}

enum {
    M_CHISQ = 0,
    M_CHK0 = 1,
    M_SAREA = 4,
    M_CL = 5,
    M_CLS = 6,
    M_OMG = 7,
    M_P1 = 8,
    M_P2 = 9,
    M_P3 = 10,
    M_WORK = 11,
    M_ABORT = 12  // a bounded wait of the last evaluation gave up
};

struct MPtr {
    uint8_t* base;  // 1024-aligned
    MLayout L;
    double* dbl;
    float* flt;
    int* ints;
    __device__ double* d(int off) const { return dbl + off; }
};

__device__ inline MPtr mptrs(const DevProblem& P, uint8_t* raw) {
    MPtr m;
    const uint32_t b = umma::smem_u32(raw);
    m.base = raw + (((b + 1023u) & ~1023u) - b);
    m.L = make_mlayout(P);
    m.dbl = (double*)(m.base + m.L.dbl);
    m.flt = (float*)(m.base + m.L.flt);
    m.ints = (int*)(m.base + m.L.ints);
    return m;
}

// One model evaluation in the mixed form (the reference's mrqcof,
// mrqcof.c:16-148).  alpha_out/beta_out in shared memory (FP64); chi2, the
// convexity residuals and the facet-area sum in misc.  Jf: FP32 Jacobian
// columns (ma x npad), yt: FP64 model (npad).  gc: running chunk counter of
// this CTA (selects operand buffer and mbarrier phase).
__device__ __noinline__ void evaluate_mixed(const DevProblem* __restrict__ Pp, uint8_t* raw, const double* a,
                                            double* alpha_out, double* beta_out, float* Jf, double* yt,
                                            uint32_t tmem, uint32_t* gc_io) {
    const DevProblem& P = *Pp;
    const MPtr M = mptrs(P, raw);
    const MLayout& L = M.L;
    const int tid = threadIdx.x;
    const int F = P.F, C = P.C, ma = P.ma, npad = P.npad, mfit = P.mfit;
    double* area = M.d(L.area);
    double* misc = M.d(L.misc);
    double* B = M.d(L.blm);
    double* D = B + 9;
    double* dres = M.d(L.dres);
    float* area32 = M.flt + L.area32;
    float* dga32 = M.flt + L.dga32;
    uint64_t* mbar = (uint64_t*)(M.base + L.mbar);
    uint32_t gc = *gc_io;
    bool aborted = false;

    if (tid == 0) {
        blmatrix(a[C], a[C + 1], B, D);
        misc[M_CL] = exp(a[C + 6]);
        misc[M_CLS] = a[C + 7];
        misc[M_OMG] = a[C + 2];
        misc[M_P1] = a[C + 3];
        misc[M_P2] = a[C + 4];
        misc[M_P3] = a[C + 5];
    }
    // curv (curv.c:15-37) in FP64
    for (int f = tid; f < F; f += kThreads) {
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
        const double darea = P.fac[(size_t)f * 4 + 3];
        area[f] = darea * gi;
        area32[f] = (float)(darea * gi);
        dga32[f] = (float)(darea * gi);
    }
    __syncthreads();
    // convexity residuals, facet-area sum and convexity-row derivatives
    // (conv.c:12-29), FP64, one thread per sum
    for (int job = tid; job < 4 + 3 * C; job += kThreads) {
        double s = 0;
        if (job < 3) {
            for (int f = 0; f < F; f++) s = fma(area[f], P.fac[(size_t)f * 4 + job], s);
            misc[M_CHK0 + job] = s;
        } else if (job == 3) {
            for (int f = 0; f < F; f++) s += area[f];
            misc[M_SAREA] = s;
        } else {
            const int nc = (job - 4) / C, j = (job - 4) - nc * C;
            for (int f = 0; f < F; f++)
                s = fma(area[f] * P.dsph[(size_t)f * P.NCB + j], P.fac[(size_t)f * 4 + nc], s);
            dres[nc * C + j] = s;
        }
    }
    const double cl = misc[M_CL], cls = misc[M_CLS];
    const float clf = (float)cl, clsf = (float)cls;
    const uint32_t idesc = umma::idesc_bf16_f32(kTileP, kNc);
    const int pl_ = tid & (kTileP - 1), half = tid >> 7;
    const int nch = P.nchunk;
    for (int base = 0; base < P.n_points; base += kTileP) {
        const int p = base + pl_;
        const bool act = p < P.n_points;
        PointGeom G;
        if (act) point_geometry(P, p, B, D, misc[M_OMG], misc[M_P1], misc[M_P2], misc[M_P3], G);
        double br = 0;
        float T0 = 0, T1 = 0, T2 = 0, S0 = 0, S1 = 0, S2 = 0, scl = 0, scls = 0;
        for (int ch = 0; ch < nch; ch++, gc++) {
            const int buf = gc & 1;
            // operand buffer `buf` is free once the MMAs of chunk gc - 2 are done
            bool fail = false;
            if (tid == 0 && gc >= 2) fail = !umma::mbar_wait(&mbar[buf], ((gc - 2) >> 1) & 1, P.max_polls);
            if (__syncthreads_or(fail)) {
                aborted = true;
                break;
            }
            // Y chunk (hi, lo) into the B tiles: 16 KB, 4 x 16 B per thread
            {
                const uint4* src = (const uint4*)(P.bsw + (size_t)ch * 2 * kNc * kKc);
                uint4* dhi = (uint4*)(M.base + L.b_hi[buf]);
                uint4* dlo = (uint4*)(M.base + L.b_lo[buf]);
                for (int i = tid; i < 512; i += kThreads) {
                    dhi[i] = src[i];
                    dlo[i] = src[512 + i];
                }
            }
            // U for this thread's point and 32 facets, 4 groups of 8
            uint8_t* ahi = M.base + L.a_hi[buf] + pl_ * 128;
            uint8_t* alo = M.base + L.a_lo[buf] + pl_ * 128;
#pragma unroll 1
            for (int g8 = 0; g8 < 4; g8++) {
                float u[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    u[q] = 0.f;
                    const int f = ch * kKc + half * 32 + g8 * 8 + q;
                    if (act && f < F) {
                        const double4 n = *(const double4*)(P.fac + (size_t)f * 4);
                        const double mu = G.e[0] * n.x + G.e[1] * n.y + G.e[2] * n.z;
                        const double mu0 = G.e0[0] * n.x + G.e0[1] * n.y + G.e0[2] * n.z;
                        if ((mu > kTinyD) && (mu0 > kTinyD)) {
                            const double r = 1.0 / (mu + mu0);
                            const double s = mu * mu0 * (cl + cls * r);
                            br = fma(area[f], s, br);
                            const float m = (float)mu, m0 = (float)mu0, rf = (float)r;
                            const float a32 = area32[f];
                            const float q0 = m0 * rf, q1 = m * rf;
                            const float dsmu = clsf * q0 * q0 + clf * m0;
                            const float dsmu0 = clsf * q1 * q1 + clf * m;
                            const float4 nf = *(const float4*)(P.fac32 + (size_t)f * 4);
                            const float w = a32 * dsmu, w0 = a32 * dsmu0;
                            T0 = fmaf(w, nf.x, T0);
                            T1 = fmaf(w, nf.y, T1);
                            T2 = fmaf(w, nf.z, T2);
                            S0 = fmaf(w0, nf.x, S0);
                            S1 = fmaf(w0, nf.y, S1);
                            S2 = fmaf(w0, nf.z, S2);
                            const float mm = m * m0 * a32;
                            scl += mm;
                            scls = fmaf(mm, rf, scls);
                            u[q] = dga32[f] * (float)s;
                        }
                    }
                }
                uint32_t hw[4], lw[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    __nv_bfloat16 h0, l0, h1, l1;
                    umma::split_bf16(u[2 * q], h0, l0);
                    umma::split_bf16(u[2 * q + 1], h1, l1);
                    hw[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
                    lw[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
                }
                const uint32_t chunk16 = (uint32_t)(half * 4 + g8) ^ (uint32_t)(pl_ & 7);
                *(uint4*)(ahi + chunk16 * 16) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                *(uint4*)(alo + chunk16 * 16) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
            }
            umma::fence_proxy_async();
            __syncthreads();
            if (tid == 0) {
                umma::fence_after_sync();
                const uint32_t sa_hi = umma::smem_u32(M.base + L.a_hi[buf]);
                const uint32_t sa_lo = umma::smem_u32(M.base + L.a_lo[buf]);
                const uint32_t sb_hi = umma::smem_u32(M.base + L.b_hi[buf]);
                const uint32_t sb_lo = umma::smem_u32(M.base + L.b_lo[buf]);
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const uint32_t o = kk * 32;
                    umma::mma_bf16(tmem, umma::desc_kmajor_sw128(sa_hi + o), umma::desc_kmajor_sw128(sb_hi + o), idesc,
                                   (ch > 0 || kk > 0) ? 1u : 0u);
                    umma::mma_bf16(tmem, umma::desc_kmajor_sw128(sa_hi + o), umma::desc_kmajor_sw128(sb_lo + o), idesc,
                                   1u);
                    umma::mma_bf16(tmem, umma::desc_kmajor_sw128(sa_lo + o), umma::desc_kmajor_sw128(sb_hi + o), idesc,
                                   1u);
                }
                umma::commit(&mbar[buf]);
            }
        }
        // partial sums of the second thread of each point
        double* ex_d = (double*)(M.base + L.exch);
        float* ex_f = (float*)(M.base + L.exch + kTileP * 8);
        if (half == 1) {
            ex_d[pl_] = br;
            float* e = ex_f + pl_ * 8;
            e[0] = T0;
            e[1] = T1;
            e[2] = T2;
            e[3] = S0;
            e[4] = S1;
            e[5] = S2;
            e[6] = scl;
            e[7] = scls;
        }
        if (aborted) break;
        // wait for the tile's last MMA before reading the accumulator
        {
            const uint32_t last = gc - 1;
            bool fail = false;
            if (tid == 0) fail = !umma::mbar_wait(&mbar[last & 1], (last >> 1) & 1, P.max_polls);
            if (__syncthreads_or(fail)) {
                aborted = true;
                break;
            }
        }
        umma::fence_after_sync();
        if (half == 0) {
            // warps 0-3: TMEM lanes 32w..32w+31 hold points base + 32w + lane
            float acc[16];
            const uint32_t lane_base = (uint32_t)((tid >> 5) * 32) << 16;
            if (act) {
                br += ex_d[pl_];
                const float* e = ex_f + pl_ * 8;
                T0 += e[0];
                T1 += e[1];
                T2 += e[2];
                S0 += e[3];
                S1 += e[4];
                S2 += e[5];
                scl += e[6];
                scls += e[7];
            }
            const float sc = (float)G.scale;
#pragma unroll 1
            for (int q4 = 0; q4 < 4; q4++) {
                umma::tmem_ld16(tmem + lane_base + q4 * 16, acc);
                if (act) {
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const int k = q4 * 16 + i;
                        if (k < C) Jf[(size_t)k * npad + p] = sc * acc[i];
                    }
                }
            }
            if (act) {
                const double scale = G.scale;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const float d = T0 * (float)G.de[0][k] + T1 * (float)G.de[1][k] + T2 * (float)G.de[2][k] +
                                    S0 * (float)G.de0[0][k] + S1 * (float)G.de0[1][k] + S2 * (float)G.de0[2][k];
                    Jf[(size_t)(C + k) * npad + p] = sc * d;
                }
                Jf[(size_t)(C + 3) * npad + p] = (float)(br * G.dphp[0]);
                Jf[(size_t)(C + 4) * npad + p] = (float)(br * G.dphp[1]);
                Jf[(size_t)(C + 5) * npad + p] = (float)(br * G.dphp[2]);
                Jf[(size_t)(C + 6) * npad + p] = (float)(scale * (double)scl * cl);
                Jf[(size_t)(C + 7) * npad + p] = (float)(scale * (double)scls);
                yt[p] = br * scale;
            }
        }
        umma::fence_before_sync();
        __syncthreads();
    }
    __syncthreads();
    if (aborted) {
        if (tid == 0) {
            atomicAdd(P.err, 1);
            misc[M_CHISQ] = __longlong_as_double(0x7ff8000000000000ll);
            misc[M_ABORT] = 1;
        }
        *gc_io = gc;
        __syncthreads();
        return;
    }
    // convexity rows
    for (int job = tid; job < 3 * ma; job += kThreads) {
        const int nc = job / ma, l = job - nc * ma;
        const int row = P.n_points + nc;
        Jf[(size_t)l * npad + row] = l < C ? (float)dres[nc * C + l] : 0.f;
        if (l == 0) yt[row] = misc[M_CHK0 + nc];
    }
    __syncthreads();
    // relative-lightcurve normalisation (mrqcof.c:53-104), sums in FP64
    double* dave = M.d(L.dave);
    for (int lc = 0; lc < P.n_lc; lc++) {
        if (!P.lc_rel[lc]) continue;
        const int r0 = P.lc_start[lc], r1 = P.lc_start[lc + 1];
        for (int job = tid; job <= ma; job += kThreads) {
            double s = 0;
            if (job < ma) {
                const float* col = Jf + (size_t)job * npad;
                for (int r = r0; r < r1; r++) s += (double)col[r];
            } else {
                for (int r = r0; r < r1; r++) s += yt[r];
            }
            dave[job] = s;
        }
        __syncthreads();
        const double ave = dave[ma];
        const double lpts = (double)P.lc_npts[lc];
        for (int r = r0 + tid; r < r1; r += kThreads) {
            const double coef = P.sig[r] * lpts / ave;
            const double y = yt[r];
            const double ya = y / ave;
            for (int l = 1; l < ma; l++) {
                float* d = Jf + (size_t)l * npad + r;
                *d = (float)(coef * ((double)*d - ya * dave[l]));
            }
            yt[r] = coef * y;
            Jf[r] = 0.f;
        }
        __syncthreads();
    }
    // alpha = J^T W J on the tensor cores (kind::tf32 with split-TF32
    // operands: hi*hi + hi*lo + lo*hi, FP32 accumulation in TMEM), kRtM = 32
    // rows per chunk (one 128-byte K row of FP32): A = the free parameters'
    // rows of (J w)^T, zero past mfit (M = 128), B = those of J^T (N = 64),
    // both K-major over the chunk's rows, in the point loop's operand buffers
    // and TMEM columns and with its mbarrier protocol.  beta and chi2 stay FP64
    // on the SIMT pipes: the thread that stages an item (a parameter and 4
    // rows) accumulates its share of beta, the item sums of a parameter are
    // added in a fixed order at the end; chi2 is summed in row order by one
    // thread.
    {
        constexpr int nq = kRtM / 4;      // items per parameter and chunk
        double* dyw = M.d(L.gwork);       // [kRtM] dy sig2i w
        double* dyv = dyw + kRtM;         // [kRtM] dy
        float* wf = (float*)(dyv + kRtM);  // [kRtM] sig2i w in FP32 (for A)
        double* bpart = M.d(L.covar);     // [mfit][nq] item sums of beta (covar is free here)
        const int nitems = mfit * nq;
        double bacc[2] = {0.0, 0.0}, cacc = 0.0;
        // rows past mfit are zero in every chunk: clear them once in both buffers
        for (int b = 0; b < 2; b++) {
            for (int i = tid; i < (kTileP - mfit) * 8; i += kThreads) {
                const uint32_t o = (uint32_t)(mfit + (i >> 3)) * 128 + (uint32_t)(i & 7) * 16;
                *(uint4*)(M.base + L.a_hi[b] + o) = make_uint4(0u, 0u, 0u, 0u);
                *(uint4*)(M.base + L.a_lo[b] + o) = make_uint4(0u, 0u, 0u, 0u);
            }
            for (int i = tid; i < (kNc - mfit) * 8; i += kThreads) {
                const uint32_t o = (uint32_t)(mfit + (i >> 3)) * 128 + (uint32_t)(i & 7) * 16;
                *(uint4*)(M.base + L.b_hi[b] + o) = make_uint4(0u, 0u, 0u, 0u);
                *(uint4*)(M.base + L.b_lo[b] + o) = make_uint4(0u, 0u, 0u, 0u);
            }
        }
        const uint32_t idesc_a = umma::idesc_tf32_f32(kTileP, kNc);
        const int nch_a = (P.n_rows + kRtM - 1) / kRtM;
        for (int ch = 0; ch < nch_a; ch++, gc++) {
            const int buf = gc & 1, r0 = ch * kRtM;
            bool fail = false;
            if (tid == 0 && gc >= 2) fail = !umma::mbar_wait(&mbar[buf], ((gc - 2) >> 1) & 1, P.max_polls);
            if (__syncthreads_or(fail)) {
                aborted = true;
                break;
            }
            if (tid < kRtM) {
                const int row = r0 + tid;
                double dy = 0.0, dw = 0.0, w = 0.0;
                if (row < P.n_rows) {
                    dy = P.yobs[row] - yt[row];
                    dw = dy * P.sig2i[row] * P.wght[row];
                    w = P.sig2i[row] * P.wght[row];
                }
                dyv[tid] = dy;
                dyw[tid] = dw;
                wf[tid] = (float)w;
            }
            __syncthreads();
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int it = tid + s * kThreads;
                if (it < nitems) {
                    const int j = it / nq, rr = 4 * (it - j * nq);
                    const float* src = Jf + (size_t)P.free_idx[j] * npad + r0 + rr;
                    uint32_t ah[4], al[4], bh[4], bl[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float jv = r0 + rr + i < P.n_rows ? src[i] : 0.f;
                        umma::split_tf32(jv * wf[rr + i], ah[i], al[i]);
                        umma::split_tf32(jv, bh[i], bl[i]);
                        bacc[s] = fma((double)jv, dyw[rr + i], bacc[s]);
                    }
                    const uint32_t o = umma::sw128_off32(j, rr);  // four consecutive rows: one 16-byte chunk
                    *(uint4*)(M.base + L.a_hi[buf] + o) = make_uint4(ah[0], ah[1], ah[2], ah[3]);
                    *(uint4*)(M.base + L.a_lo[buf] + o) = make_uint4(al[0], al[1], al[2], al[3]);
                    *(uint4*)(M.base + L.b_hi[buf] + o) = make_uint4(bh[0], bh[1], bh[2], bh[3]);
                    *(uint4*)(M.base + L.b_lo[buf] + o) = make_uint4(bl[0], bl[1], bl[2], bl[3]);
                }
            }
            if (tid == kThreads - 1)
                for (int r = 0; r < kRtM; r++) cacc = fma(dyv[r], dyw[r], cacc);
            umma::fence_proxy_async();
            __syncthreads();
            if (tid == 0) {
                umma::fence_after_sync();
                const uint32_t sa_hi = umma::smem_u32(M.base + L.a_hi[buf]);
                const uint32_t sa_lo = umma::smem_u32(M.base + L.a_lo[buf]);
                const uint32_t sb_hi = umma::smem_u32(M.base + L.b_hi[buf]);
                const uint32_t sb_lo = umma::smem_u32(M.base + L.b_lo[buf]);
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const uint32_t o = kk * 32;
                    umma::mma_tf32(tmem, umma::desc_kmajor_sw128(sa_hi + o), umma::desc_kmajor_sw128(sb_hi + o),
                                   idesc_a, (ch > 0 || kk > 0) ? 1u : 0u);
                    umma::mma_tf32(tmem, umma::desc_kmajor_sw128(sa_hi + o), umma::desc_kmajor_sw128(sb_lo + o),
                                   idesc_a, 1u);
                    umma::mma_tf32(tmem, umma::desc_kmajor_sw128(sa_lo + o), umma::desc_kmajor_sw128(sb_hi + o),
                                   idesc_a, 1u);
                }
                umma::commit(&mbar[buf]);
            }
        }
        if (!aborted) {
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int it = tid + s * kThreads;
                if (it < nitems) bpart[it] = bacc[s];
            }
            // the last chunk's MMAs (and with them all earlier ones) before the read-back
            const uint32_t last = gc - 1;
            bool fail = false;
            if (tid == 0) fail = !umma::mbar_wait(&mbar[last & 1], (last >> 1) & 1, P.max_polls);
            if (__syncthreads_or(fail)) aborted = true;
        }
        if (!aborted) {
            umma::fence_after_sync();
            if (tid < kTileP) {
                // warps 0-3: TMEM lanes 32w..32w+31 hold parameter rows j
                const int j = tid;
                const uint32_t lane_base = (uint32_t)((tid >> 5) * 32) << 16;
                float acc[16];
#pragma unroll 1
                for (int q4 = 0; q4 < kNc / 16; q4++) {
                    umma::tmem_ld16(tmem + lane_base + q4 * 16, acc);
                    if (j < mfit) {
#pragma unroll
                        for (int i = 0; i < 16; i++) {
                            const int k = q4 * 16 + i;
                            if (k <= j) {  // the lower triangle, mirrored: alpha exactly symmetric
                                alpha_out[j * mfit + k] = (double)acc[i];
                                alpha_out[k * mfit + j] = (double)acc[i];
                            }
                        }
                    }
                }
            }
            if (tid < mfit) {
                double b = 0.0;
                for (int q = 0; q < nq; q++) b += bpart[tid * nq + q];
                beta_out[tid] = b;
            }
            if (tid == kThreads - 1) misc[M_CHISQ] = cacc;
            umma::fence_before_sync();
        } else if (tid == 0) {
            atomicAdd(P.err, 1);
            misc[M_CHISQ] = __longlong_as_double(0x7ff8000000000000ll);
            misc[M_ABORT] = 1;
        }
    }
    *gc_io = gc;
    __syncthreads();
}

// The model alone at a trial point (fitimpl::model_pass: FP64, the fast
// form's arithmetic), with the operand-tile region -- idle between
// evaluations -- as its g, work and perm buffers and, when they fit, its
// model rows (nothing reads them after the pass), else yt.
__device__ __noinline__ void evaluate_model_mixed(const DevProblem* __restrict__ Pp, uint8_t* raw, const double* a,
                                                  double* yt) {
    const DevProblem& P = *Pp;
    const MPtr M = mptrs(P, raw);
    const MLayout& L = M.L;
    double* g = (double*)M.base;
    const size_t work_off = (((size_t)P.F * 8) + 255) & ~(size_t)255;
    double* work = (double*)(M.base + work_off);
    int* perm = (int*)(M.base + work_off + (size_t)model_work_doubles(P) * 8);
    const size_t y_off = (work_off + (size_t)model_work_doubles(P) * 8 + (size_t)P.sortseg * 4 + 15) & ~(size_t)15;
    double* ym = y_off + (size_t)P.npad * 8 <= (size_t)(4 * kTileP * 128 + 4 * kNc * 128) ? (double*)(M.base + y_off)
                                                                                           : yt;
    fitimpl::model_pass<true>(P, a, g, M.d(L.area), M.d(L.misc), M.d(L.blm), M.d(L.blm) + 9, work, perm, ym);
}

__device__ void tmem_setup(const DevProblem& P, uint8_t* raw, uint32_t* tmem) {
    const MPtr M = mptrs(P, raw);
    uint32_t* slot = (uint32_t*)(M.base + M.L.tslot);
    uint64_t* mbar = (uint64_t*)(M.base + M.L.mbar);
    if ((threadIdx.x >> 5) == 0) umma::tmem_alloc(slot, kTmemCols);
    if (threadIdx.x == 0) {
        umma::mbar_init(&mbar[0], 1);
        umma::mbar_init(&mbar[1], 1);
        umma::mbar_init(&mbar[2], 1);  // the final drain
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    *tmem = *slot;
}

// Every MMA this CTA issued completes (bounded by the fixed drain limit,
// which no setting lowers) before its TMEM is freed.
__device__ void tmem_teardown(const DevProblem& P, uint8_t* raw, uint32_t tmem) {
    const MPtr M = mptrs(P, raw);
    uint64_t* mbar = (uint64_t*)(M.base + M.L.mbar);
    if (threadIdx.x == 0) {
        umma::commit(&mbar[2]);
        if (!umma::mbar_wait(&mbar[2], 0, kDrainPolls)) atomicAdd(P.err, 1);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if ((threadIdx.x >> 5) == 0) umma::tmem_dealloc(tmem, kTmemCols);
}

// Persistent: one fit per CTA at a time from the work queue.  In a batch
// (Bt.n_ast > 1) the problems Parr[a] share lmax, mmax and nrows and differ
// in their data and in mfit (calibrated lightcurves free one more
// parameter), so the shared-memory layout is set per fit (the launch gives
// the largest); only the byte regions before the doubles (operand tiles,
// mbarriers, TMEM slot, work slots) are the same for all.  The fits of
// asteroid a are [ast_fit_off[a], ast_fit_off[a + 1]) of the queue, in queue
// order ast_order when it is given (largest asteroid first).
__global__ void __launch_bounds__(kThreads, 1) mixed_fit_kernel(const DevProblem* __restrict__ Parr, FitBatch Bt) {
    extern __shared__ uint8_t smem_raw[];
    const int tid = threadIdx.x;
    uint32_t tmem;
    tmem_setup(Parr[0], smem_raw, &tmem);
    int* qslot;  // [0] work item, [1] asteroid
    {
        const MPtr M0 = mptrs(Parr[0], smem_raw);
        qslot = (int*)(M0.base + M0.L.tslot) + 1;
    }
    uint32_t gc = 0;
    bool aborted = false;

    while (!aborted) {
        __syncthreads();
        if (tid == 0) {
            const int nf = Bt.n_fits_dev ? *Bt.n_fits_dev : Bt.n_fits;
            int w = atomicAdd(Bt.queue, 1);
            int a = 0;
            if (w >= nf) {
                w = -1;
            } else if (Bt.n_ast > 1) {
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
            qslot[0] = w;
            qslot[1] = a;
        }
        __syncthreads();
        const int w = qslot[0];
        if (w < 0) break;
        const unsigned long long t_start = fitimpl::global_ns();
        const int ast = qslot[1];
        const DevProblem* Pp = Parr + ast;
        const DevProblem& P = *Pp;
        const MPtr M = mptrs(P, smem_raw);
        const MLayout& L = M.L;
        const int C = P.C, ma = P.ma, mfit = P.mfit;
        double* cg = M.d(L.cg);
        double* atry = M.d(L.atry);
        double* misc = M.d(L.misc);
        if (tid == 0) misc[M_ABORT] = 0;
        float* Jf = (float*)(Bt.scratch + (size_t)blockIdx.x * Bt.scratch_stride);
        double* yt = Bt.scratch + (size_t)blockIdx.x * Bt.scratch_stride + ((size_t)ma * P.npad + 1) / 2;
        double freq;
        int pole;
        if (Bt.pole_override) {
            freq = Bt.freq_override;
            pole = Bt.pole_override;
        } else {
            const int local = Bt.n_ast > 1 ? w - Bt.ast_fit_off[ast] : w;
            const int n = (Bt.n_ast > 1 ? Bt.ast_n_from[ast] : Bt.n_from) + local / 10;
            pole = local % 10 + 1;
            freq = P.freq_start - (n - 1) * P.freq_step;
        }
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
        double* alpha = M.d(L.alpha);
        double* covar = M.d(L.covar);
        double* beta = M.d(L.beta);
        double* da = M.d(L.da);
        // LM loop as in the FP64 fit kernels: a trial point gets the model
        // alone (FP64), alpha and beta are evaluated at an accepted point when
        // the next step needs them.
        double alamda = -1, ochisq = 0, chisq = 0, iter_diff = 1e40, dev_old = 1e30, dev_new = 0, rchisq = -1;
        double chk0 = 0, chk1 = 0, chk2 = 0, cur0 = 0, cur1 = 0, cur2 = 0, s_cur = 0, s_last = 0;
        int niter = 0, status = 0;
        bool j_stale = false;
        while (((niter < P.n_iter_max) && (iter_diff > P.iter_diff_max)) || (niter < P.n_iter_min)) {
            if (alamda < 0) {
                alamda = P.alamda_start;
                evaluate_mixed(Pp, smem_raw, cg, alpha, beta, Jf, yt, tmem, &gc);
                if (misc[M_ABORT] != 0) {
                    aborted = true;
                    break;
                }
                ochisq = misc[M_CHISQ];
                cur0 = misc[M_CHK0];
                cur1 = misc[M_CHK0 + 1];
                cur2 = misc[M_CHK0 + 2];
                s_cur = s_last = misc[M_SAREA];
                for (int i = tid; i < ma; i += kThreads) atry[i] = cg[i];
            } else if (j_stale) {
                evaluate_mixed(Pp, smem_raw, cg, alpha, beta, Jf, yt, tmem, &gc);
                if (misc[M_ABORT] != 0) {
                    aborted = true;
                    break;
                }
                j_stale = false;
            }
            for (int idx = tid; idx < mfit * mfit; idx += kThreads) {
                const int j = idx / mfit, k = idx - j * mfit;
                covar[idx] = (j == k) ? alpha[idx] * (1 + alamda) : alpha[idx];
            }
            for (int j = tid; j < mfit; j += kThreads) da[j] = beta[j];
            __syncthreads();
            // as in the fast FP64 form: diagonal pivots, full pivoting where they fail
            int err = solve_spd<72>(covar, da, mfit, M.d(L.gwork));
            if (err < 0) err = gauss_jordan<72>(covar, da, mfit, M.d(L.gwork));
            __syncthreads();
            if (err == 0) {
                for (int j = tid; j < mfit; j += kThreads) {
                    const int l = P.free_idx[j];
                    atry[l] = cg[l] + da[j];
                }
                __syncthreads();
                evaluate_model_mixed(Pp, smem_raw, atry, yt);
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
            o.chisq = aborted ? __longlong_as_double(0x7ff8000000000000ll) : chisq;
            o.niter = niter;
            o.status = aborted ? -1 : status;
            const unsigned long long t_end = fitimpl::global_ns();
            o.dur_us = (unsigned int)((t_end - t_start) / 1000ull);
            o.end_us = (unsigned int)(t_end / 1000ull);
            Bt.out[w] = o;
        }
        // a single fit (ps_fit) leaves its final parameters at the start of
        // the CTA's scratch, which no thread reads any more
        if (Bt.pole_override)
            for (int i = tid; i < ma; i += kThreads) Bt.scratch[(size_t)blockIdx.x * Bt.scratch_stride + i] = cg[i];
    }
    tmem_teardown(Parr[0], smem_raw, tmem);
}

__global__ void __launch_bounds__(kThreads, 1) mixed_eval_kernel(const DevProblem* __restrict__ Pp, EvalOut E) {
    extern __shared__ uint8_t smem_raw[];
    const DevProblem& P = *Pp;
    const MPtr M = mptrs(P, smem_raw);
    const MLayout& L = M.L;
    const int tid = threadIdx.x;
    double* cg = M.d(L.cg);
    uint32_t tmem;
    tmem_setup(P, smem_raw, &tmem);
    uint32_t gc = 0;
    float* Jf = (float*)E.scratch;
    double* yt = E.scratch + ((size_t)P.ma * P.npad + 1) / 2;
    for (int i = tid; i < P.ma; i += kThreads) cg[i] = E.a[i];
    __syncthreads();
    evaluate_mixed(Pp, smem_raw, cg, M.d(L.alpha), M.d(L.beta), Jf, yt, tmem, &gc);
    for (int i = tid; i < P.mfit * P.mfit; i += kThreads) E.alpha[i] = M.d(L.alpha)[i];
    for (int i = tid; i < P.mfit; i += kThreads) E.beta[i] = M.d(L.beta)[i];
    if (tid == 0) E.chisq[0] = M.d(L.misc)[M_CHISQ];
    for (int idx = tid; idx < P.n_rows * P.ma; idx += kThreads) {
        const int r = idx / P.ma, l = idx - r * P.ma;
        E.J[idx] = (double)Jf[(size_t)l * P.npad + r];
    }
    for (int r = tid; r < P.n_rows; r += kThreads) E.y[r] = yt[r];
    tmem_teardown(P, smem_raw, tmem);
}

bool mixed_supported(const DevProblem& P) {
    return P.C <= kNc && P.nchunk * kKc >= P.F && P.mfit >= 8 && P.mfit <= kNc &&
           P.mfit <= 0xffff && P.bsw && P.fac32 && P.err &&
           ((((size_t)P.F * 8) + 255) & ~(size_t)255) + (size_t)model_work_doubles(P) * 8 + (size_t)P.sortseg * 4 <=
               (size_t)(4 * kTileP * 128 + 4 * kNc * 128);
}

}  // namespace

size_t mixed_smem_bytes(const DevProblem& P) { return make_mlayout(P).bytes; }

int mixed_max_blocks_per_sm(const DevProblem& P, int* threads) {
    if (threads) *threads = kThreads;
    const size_t bytes = make_mlayout(P).bytes;
    if (cudaFuncSetAttribute(mixed_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mixed_fit_kernel, kThreads, bytes) != cudaSuccess) return 0;
    // TMEM: 512 columns per SM, kTmemCols per resident CTA
    if (nb > (int)(512 / kTmemCols)) nb = 512 / kTmemCols;
    return nb;
}

cudaError_t launch_mixed_fits(const DevProblem& P, const DevProblem* dP, const FitBatch& B, int grid, cudaStream_t s) {
    if (!mixed_supported(P)) return cudaErrorInvalidValue;
    const size_t bytes = make_mlayout(P).bytes;
    cudaError_t e = cudaFuncSetAttribute(mixed_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    mixed_fit_kernel<<<grid, kThreads, bytes, s>>>(dP, B);
    return cudaGetLastError();
}

cudaError_t launch_mixed_eval(const DevProblem& P, const DevProblem* dP, const EvalOut& E, cudaStream_t s) {
    if (!mixed_supported(P)) return cudaErrorInvalidValue;
    const size_t bytes = make_mlayout(P).bytes;
    cudaError_t e = cudaFuncSetAttribute(mixed_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    mixed_eval_kernel<<<1, kThreads, bytes, s>>>(dP, E);
    return cudaGetLastError();
}

}  // namespace psb

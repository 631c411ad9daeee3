// C ABI of the B200 period scan (include/period_search_b200.h): context
// lifetime, the per-asteroid device tables, the convexity-weight pre-pass
// and the period scan driver.  Replaces CUDAPrepare / CUDAPrecalc /
// CUDAStart / CUDAUnprepare (period_search_cuda/period_search/start_CUDA.h)
// and the period/pole loops of period_search/period_search_BOINC.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/period_search_b200.h"
#include "ps_adjoint.hpp"
#include "ps_ctx.hpp"
#include "ps_device.hpp"
#include "ps_host.hpp"

using psb::Problem;

namespace {

thread_local std::string g_err;
std::atomic<long long> g_launches{0};

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return PS_ERR_CUDA;
}

}  // namespace

namespace psb {
int set_error(int code, const std::string& msg) { return fail(code, msg); }

cudaError_t note_caller_stream(ps_ctx* c, cudaStream_t s) {
    if (s == c->stream || !c->caller_done) return cudaSuccess;
    c->caller_pending = true;
    return cudaEventRecord(c->caller_done, s);
}
void count_launch() { g_launches++; }

namespace {
struct PoolEntry {
    int device;
    void* p;
    size_t cap;
};
std::mutex g_pool_mu;
std::vector<PoolEntry> g_pool;
constexpr int kPoolMaxBuffers = 512;
constexpr size_t kPoolMaxBytes = 4ull << 30;
}  // namespace

cudaError_t pool_take(int device, size_t bytes, void** p, size_t* cap) {
    if (bytes == 0) bytes = 1;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        const size_t limit = std::max(2 * bytes, bytes + (1u << 20));
        int best = -1;
        for (int i = 0; i < (int)g_pool.size(); i++) {
            const PoolEntry& e = g_pool[i];
            if (e.device == device && e.cap >= bytes && e.cap <= limit && (best < 0 || e.cap < g_pool[best].cap))
                best = i;
        }
        if (best >= 0) {
            *p = g_pool[best].p;
            *cap = g_pool[best].cap;
            g_pool.erase(g_pool.begin() + best);
            return cudaSuccess;
        }
    }
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) *cap = bytes;
    return e;
}

void pool_give(int device, void* p, size_t cap) {
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        g_pool.push_back({device, p, cap});
        for (;;) {
            int count = 0, smallest = -1, largest = -1;
            size_t bytes = 0;
            for (int i = 0; i < (int)g_pool.size(); i++) {
                if (g_pool[i].device != device) continue;
                count++;
                bytes += g_pool[i].cap;
                if (smallest < 0 || g_pool[i].cap < g_pool[smallest].cap) smallest = i;
                if (largest < 0 || g_pool[i].cap > g_pool[largest].cap) largest = i;
            }
            int victim = bytes > kPoolMaxBytes ? largest : (count > kPoolMaxBuffers ? smallest : -1);
            if (victim < 0) break;
            drop.push_back(g_pool[victim].p);
            g_pool.erase(g_pool.begin() + victim);
        }
    }
    if (drop.empty()) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    for (void* q : drop) cudaFree(q);
    if (cur != device) cudaSetDevice(cur);
}
}  // namespace psb

namespace {

using psb::DevBuf;

#define PSB_CUDA(call)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// FP32 -> BF16, round to nearest even (finite inputs).
uint16_t f2bf(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
float bf2f(uint16_t h) {
    uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// Tables of the mixed-precision form: FP32 facet normals and Dsph split into
// BF16 hi/lo, laid out as the 128-byte-swizzled K-major tiles the tensor core
// reads (per chunk of 64 facets: 64 coefficient rows x 64 facets, hi then lo).
int upload_mixed(ps_ctx* c) {
    const Problem& p = c->prob;
    const int F = p.numfac, C = p.ncoef;
    if (C > 64) return fail(PS_ERR_LIMIT, "the mixed form supports up to 64 shape coefficients (lmax <= 7)");
    const int nchunk = (F + 63) / 64;
    std::vector<uint16_t> bsw((size_t)nchunk * 2 * 64 * 64, 0);
    for (int ch = 0; ch < nchunk; ch++) {
        uint16_t* hi = &bsw[(size_t)ch * 2 * 4096];
        uint16_t* lo = hi + 4096;
        for (int n = 0; n < 64; n++)
            for (int k = 0; k < 64; k++) {
                const int f = ch * 64 + k;
                const float v = (f < F && n < C) ? (float)p.dsph[(size_t)f * C + n] : 0.f;
                const uint16_t h = f2bf(v);
                const uint16_t l = f2bf(v - bf2f(h));
                const size_t off = ((size_t)n * 128 + (((size_t)2 * k) ^ ((size_t)(n & 7) << 4))) / 2;
                hi[off] = h;
                lo[off] = l;
            }
    }
    PSB_CUDA(c->d_bsw.upload(bsw, c->stream));
    PSB_CUDA(c->d_err.ensure(1));
    PSB_CUDA(cudaMemsetAsync(c->d_err.p, 0, sizeof(int), c->stream));
    c->dp.bsw = c->d_bsw.p;
    c->dp.nchunk = nchunk;
    c->dp.err = c->d_err.p;
    // PS_B200_MAX_POLLS lowers the wait limit (a test makes the waits give up
    // this way); the default is far above any wait a healthy GPU needs
    c->dp.max_polls = 1u << 24;
    if (const char* v = std::getenv("PS_B200_MAX_POLLS")) {
        const long n = std::strtol(v, nullptr, 10);
        if (n >= 0 && n <= (1l << 30)) c->dp.max_polls = (unsigned int)n;  // 0: give up at once
    }
    return PS_OK;
}

// A bounded device wait that gave up shows up here after a synchronisation.
int check_device_error(ps_ctx* c) {
    if (c->form != PS_FORM_MIXED || !c->d_err.p) return PS_OK;
    int e = 0;
    PSB_CUDA(cudaMemcpy(&e, c->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        // reported once; the context stays usable
        PSB_CUDA(cudaMemset(c->d_err.p, 0, sizeof(int)));
        return fail(PS_ERR_DEVICE_LOOP, "a device wait on the tensor-core pipeline gave up (" + std::to_string(e) +
                                            "); the fits it ended carry status -1");
    }
    return PS_OK;
}

// Stop rule as the reference sets it up per fit (period_search_BOINC.cpp:846-859).
void stop_rule(Problem& p, int& n_iter_max, double& iter_diff_max, int& n_iter_min) {
    n_iter_max = 0;
    iter_diff_max = -1;
    if (p.stop_condition > 1) {
        n_iter_max = (int)p.stop_condition;
        iter_diff_max = 0;
        p.n_iter_min = 0;  // the reference overwrites its global n_iter_min
    }
    if (p.stop_condition < 1) {
        n_iter_max = psb::kMaxNIter;
        iter_diff_max = p.stop_condition;
    }
    n_iter_min = p.n_iter_min;
}

int upload_static(ps_ctx* c) {
    Problem& p = c->prob;
    cudaStream_t s = c->stream;
    const int N = p.n_points, F = p.numfac, C = p.ncoef;
    const int NCB = ((C + 7) / 8) * 8;
    if (NCB > 88) return fail(PS_ERR_LIMIT, "the FP64 forms support up to 88 shape coefficients (lmax <= 8)");
    // points SoA: t, ex, ey, ez, e0x, e0y, e0z, alpha
    std::vector<double> pts((size_t)8 * N);
    for (int i = 0; i < N; i++) {
        const double* e = &p.ee[(size_t)i * 3];
        const double* e0 = &p.ee0[(size_t)i * 3];
        pts[(size_t)0 * N + i] = p.tim[i];
        pts[(size_t)1 * N + i] = e[0];
        pts[(size_t)2 * N + i] = e[1];
        pts[(size_t)3 * N + i] = e[2];
        pts[(size_t)4 * N + i] = e0[0];
        pts[(size_t)5 * N + i] = e0[1];
        pts[(size_t)6 * N + i] = e0[2];
        // bright.c:29-30: phase angle from the unit vectors (dot_product.c)
        const double cos_alpha = e[0] * e0[0] + e[1] * e0[1] + e[2] * e0[2];
        pts[(size_t)7 * N + i] = std::acos(cos_alpha);
    }
    PSB_CUDA(c->d_pts.upload(pts, s));
    // lightcurves incl. the convexity pseudo-curve
    const int L = p.n_lc();
    std::vector<int> lc((size_t)3 * (L + 1) + 1);
    int* lc_start = lc.data();
    int* lc_rel = lc.data() + (L + 2);
    int* lc_npts = lc_rel + (L + 1);
    lc_start[0] = 0;
    for (int i = 0; i < L; i++) {
        lc_start[i + 1] = lc_start[i] + p.lc_points[i];
        lc_rel[i] = p.lc_rel[i];
        lc_npts[i] = p.lc_points[i];
    }
    lc_start[L + 1] = lc_start[L] + 3;
    lc_rel[L] = 0;
    lc_npts[L] = 3;
    // facets
    std::vector<double> fac((size_t)F * 4), dsph((size_t)F * NCB, 0.0);
    int nq = 0;
    for (int m = 0; m <= p.mmax; m++) nq += p.lmax - m + 1;
    std::vector<double> cpl((size_t)F * nq), cfc((size_t)F * (p.mmax + 1)), cfs((size_t)F * (p.mmax + 1));
    const int L1 = p.lmax + 1;
    for (int f = 0; f < F; f++) {
        fac[(size_t)f * 4 + 0] = p.nor[(size_t)f * 3 + 0];
        fac[(size_t)f * 4 + 1] = p.nor[(size_t)f * 3 + 1];
        fac[(size_t)f * 4 + 2] = p.nor[(size_t)f * 3 + 2];
        fac[(size_t)f * 4 + 3] = p.darea[f];
        for (int k = 0; k < C; k++) dsph[(size_t)f * NCB + k] = p.dsph[(size_t)f * C + k];
        int q = 0;
        for (int m = 0; m <= p.mmax; m++)
            for (int l = m; l <= p.lmax; l++) cpl[(size_t)f * nq + q++] = p.pleg[((size_t)f * L1 + l) * L1 + m];
        for (int m = 0; m <= p.mmax; m++) {
            cfc[(size_t)f * (p.mmax + 1) + m] = p.fc[(size_t)f * (p.mmax + 1) + m];
            cfs[(size_t)f * (p.mmax + 1) + m] = p.fs[(size_t)f * (p.mmax + 1) + m];
        }
    }
    PSB_CUDA(c->d_fac.upload(fac, s));
    // FP32 copies of the normals (the mixed form reads them)
    std::vector<float> fac32((size_t)F * 4, 0.f);
    for (int f = 0; f < F; f++)
        for (int k = 0; k < 3; k++) fac32[(size_t)f * 4 + k] = (float)p.nor[(size_t)f * 3 + k];
    PSB_CUDA(c->d_fac32.upload(fac32, s));
    PSB_CUDA(c->d_dsph.upload(dsph, s));
    PSB_CUDA(c->d_cpl.upload(cpl, s));
    PSB_CUDA(c->d_cfc.upload(cfc, s));
    PSB_CUDA(c->d_cfs.upload(cfs, s));
    PSB_CUDA(c->d_cgf.upload(p.cg_first, s));
    // initial poles (period_search_BOINC.cpp:197-206, 825-830)
    static const double beta_pole[10] = {0, 0, 0, 0, 60, 60, 60, -60, -60, -60};
    static const double lambda_pole[10] = {0, 90, 180, 270, 60, 180, 300, 60, 180, 300};
    const double deg2rad = M_PI / 180;
    std::vector<double> pole(20);
    for (int m = 0; m < 10; m++) {
        double b = beta_pole[m];
        b = 90 - b;
        pole[m * 2] = deg2rad * b;
        pole[m * 2 + 1] = deg2rad * lambda_pole[m];
    }
    PSB_CUDA(c->d_pole.upload(pole, s));
    c->free_idx.clear();
    for (int i = 0; i < p.ma; i++)
        if (p.ia[i]) c->free_idx.push_back(i);
    std::vector<int> ints(lc);
    ints.insert(ints.end(), c->free_idx.begin(), c->free_idx.end());
    PSB_CUDA(c->d_lc.upload(ints, s));
    PSB_CUDA(c->d_queue.ensure(1));

    psb::DevProblem& d = c->dp;
    d.n_points = N;
    d.n_rows = N + 3;
    d.n_lc = L + 1;
    d.F = F;
    d.C = C;
    d.NCB = NCB;
    d.nq = nq;
    d.lmax = p.lmax;
    d.mmax = p.mmax;
    d.ma = p.ma;
    d.mfit = p.mfit;
    d.npad = ((N + 3) + 31) / 32 * 32;
    const double* P0 = c->d_pts.p;
    d.t = P0;
    d.ex = P0 + (size_t)1 * N;
    d.ey = P0 + (size_t)2 * N;
    d.ez = P0 + (size_t)3 * N;
    d.e0x = P0 + (size_t)4 * N;
    d.e0y = P0 + (size_t)5 * N;
    d.e0z = P0 + (size_t)6 * N;
    d.alpha = P0 + (size_t)7 * N;
    d.lc_start = c->d_lc.p;
    d.lc_rel = c->d_lc.p + (L + 2);
    d.lc_npts = c->d_lc.p + (L + 2) + (L + 1);
    d.free_idx = c->d_lc.p + lc.size();
    d.fac = c->d_fac.p;
    d.fac32 = c->d_fac32.p;
    d.dsph = c->d_dsph.p;
    d.cpl = c->d_cpl.p;
    d.cfc = c->d_cfc.p;
    d.cfs = c->d_cfs.p;
    d.fch = 40;  // the largest chunk that keeps two c2-size fits (C = 49, mfit = 55) per SM
    d.rt = 32;
    d.sortseg = 1024;
    d.cg_first = c->d_cgf.p;
    d.pole0 = c->d_pole.p;
    d.phi0 = p.phi0;
    d.alamda_start = p.alamda_start;
    d.alamda_incr = p.alamda_incr;
    d.log_cl = std::log(p.cl);
    d.par1 = p.par[1];
    d.par2 = p.par[2];
    d.par3 = p.par[3];
    d.ndata_m3 = (double)N;
    d.freq_start = p.freq_start;
    d.freq_step = p.freq_step;
    stop_rule(p, d.n_iter_max, d.iter_diff_max, d.n_iter_min);
    int threads = 0;
    if (c->form == PS_FORM_MIXED) {
        int rc = upload_mixed(c);
        if (rc) return rc;
        c->blocks_per_sm = psb::mixed_max_blocks_per_sm(d, &threads);
    } else if (c->form == PS_FORM_FAST) {
        c->blocks_per_sm = psb::fast_max_blocks_per_sm(d, &threads);
    } else {
        c->blocks_per_sm = psb::fp64_max_blocks_per_sm(d, &threads);
    }
    if (c->blocks_per_sm <= 0)
        return fail(PS_ERR_LIMIT, "fit kernel does not fit on the device (shared memory or registers)");
    return PS_OK;
}

// Data rows for a given conw_r: the 3 convexity rows have brightness 0,
// sigma 1/conw_r and weight 1 (period_search_BOINC.cpp:491-496, 444-456).
// rows: yobs, sig, sig2i, weight, each n_points + 3 long.
void build_rows(const Problem& p, double conw_r, double* rows) {
    const int N = p.n_points, R = N + 3;
    double* yobs = rows;
    double* sig = yobs + R;
    double* sig2i = sig + R;
    double* wght = sig2i + R;
    for (int i = 0; i < N; i++) {
        yobs[i] = p.brightness[i];
        sig[i] = p.sig[i];
        wght[i] = p.weight[i];
    }
    for (int j = 0; j < 3; j++) {
        yobs[N + j] = 0;
        sig[N + j] = 1 / conw_r;
        wght[N + j] = 1;
    }
    for (int i = 0; i < R; i++) sig2i[i] = 1 / (sig[i] * sig[i]);  // mrqcof.c:113
}

int upload_rows(ps_ctx* c) {
    Problem& p = c->prob;
    const int N = p.n_points, R = N + 3;
    std::vector<double> rows((size_t)4 * R);
    build_rows(p, p.conw_r, rows.data());
    PSB_CUDA(c->d_rows.upload(rows, c->stream));
    c->dp.yobs = c->d_rows.p;
    c->dp.sig = c->d_rows.p + R;
    c->dp.sig2i = c->d_rows.p + 2 * R;
    c->dp.wght = c->d_rows.p + 3 * R;
    c->dp.conw_r = p.conw_r;
    PSB_CUDA(c->d_dp.ensure(1));
    PSB_CUDA(cudaMemcpyAsync(c->d_dp.p, &c->dp, sizeof(psb::DevProblem), cudaMemcpyHostToDevice, c->stream));
    // The copies above are from pageable host memory: the call may return
    // before the device holds the data.  A scan launched later on a caller's
    // stream is not ordered after the context's own stream, so the tables
    // must be in place before this returns.
    PSB_CUDA(cudaStreamSynchronize(c->stream));
    c->rows_ready = true;
    return PS_OK;
}

size_t scratch_stride(const ps_ctx* c) {
    return c->form == PS_FORM_MIXED ? (size_t)psb::mixed_scratch_doubles(c->dp) : (size_t)(c->dp.ma + 1) * c->dp.npad;
}

int ensure_scratch(ps_ctx* c, int slots) {
    const size_t stride = scratch_stride(c);
    PSB_CUDA(c->d_scratch.ensure(stride * slots));
    return PS_OK;
}

// Run fits [n_from, n_to] x 10 poles (or one override fit) into d_fits.
int run_fits(ps_ctx* c, int n_from, int n_fits, int pole_override, double freq_override) {
    PSB_CUDA(c->d_fits.ensure(n_fits));
    int grid = c->sms * c->blocks_per_sm;
    if (grid > n_fits) grid = n_fits;
    int rc = ensure_scratch(c, grid);
    if (rc) return rc;
    PSB_CUDA(cudaMemsetAsync(c->d_queue.p, 0, sizeof(int), c->stream));
    psb::FitBatch b{};
    b.n_from = n_from;
    b.n_fits = n_fits;
    b.pole_override = pole_override;
    b.freq_override = freq_override;
    b.queue = c->d_queue.p;
    b.out = c->d_fits.p;
    b.scratch = c->d_scratch.p;
    b.scratch_stride = (long long)scratch_stride(c);
    if (c->form == PS_FORM_MIXED)
        PSB_CUDA(psb::launch_mixed_fits(c->dp, c->d_dp.p, b, grid, c->stream));
    else if (c->form == PS_FORM_FAST)
        PSB_CUDA(psb::launch_fast_fits(c->dp, c->d_dp.p, b, grid, c->stream));
    else
        PSB_CUDA(psb::launch_fp64_fits(c->dp, c->d_dp.p, b, grid, c->stream));
    g_launches++;
    return PS_OK;
}

int scan_into(ps_ctx* c, int n_from, int n_to, ps_record* d_out) {
    const int np = n_to - n_from + 1;
    int rc = run_fits(c, n_from, np * 10, 0, 0.0);
    if (rc) return rc;
    PSB_CUDA(psb::launch_period_reduce(c->d_fits.p, np, c->dp.ndata_m3, 0, d_out, c->stream));
    g_launches++;
    return PS_OK;
}

int open_device(ps_ctx* c, int device) {
    c->device = device;
    PSB_CUDA(cudaSetDevice(device));
    PSB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    PSB_CUDA(cudaEventCreateWithFlags(&c->caller_done, cudaEventDisableTiming));
    PSB_CUDA(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
    c->host_only = false;
    int rc = upload_static(c);
    if (rc) return rc;
    PSB_CUDA(cudaStreamSynchronize(c->stream));  // tables in place before any caller stream uses them
    return PS_OK;
}

int check_ready(const ps_ctx* c, bool need_rows) {
    if (!c) return fail(PS_ERR_ARG, "null context");
    if (c->host_only) return fail(PS_ERR_ARG, "context was opened without a device");
    if (need_rows && !c->rows_ready) return fail(PS_ERR_ARG, "call ps_precalc or ps_set_conw_r first");
    return PS_OK;
}

}  // namespace

extern "C" {

const char* ps_last_error(void) { return g_err.c_str(); }

void ps_release_cached_memory(void) {
    std::vector<psb::PoolEntry> all;
    {
        std::lock_guard<std::mutex> lk(psb::g_pool_mu);
        all.swap(psb::g_pool);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (const auto& e : all) {
        cudaSetDevice(e.device);
        cudaFree(e.p);
    }
    cudaSetDevice(cur);
}
long long ps_kernel_launches(void) { return g_launches.load(); }

int ps_open_host_only(const char* path, ps_ctx** out) {
    if (!path || !out) return fail(PS_ERR_ARG, "null argument");
    *out = nullptr;
    ps_ctx* c = new ps_ctx();
    std::string err;
    int rc = psb::parse_input(path, c->prob, err);
    if (rc == 0) rc = psb::setup_geometry(c->prob, err);
    if (rc != 0) {
        delete c;
        return fail(rc == -1 ? PS_ERR_IO : rc, err);
    }
    *out = c;
    return PS_OK;
}

int ps_open_file(const char* path, int device, int form, ps_ctx** out) {
    if (form != PS_FORM_FP64 && form != PS_FORM_MIXED && form != PS_FORM_FAST) return fail(PS_ERR_ARG, "unknown form");
    int rc = ps_open_host_only(path, out);
    if (rc) return rc;
    (*out)->form = form;
    rc = open_device(*out, device);
    if (rc) {
        ps_close(*out);
        *out = nullptr;
    }
    return rc;
}

int ps_open(const ps_problem_desc* d, int device, int form, ps_ctx** out) {
    if (!d || !out) return fail(PS_ERR_ARG, "null argument");
    if (form != PS_FORM_FP64 && form != PS_FORM_MIXED && form != PS_FORM_FAST) return fail(PS_ERR_ARG, "unknown form");
    *out = nullptr;
    if (d->n_points < 1 || d->n_lc < 1 || !d->lc_points || !d->lc_relative || !d->tim || !d->ee || !d->ee0 ||
        !d->brightness || !d->sig || !d->weight)
        return fail(PS_ERR_ARG, "missing arrays in the problem description");
    ps_ctx* c = new ps_ctx();
    Problem& p = c->prob;
    int total = 0;
    for (int i = 0; i < d->n_lc; i++) {
        if (d->lc_points[i] < 1) {
            delete c;
            return fail(PS_ERR_LIMIT, "empty lightcurve");
        }
        total += d->lc_points[i];
    }
    if (total != d->n_points) {
        delete c;
        return fail(PS_ERR_ARG, "lightcurve sizes do not add up to n_points");
    }
    p.per_start = d->per_start;
    p.per_step_coef = d->per_step_coef;
    p.per_end = d->per_end;
    p.ia_prd = d->ia_prd;
    p.phi0 = d->phi0_rad;
    p.conw = d->conw;
    p.lmax = d->lmax;
    p.mmax = d->mmax;
    p.nrows = d->nrows;
    for (int i = 0; i < 3; i++) {
        p.par[i + 1] = d->par[i];
        p.ia_par[i + 1] = d->ia_par[i];
    }
    p.cl = d->cl;
    p.ia_cl = d->ia_cl;
    p.stop_condition = d->stop_condition;
    p.n_iter_min = d->n_iter_min;
    p.alamda_incr = d->alamda_incr;
    p.alamda_start = d->alamda_start;
    p.n_points = d->n_points;
    p.lc_points.assign(d->lc_points, d->lc_points + d->n_lc);
    p.lc_rel.assign(d->lc_relative, d->lc_relative + d->n_lc);
    p.tim.assign(d->tim, d->tim + d->n_points);
    p.ee.assign(d->ee, d->ee + (size_t)3 * d->n_points);
    p.ee0.assign(d->ee0, d->ee0 + (size_t)3 * d->n_points);
    p.brightness.assign(d->brightness, d->brightness + d->n_points);
    p.sig.assign(d->sig, d->sig + d->n_points);
    p.weight.assign(d->weight, d->weight + d->n_points);
    p.jd_min = d->jd_min;
    p.jd_max = d->jd_max;
    p.escl = d->escl;
    std::string err;
    int rc = psb::finish_from_arrays(p, err);
    if (rc == 0) rc = psb::setup_geometry(p, err);
    if (rc != 0) {
        delete c;
        return fail(rc, err);
    }
    c->form = form;
    rc = open_device(c, device);
    if (rc) {
        ps_close(c);
        return rc;
    }
    *out = c;
    return PS_OK;
}

void ps_close(ps_ctx* c) {
    if (!c) return;
    if (!c->host_only) {
        cudaSetDevice(c->device);
        if (c->stream) cudaStreamSynchronize(c->stream);
        if (c->caller_pending) cudaEventSynchronize(c->caller_done);
        c->d_pts.release();
        c->d_rows.release();
        c->d_fac.release();
        c->d_dsph.release();
        c->d_cpl.release();
        c->d_cfc.release();
        c->d_cfs.release();
        c->d_cgf.release();
        c->d_pole.release();
        c->d_lc.release();
        c->d_free.release();
        c->d_queue.release();
        c->d_scratch.release();
        c->d_fits.release();
        c->d_rec.release();
        c->d_eval.release();
        c->d_adj.release();
        c->d_dp.release();
        c->d_fac32.release();
        c->d_bsw.release();
        c->d_err.release();
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->caller_done) cudaEventDestroy(c->caller_done);
    }
    delete c;
}

// The fits of several convexity pre-pass rounds in one launch, round k with
// convexity weight cw[k]: every round's fits read their own copy of the
// problem (the rows differ only in the convexity rows' sigma), fits
// [k np 10, (k + 1) np 10) belong to round k.  Records (prepass rule) land in
// rec, np per round.
int prepass_rounds(ps_ctx* c, const std::vector<double>& cw, int np, std::vector<ps_record>& rec) {
    const Problem& p = c->prob;
    const int R = (int)cw.size(), rows_n = 4 * (p.n_points + 3);
    std::vector<double> rows((size_t)R * rows_n);
    std::vector<psb::DevProblem> dps(R, c->dp);
    PSB_CUDA(c->d_pre_rows.ensure(rows.size()));
    for (int k = 0; k < R; k++) {
        build_rows(p, cw[k], rows.data() + (size_t)k * rows_n);
        const double* base = c->d_pre_rows.p + (size_t)k * rows_n;
        const int nr = p.n_points + 3;
        dps[k].yobs = base;
        dps[k].sig = base + nr;
        dps[k].sig2i = base + 2 * nr;
        dps[k].wght = base + 3 * nr;
        dps[k].conw_r = cw[k];
    }
    std::vector<int> ctl(2 * R + 1);
    for (int k = 0; k <= R; k++) ctl[k] = k * np * 10;
    for (int k = 0; k < R; k++) ctl[R + 1 + k] = 1;
    PSB_CUDA(c->d_pre_rows.upload(rows, c->stream));
    PSB_CUDA(c->d_pre_dp.upload(dps, c->stream));
    PSB_CUDA(c->d_pre_ctl.upload(ctl, c->stream));
    const int n_fits = R * np * 10;
    PSB_CUDA(c->d_fits.ensure(n_fits));
    int grid = c->sms * c->blocks_per_sm;
    if (grid > n_fits) grid = n_fits;
    int rc = ensure_scratch(c, grid);
    if (rc) return rc;
    PSB_CUDA(cudaMemsetAsync(c->d_queue.p, 0, sizeof(int), c->stream));
    psb::FitBatch b{};
    b.n_from = 1;
    b.n_fits = n_fits;
    b.queue = c->d_queue.p;
    b.out = c->d_fits.p;
    b.scratch = c->d_scratch.p;
    b.scratch_stride = (long long)scratch_stride(c);
    b.n_ast = R;
    b.ast_fit_off = c->d_pre_ctl.p;
    b.ast_n_from = c->d_pre_ctl.p + R + 1;
    if (c->form == PS_FORM_MIXED)
        PSB_CUDA(psb::launch_mixed_fits(c->dp, c->d_pre_dp.p, b, grid, c->stream));
    else if (c->form == PS_FORM_FAST)
        PSB_CUDA(psb::launch_fast_fits(c->dp, c->d_pre_dp.p, b, grid, c->stream));
    else
        PSB_CUDA(psb::launch_fp64_fits(c->dp, c->d_pre_dp.p, b, grid, c->stream));
    g_launches++;
    PSB_CUDA(c->d_rec.ensure((size_t)R * np));
    PSB_CUDA(psb::launch_period_reduce(c->d_fits.p, R * np, c->dp.ndata_m3, 1, c->d_rec.p, c->stream));
    g_launches++;
    rec.resize((size_t)R * np);
    PSB_CUDA(cudaMemcpyAsync(rec.data(), c->d_rec.p, sizeof(ps_record) * R * np, cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int ps_precalc(ps_ctx* c, double* conw_r) {
    int rc = check_ready(c, false);
    if (rc) return rc;
    PSB_CUDA(cudaSetDevice(c->device));
    Problem& p = c->prob;
    int new_conw = 0;
    c->prepass_fits = 0;
    std::vector<ps_record> rec(10);
    // period_search_BOINC.cpp:488-715, with the rounds the loop may still
    // need run together: round k (convexity weight conw_r 2^k, while
    // conw_r 2^k escl^2 < 10) has the fits it would have on its own, so the
    // first round whose mean dark-facet percentage is below 1 %, and with it
    // conw_r, is the one the sequential loop stops at.
    if (p.n_periods() < 1) return fail(PS_ERR_LIMIT, "the period range holds no trial period");
    const int np = std::min(10, p.n_periods());
    while (!new_conw && p.conw_r * p.escl * p.escl < 10.0) {
        std::vector<double> cw;
        for (double w = p.conw_r; (int)cw.size() < 8 && w * p.escl * p.escl < 10.0; w = w * 2) cw.push_back(w);
        rc = prepass_rounds(c, cw, np, rec);
        if (rc) return rc;
        for (int k = 0; k < (int)cw.size() && !new_conw; k++) {
            c->prepass_fits += 10 * np;
            double sum_dark_facet = 0.0;
            for (int n = 0; n < np; n++) sum_dark_facet = sum_dark_facet + rec[(size_t)k * np + n].dark_pct;
            const double ave_dark_facet = sum_dark_facet / np;
            if (ave_dark_facet < 1.0)
                new_conw = 1;
            else
                p.conw_r = p.conw_r * 2;
        }
    }
    rc = upload_rows(c);
    if (rc) return rc;
    if (conw_r) *conw_r = p.conw_r;
    return PS_OK;
}

int ps_set_conw_r(ps_ctx* c, double conw_r) {
    int rc = check_ready(c, false);
    if (rc) return rc;
    if (!(conw_r > 0)) return fail(PS_ERR_ARG, "conw_r must be positive");
    PSB_CUDA(cudaSetDevice(c->device));
    c->prob.conw_r = conw_r;
    return upload_rows(c);
}

int ps_set_tiles(ps_ctx* c, int fch, int rt, int sortseg) {
    int rc = check_ready(c, false);
    if (rc) return rc;
    if (c->form == PS_FORM_MIXED) return fail(PS_ERR_ARG, "the mixed form has fixed tiles");
    if (fch < 4 || fch > 128 || fch % 4 || rt < 4 || rt > 256 || rt % 4 || sortseg < 32 || sortseg > 4096 ||
        (sortseg & (sortseg - 1)))
        return fail(PS_ERR_ARG, "tiles: fch and rt multiples of 4 (4..128, 4..256), sortseg a power of 2 (32..4096)");
    PSB_CUDA(cudaSetDevice(c->device));
    psb::DevProblem& d = c->dp;
    const int old[3] = {d.fch, d.rt, d.sortseg};
    d.fch = fch;
    d.rt = rt;
    d.sortseg = sortseg;
    int threads = 0;
    const int bps = c->form == PS_FORM_FAST ? psb::fast_max_blocks_per_sm(d, &threads)
                                            : psb::fp64_max_blocks_per_sm(d, &threads);
    if (bps <= 0) {
        d.fch = old[0];
        d.rt = old[1];
        d.sortseg = old[2];
        return fail(PS_ERR_LIMIT, "these tiles do not fit in shared memory");
    }
    c->blocks_per_sm = bps;
    if (c->rows_ready) {
        PSB_CUDA(cudaMemcpyAsync(c->d_dp.p, &c->dp, sizeof(psb::DevProblem), cudaMemcpyHostToDevice, c->stream));
        PSB_CUDA(cudaStreamSynchronize(c->stream));
    }
    return PS_OK;
}

int ps_autotune(ps_ctx* c, int n_periods, int* tiles, double* seconds) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (c->form != PS_FORM_FP64 && c->form != PS_FORM_FAST) return fail(PS_ERR_ARG, "autotune runs the FP64 forms");
    // at least two waves of fits at two CTAs per SM, so that tiles which
    // cost occupancy show it
    const int waves = (2 * 2 * c->sms + 9) / 10;
    const int np = std::max(1, std::min(std::max(n_periods, waves), c->prob.n_periods()));
    PSB_CUDA(cudaSetDevice(c->device));
    PSB_CUDA(c->d_rec.ensure(np));
    auto timed = [&](double& t) -> int {
        PSB_CUDA(cudaStreamSynchronize(c->stream));
        const auto t0 = std::chrono::steady_clock::now();
        int r = scan_into(c, 1, np, c->d_rec.p);
        if (r) return r;
        PSB_CUDA(cudaStreamSynchronize(c->stream));
        t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return check_device_error(c);
    };
    const int start[3] = {c->dp.fch, c->dp.rt, c->dp.sortseg};
    double t = 0;
    rc = timed(t);  // warm-up with the current tiles
    if (rc) return rc;
    int best[3] = {start[0], start[1], start[2]};
    double tbest = 1e300;
    static const int fchs[] = {16, 32, 40, 48, 56, 64}, rts[] = {16, 32, 64}, segs[] = {256, 1024};
    for (int fch : fchs)
        for (int rt : rts)
            for (int seg : segs) {
                if (c->form == PS_FORM_FP64 && (fch != start[0] || rt != start[1])) continue;  // only the sort segment
                if (ps_set_tiles(c, fch, rt, seg) != PS_OK) continue;
                rc = timed(t);
                if (rc) return rc;
                if (t < tbest) {
                    tbest = t;
                    best[0] = fch;
                    best[1] = rt;
                    best[2] = seg;
                }
            }
    rc = ps_set_tiles(c, best[0], best[1], best[2]);
    if (rc) return rc;
    if (tiles) {
        tiles[0] = best[0];
        tiles[1] = best[1];
        tiles[2] = best[2];
    }
    if (seconds) *seconds = tbest;
    return PS_OK;
}

int ps_n_periods(const ps_ctx* c) { return c ? c->prob.n_periods() : -1; }

int ps_scan_device(ps_ctx* c, int n_from, int n_to, ps_record* d_out, void* stream) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (n_from < 1 || n_to < n_from || n_to > c->prob.n_periods() || !d_out)
        return fail(PS_ERR_ARG, "period range out of bounds");
    PSB_CUDA(cudaSetDevice(c->device));
    cudaStream_t saved = c->stream;
    if (stream) c->stream = (cudaStream_t)stream;
    rc = scan_into(c, n_from, n_to, d_out);
    c->stream = saved;
    if (rc) return rc;
    if (stream) PSB_CUDA(psb::note_caller_stream(c, (cudaStream_t)stream));
    return PS_OK;
}

int ps_scan(ps_ctx* c, int n_from, int n_to, ps_record* out) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (n_from < 1 || n_to < n_from || n_to > c->prob.n_periods() || !out)
        return fail(PS_ERR_ARG, "period range out of bounds");
    PSB_CUDA(cudaSetDevice(c->device));
    const int np = n_to - n_from + 1;
    PSB_CUDA(c->d_rec.ensure(np));
    rc = scan_into(c, n_from, n_to, c->d_rec.p);
    if (rc) return rc;
    PSB_CUDA(cudaMemcpyAsync(out, c->d_rec.p, sizeof(ps_record) * np, cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int ps_fit(ps_ctx* c, double freq, int pole, ps_fit_result* out, double* cg_out) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (pole < 1 || pole > 10 || !(freq > 0) || !out) return fail(PS_ERR_ARG, "bad fit arguments");
    PSB_CUDA(cudaSetDevice(c->device));
    rc = run_fits(c, 1, 1, pole, freq);
    if (rc) return rc;
    psb::FitOut o;
    PSB_CUDA(cudaMemcpyAsync(&o, c->d_fits.p, sizeof(o), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaStreamSynchronize(c->stream));
    rc = check_device_error(c);
    if (rc) return rc;
    out->dev = o.dev;
    out->dark = o.dark;
    out->totarea = o.totarea;
    out->period_d = o.prd;
    out->lambda_deg = o.la;
    out->beta_deg = o.be;
    out->chisq = o.chisq;
    out->niter = o.niter;
    out->status = o.status;
    // a single fit leaves its final parameters at the start of its CTA's scratch
    if (cg_out)
        PSB_CUDA(cudaMemcpy(cg_out, c->d_scratch.p, (size_t)c->dp.ma * sizeof(double), cudaMemcpyDeviceToHost));
    return PS_OK;
}

static int run_eval(ps_ctx* c, const double* a, std::vector<double>& alpha, std::vector<double>& beta,
                    double& chisq, std::vector<double>* y, std::vector<double>* J) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (!a) return fail(PS_ERR_ARG, "null parameter vector");
    PSB_CUDA(cudaSetDevice(c->device));
    const psb::DevProblem& d = c->dp;
    const size_t na = d.ma, nal = (size_t)d.mfit * d.mfit, nb = d.mfit, ny = d.n_rows, nJ = (size_t)d.n_rows * d.ma;
    const size_t scratch = scratch_stride(c);
    const size_t total = na + nal + nb + 1 + ny + nJ + scratch;
    PSB_CUDA(c->d_eval.ensure(total));
    double* base = c->d_eval.p;
    psb::EvalOut E;
    E.a = base;
    E.alpha = base + na;
    E.beta = E.alpha + nal;
    E.chisq = E.beta + nb;
    E.y = E.chisq + 1;
    E.J = E.y + ny;
    E.scratch = E.J + nJ;
    PSB_CUDA(cudaMemcpyAsync(base, a, na * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (c->form == PS_FORM_MIXED)
        PSB_CUDA(psb::launch_mixed_eval(d, c->d_dp.p, E, c->stream));
    else if (c->form == PS_FORM_FAST)
        PSB_CUDA(psb::launch_fast_eval(d, c->d_dp.p, E, c->stream));
    else
        PSB_CUDA(psb::launch_fp64_eval(d, c->d_dp.p, E, c->stream));
    g_launches++;
    alpha.resize(nal);
    beta.resize(nb);
    PSB_CUDA(cudaMemcpyAsync(alpha.data(), E.alpha, nal * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaMemcpyAsync(beta.data(), E.beta, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaMemcpyAsync(&chisq, E.chisq, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (y) {
        y->resize(ny);
        PSB_CUDA(cudaMemcpyAsync(y->data(), E.y, ny * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (J) {
        J->resize(nJ);
        PSB_CUDA(cudaMemcpyAsync(J->data(), E.J, nJ * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    PSB_CUDA(cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int ps_mrqcof(ps_ctx* c, const double* a, double* alpha, double* beta, double* chisq) {
    std::vector<double> al, be;
    double x2 = 0;
    int rc = run_eval(c, a, al, be, x2, nullptr, nullptr);
    if (rc) return rc;
    if (alpha) std::memcpy(alpha, al.data(), al.size() * sizeof(double));
    if (beta) std::memcpy(beta, be.data(), be.size() * sizeof(double));
    if (chisq) *chisq = x2;
    return PS_OK;
}

// Matrix-free chi2 / beta (v == nullptr) or Gauss-Newton product (v over
// the mfit free parameters) at parameters a.
static int run_adjoint(ps_ctx* c, const double* a, const double* v, double* chi2, double* out) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (!a) return fail(PS_ERR_ARG, "null parameter vector");
    PSB_CUDA(cudaSetDevice(c->device));
    const psb::DevProblem& d = c->dp;
    const size_t work = psb::adjoint_work_doubles(d);
    PSB_CUDA(c->d_adj.ensure(work + 2 * (size_t)d.ma + d.mfit + 2));
    double* d_work = c->d_adj.p;
    double* d_a = d_work + work;
    double* d_v = d_a + d.ma;
    double* d_out = d_v + d.ma;
    double* d_chi2 = d_out + d.mfit;
    PSB_CUDA(cudaMemcpyAsync(d_a, a, d.ma * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (v) {
        std::vector<double> vf(d.ma, 0.0);
        for (int i = 0; i < d.mfit; i++) vf[c->free_idx[i]] = v[i];
        PSB_CUDA(cudaMemcpyAsync(d_v, vf.data(), d.ma * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        PSB_CUDA(cudaStreamSynchronize(c->stream));  // vf leaves scope
    }
    PSB_CUDA(psb::launch_adjoint(d, c->d_dp.p, d_work, d_a, v ? d_v : nullptr, d_out, d_chi2, c->stream));
    for (int k = 0; k < psb::kAdjointLaunches; k++) psb::count_launch();
    double x2 = 0;
    if (out) PSB_CUDA(cudaMemcpyAsync(out, d_out, d.mfit * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaMemcpyAsync(&x2, d_chi2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaStreamSynchronize(c->stream));
    if (chi2) *chi2 = x2;
    return PS_OK;
}

int ps_chi2_grad(ps_ctx* c, const double* a, double* chi2, double* beta) {
    return run_adjoint(c, a, nullptr, chi2, beta);
}

int ps_gn_product(ps_ctx* c, const double* a, const double* v, double* out) {
    if (!v) return fail(PS_ERR_ARG, "null direction vector");
    return run_adjoint(c, a, v, nullptr, out);
}

}  // extern "C"

namespace {

// Gauss-Jordan solve of a x = b (a n x n row-major, overwritten; b becomes
// x) with full pivoting as gauss_errc does it: the pivot is the last element
// of largest magnitude in row-major order among the rows and columns not yet
// used (a NaN never wins).  Returns 0, 1 when no pivot can be found, 2 on a
// zero pivot (the reference's error codes).
int host_gauss_jordan(std::vector<double>& a, std::vector<double>& b, int n) {
    std::vector<int> used(n, 0);
    for (int step = 0; step < n; step++) {
        int prow = -1, pcol = -1;
        double big = -1.0;
        for (int j = 0; j < n; j++) {
            if (used[j]) continue;
            for (int k = 0; k < n; k++) {
                if (used[k]) continue;
                const double m = std::fabs(a[(size_t)j * n + k]);
                if (m >= big) {  // NaN compares false
                    big = m;
                    prow = j;
                    pcol = k;
                }
            }
        }
        if (prow < 0) return 1;
        used[pcol] = 1;
        if (prow != pcol) {
            for (int l = 0; l < n; l++) std::swap(a[(size_t)prow * n + l], a[(size_t)pcol * n + l]);
            std::swap(b[prow], b[pcol]);
        }
        const double piv = a[(size_t)pcol * n + pcol];
        if (piv == 0.0) return 2;
        const double inv = 1.0 / piv;
        a[(size_t)pcol * n + pcol] = 1.0;
        for (int l = 0; l < n; l++) a[(size_t)pcol * n + l] *= inv;
        b[pcol] *= inv;
        for (int r = 0; r < n; r++) {
            if (r == pcol) continue;
            const double f = a[(size_t)r * n + pcol];
            a[(size_t)r * n + pcol] = 0.0;
            for (int l = 0; l < n; l++) a[(size_t)r * n + l] -= a[(size_t)pcol * n + l] * f;
            b[r] -= b[pcol] * f;
        }
    }
    return 0;
}

// Device buffers of a Jacobian-free fit, carved from d_adj.
struct JfreeBufs {
    double *work, *a, *units, *alpha, *beta, *chi2;
};

JfreeBufs jfree_bufs(ps_ctx* c) {
    const psb::DevProblem& d = c->dp;
    JfreeBufs B;
    B.work = c->d_adj.p;
    B.a = B.work + psb::adjoint_work_doubles(d);
    B.units = B.a + d.ma;
    B.alpha = B.units + (size_t)d.mfit * d.ma;
    B.beta = B.alpha + (size_t)d.mfit * d.mfit;
    B.chi2 = B.beta + d.mfit;
    return B;
}

// One evaluation at a through the matrix-free kernels: chi2, chck, the
// facet-area sum and, with full, beta and alpha (alpha's column k is the
// Gauss-Newton product with the k-th free unit vector, mfit products).
int jfree_eval(ps_ctx* c, const JfreeBufs& B, const double* a, bool full, std::vector<double>& alpha,
               std::vector<double>& beta, double* scal) {
    const psb::DevProblem& d = c->dp;
    const int mfit = d.mfit, ma = d.ma;
    PSB_CUDA(cudaMemcpyAsync(B.a, a, ma * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    PSB_CUDA(psb::launch_adjoint(d, c->d_dp.p, B.work, B.a, nullptr, B.beta, B.chi2, c->stream));
    for (int k = 0; k < psb::kAdjointLaunches; k++) psb::count_launch();
    // chck and the area sum depend on a only: read them before the products
    const double* misc = B.work + psb::adjoint_misc_offset(d);
    PSB_CUDA(cudaMemcpyAsync(scal + 1, misc + psb::kAdjMiscChk, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaMemcpyAsync(scal + 4, misc + psb::kAdjMiscSarea, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PSB_CUDA(cudaMemcpyAsync(scal, B.chi2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (full) {
        for (int k = 0; k < mfit; k++) {
            PSB_CUDA(psb::launch_adjoint(d, c->d_dp.p, B.work, B.a, B.units + (size_t)k * ma,
                                         B.alpha + (size_t)k * mfit, B.chi2 + 1, c->stream));
            for (int q = 0; q < psb::kAdjointLaunches; q++) psb::count_launch();
        }
        std::vector<double> cols((size_t)mfit * mfit);
        PSB_CUDA(cudaMemcpyAsync(cols.data(), B.alpha, cols.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
        beta.resize(mfit);
        PSB_CUDA(cudaMemcpyAsync(beta.data(), B.beta, mfit * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        PSB_CUDA(cudaStreamSynchronize(c->stream));
        // alpha[j][k] for k <= j from column k, mirrored (alpha is symmetric)
        alpha.assign((size_t)mfit * mfit, 0.0);
        for (int k = 0; k < mfit; k++)
            for (int j = k; j < mfit; j++) {
                const double v = cols[(size_t)k * mfit + j];
                alpha[(size_t)j * mfit + k] = v;
                alpha[(size_t)k * mfit + j] = v;
            }
    } else {
        PSB_CUDA(cudaStreamSynchronize(c->stream));
    }
    return PS_OK;
}

}  // namespace

extern "C" {

int ps_fit_jfree(ps_ctx* c, double freq, int pole, ps_fit_result* out, double* cg_out) {
    int rc = check_ready(c, true);
    if (rc) return rc;
    if (pole < 1 || pole > 10 || !(freq > 0) || !out) return fail(PS_ERR_ARG, "bad fit arguments");
    PSB_CUDA(cudaSetDevice(c->device));
    const psb::DevProblem& d = c->dp;
    const int ma = d.ma, mfit = d.mfit, C = d.C;
    PSB_CUDA(c->d_adj.ensure(psb::adjoint_work_doubles(d) + (size_t)ma + (size_t)mfit * ma + (size_t)mfit * mfit +
                             mfit + 2));
    const JfreeBufs B = jfree_bufs(c);
    {
        std::vector<double> units((size_t)mfit * ma, 0.0);
        for (int k = 0; k < mfit; k++) units[(size_t)k * ma + c->free_idx[k]] = 1.0;
        PSB_CUDA(cudaMemcpyAsync(B.units, units.data(), units.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 c->stream));
        PSB_CUDA(cudaStreamSynchronize(c->stream));
    }
    std::vector<double> cg(ma), atry(ma), alpha, beta, covar, da;
    psb::initial_parameters(c->prob, freq, pole, cg.data());
    double scal[5];
    // the LM loop and stop rule of the fit kernels (period_search_BOINC.cpp:846-920,
    // mrqmin.c:11-110)
    double alamda = -1, ochisq = 0, chisq = 0, iter_diff = 1e40, dev_old = 1e30, dev_new = 0, rchisq = -1;
    double chk[3] = {0, 0, 0}, cur[3] = {0, 0, 0}, s_cur = 0, s_last = 0;
    int niter = 0, status = 0;
    bool j_stale = false;
    while (((niter < d.n_iter_max) && (iter_diff > d.iter_diff_max)) || (niter < d.n_iter_min)) {
        if (alamda < 0) {
            alamda = d.alamda_start;
            rc = jfree_eval(c, B, cg.data(), true, alpha, beta, scal);
            if (rc) return rc;
            ochisq = scal[0];
            for (int i = 0; i < 3; i++) cur[i] = scal[1 + i];
            s_cur = s_last = scal[4];
            atry = cg;
        } else if (j_stale) {
            rc = jfree_eval(c, B, cg.data(), true, alpha, beta, scal);
            if (rc) return rc;
            j_stale = false;
        }
        covar = alpha;
        for (int j = 0; j < mfit; j++) covar[(size_t)j * mfit + j] = alpha[(size_t)j * mfit + j] * (1 + alamda);
        da = beta;
        const int err = host_gauss_jordan(covar, da, mfit);
        if (err == 0) {
            for (int j = 0; j < mfit; j++) atry[c->free_idx[j]] = cg[c->free_idx[j]] + da[j];
            rc = jfree_eval(c, B, atry.data(), false, alpha, beta, scal);
            if (rc) return rc;
            chisq = scal[0];
            s_last = scal[4];
            if (chisq < ochisq) {
                alamda = alamda / d.alamda_incr;
                j_stale = true;
                cg = atry;
                for (int i = 0; i < 3; i++) cur[i] = scal[1 + i];
                s_cur = scal[4];
            } else {
                alamda = d.alamda_incr * alamda;
                chisq = ochisq;
            }
        } else {
            if (status == 0) status = err;
            if (niter == 0) chisq = ochisq;
        }
        niter++;
        if ((niter == 1) || (chisq < ochisq)) {
            ochisq = chisq;
            for (int i = 0; i < 3; i++) chk[i] = cur[i];
            s_last = s_cur;
            rchisq = chisq - (chk[0] * chk[0] + chk[1] * chk[1] + chk[2] * chk[2]) * (d.conw_r * d.conw_r);
        }
        dev_new = std::sqrt(rchisq / d.ndata_m3);
        if (dev_old - dev_new > 1e-10) {
            iter_diff = dev_old - dev_new;
            dev_old = dev_new;
        }
    }
    const double kPi = 3.14159265358979323846;
    out->dev = dev_new;
    out->dark = std::sqrt(chk[0] * chk[0] + chk[1] * chk[1] + chk[2] * chk[2]);
    out->totarea = s_last;
    out->period_d = 2 * kPi / cg[C + 2];
    out->lambda_deg = (180 / kPi) * cg[C + 1];
    out->beta_deg = 90 - (180 / kPi) * cg[C];
    out->chisq = chisq;
    out->niter = niter;
    out->status = status;
    if (cg_out) std::memcpy(cg_out, cg.data(), (size_t)ma * sizeof(double));
    return PS_OK;
}

int ps_model(ps_ctx* c, const double* a, double* ymod, double* dyda) {
    std::vector<double> al, be, y, J;
    double x2 = 0;
    int rc = run_eval(c, a, al, be, x2, &y, &J);
    if (rc) return rc;
    if (ymod) std::memcpy(ymod, y.data(), y.size() * sizeof(double));
    if (dyda) std::memcpy(dyda, J.data(), J.size() * sizeof(double));
    return PS_OK;
}

int ps_info(const ps_ctx* c, int* ints, double* dbls) {
    if (!c) return fail(PS_ERR_ARG, "null context");
    const Problem& p = c->prob;
    if (ints) {
        ints[0] = p.n_points;
        ints[1] = p.n_lc() + 1;
        ints[2] = p.numfac;
        ints[3] = p.ncoef;
        ints[4] = p.ma;
        ints[5] = p.mfit;
        ints[6] = p.n_periods();
        ints[7] = c->prepass_fits;
    }
    if (dbls) {
        dbls[0] = p.escl;
        dbls[1] = p.conw_r;
        dbls[2] = p.freq_start;
        dbls[3] = p.freq_end;
        dbls[4] = p.freq_step;
    }
    return PS_OK;
}

int ps_get_array(const ps_ctx* c, const char* name, double* out) {
    if (!c || !name || !out) return -1;
    const Problem& p = c->prob;
    auto put = [&](const std::vector<double>& v) {
        std::memcpy(out, v.data(), v.size() * sizeof(double));
        return (int)v.size();
    };
    auto puti = [&](const std::vector<int>& v) {
        for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
        return (int)v.size();
    };
    const int N = p.n_points;
    if (!std::strcmp(name, "nor")) return put(p.nor);
    if (!std::strcmp(name, "darea")) return put(p.darea);
    if (!std::strcmp(name, "dsph")) return put(p.dsph);
    if (!std::strcmp(name, "cg_first")) return put(p.cg_first);
    if (!std::strcmp(name, "ia")) return puti(p.ia);
    if (!std::strcmp(name, "tim")) return put(p.tim);
    if (!std::strcmp(name, "ee")) return put(p.ee);
    if (!std::strcmp(name, "ee0")) return put(p.ee0);
    if (!std::strcmp(name, "at")) return put(p.at);
    if (!std::strcmp(name, "af")) return put(p.af);
    if (!std::strcmp(name, "ifp")) return puti(p.ifp);
    if (!std::strcmp(name, "brightness") || !std::strcmp(name, "sig") || !std::strcmp(name, "weight")) {
        const std::vector<double>& v = name[0] == 'b' ? p.brightness : (name[0] == 's' ? p.sig : p.weight);
        for (int i = 0; i < N; i++) out[i] = v[i];
        for (int j = 0; j < 3; j++) out[N + j] = name[0] == 'b' ? 0.0 : (name[0] == 's' ? 1 / p.conw_r : 1.0);
        return N + 3;
    }
    return -1;
}

int ps_format_record(const ps_record* r, int first_line, double conw_line, char* buf, int buflen) {
    if (!r || !buf || buflen <= 0) return -1;
    return std::snprintf(buf, (size_t)buflen, "%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n", r->period_h, r->rms, r->chi2,
                         first_line ? conw_line : r->dark_pct, r->lambda_deg, r->beta_deg);
}

}  // extern "C"

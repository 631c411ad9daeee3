// Batched scans: many asteroids, uneven point counts and per-fit LM
// convergence, in one persistent launch (any of the three forms).
//
// A batch holds the device copies of its contexts' problem descriptors (the
// per-asteroid tables stay where each context uploaded them), one control
// block in device memory -- total fits, total periods, the work counter, the
// fit and period offsets of every asteroid and its first period -- and the
// fit / record buffers.  A scan writes the control block into pinned host
// memory and replays a CUDA graph captured once per batch:
//   copy control block H2D -> persistent fit kernel (global work queue over
//   all asteroids' fits) -> best-of-poles reduction over all periods
// The graph reads every size from the control block, so the same graph
// serves any period ranges up to the capacity it was built for.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/period_search_b200.h"
#include "ps_ctx.hpp"
#include "ps_device.hpp"

struct ps_batch {
    int device = 0, form = PS_FORM_FP64, n = 0;
    std::vector<ps_ctx*> ctx;
    cudaStream_t stream = nullptr;
    psb::DevBuf<psb::DevProblem> d_probs;
    psb::DevBuf<int> d_ctl;
    psb::DevBuf<double> d_ndata;
    psb::DevBuf<double> d_scratch;
    psb::DevBuf<psb::FitOut> d_fits;
    psb::DevBuf<ps_record> d_rec;
    int* h_ctl = nullptr;  // pinned
    size_t ctl_ints = 0;
    long long stride = 0;
    int grid = 0;
    psb::DevProblem head{};  // the problem with the largest shared-memory layout
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t graph_fits = 0, graph_periods = 0;
    cudaStream_t last = nullptr;  // stream of the last replay
};

namespace {

// control block: [0] fits, [1] periods, [2] work counter,
// [3 .. 3+n] fit offsets, [4+n .. 3+2n] first periods, [4+2n .. 4+3n] period offsets,
// [5+3n .. 4+4n] queue order of the asteroids, [5+4n .. 5+5n] queue offsets in that order
int ctl_fit_off(int) { return 3; }
int ctl_n_from(int n) { return 4 + n; }
int ctl_per_off(int n) { return 4 + 2 * n; }
int ctl_order(int n) { return 5 + 3 * n; }
int ctl_ord_off(int n) { return 5 + 4 * n; }

#define PSB_BCUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return psb::set_error(PS_ERR_CUDA, std::string(#call) + ": " + \
                                                                      cudaGetErrorString(e_)); \
    } while (0)

size_t smem_of(const ps_batch* b, const psb::DevProblem& p) {
    if (b->form == PS_FORM_MIXED) return psb::mixed_smem_bytes(p);
    return b->form == PS_FORM_FAST ? psb::fast_smem_bytes(p) : psb::fp64_smem_bytes(p);
}

cudaError_t launch_fits(const ps_batch* b, const psb::FitBatch& fb) {
    if (b->form == PS_FORM_MIXED) return psb::launch_mixed_fits(b->head, b->d_probs.p, fb, b->grid, b->stream);
    if (b->form == PS_FORM_FAST) return psb::launch_fast_fits(b->head, b->d_probs.p, fb, b->grid, b->stream);
    return psb::launch_fp64_fits(b->head, b->d_probs.p, fb, b->grid, b->stream);
}

// The mixed form's bounded device waits report through each context's
// error flag (fits they ended carry status -1); read after a synchronisation.
int check_device_errors(ps_batch* b) {
    if (b->form != PS_FORM_MIXED) return PS_OK;
    for (int a = 0; a < b->n; a++) {
        const ps_ctx* c = b->ctx[a];
        if (!c->d_err.p) continue;
        int e = 0;
        PSB_BCUDA(cudaMemcpy(&e, c->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            PSB_BCUDA(cudaMemset(c->d_err.p, 0, sizeof(int)));
            return psb::set_error(PS_ERR_DEVICE_LOOP, "a device wait on the tensor-core pipeline gave up (" +
                                                          std::to_string(e) + "); the fits it ended carry status -1");
        }
    }
    return PS_OK;
}

void release_graph(ps_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_fits = b->graph_periods = 0;
}

int capture(ps_batch* b, size_t fits, size_t periods) {
    release_graph(b);
    PSB_BCUDA(b->d_fits.ensure(fits));
    PSB_BCUDA(b->d_rec.ensure(periods));
    int* ctl = b->d_ctl.p;
    psb::FitBatch fb{};
    fb.n_fits = 0;
    fb.n_fits_dev = ctl;
    fb.queue = ctl + 2;
    fb.out = b->d_fits.p;
    fb.scratch = b->d_scratch.p;
    fb.scratch_stride = b->stride;
    fb.n_ast = b->n;
    fb.ast_fit_off = ctl + ctl_fit_off(b->n);
    fb.ast_n_from = ctl + ctl_n_from(b->n);
    fb.ast_order = ctl + ctl_order(b->n);
    fb.ast_ord_off = ctl + ctl_ord_off(b->n);
    PSB_BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    cudaError_t e = cudaMemcpyAsync(ctl, b->h_ctl, b->ctl_ints * sizeof(int), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = launch_fits(b, fb);
    if (e == cudaSuccess)
        e = psb::launch_period_reduce_batch(b->d_fits.p, ctl + 1, (int)periods, b->n, ctl + ctl_per_off(b->n),
                                            b->d_ndata.p, b->d_rec.p, b->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return psb::set_error(PS_ERR_CUDA, std::string("graph capture: ") +
                                               cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    b->graph = g;
    PSB_BCUDA(cudaGraphInstantiate(&b->exec, g, 0));
    b->graph_fits = fits;
    b->graph_periods = periods;
    return PS_OK;
}

// Fill the control block and replay the graph; records land in d_rec.
int run(ps_batch* b, const int* n_from, const int* n_to, size_t* periods_out, cudaStream_t launch) {
    const int n = b->n;
    // the previous replay may still be reading the pinned control block
    PSB_BCUDA(cudaStreamSynchronize(b->stream));
    if (b->last && b->last != b->stream) PSB_BCUDA(cudaStreamSynchronize(b->last));
    size_t fits = 0, periods = 0;
    int* h = b->h_ctl;
    for (int a = 0; a < n; a++) {
        const int np = n_to[a] - n_from[a] + 1;
        if (n_from[a] < 1 || np < 1 || n_to[a] > b->ctx[a]->prob.n_periods())
            return psb::set_error(PS_ERR_ARG, "period range out of bounds for asteroid " + std::to_string(a));
        h[ctl_fit_off(n) + a] = (int)fits;
        h[ctl_per_off(n) + a] = (int)periods;
        h[ctl_n_from(n) + a] = n_from[a];
        fits += (size_t)np * 10;
        periods += (size_t)np;
    }
    if (fits > 0x7fffffff) return psb::set_error(PS_ERR_LIMIT, "too many fits in one batch scan");
    h[ctl_fit_off(n) + n] = (int)fits;
    h[ctl_per_off(n) + n] = (int)periods;
    // longest fits first (cost ~ points x fits), so that the persistent
    // kernel's last fits are short ones and the SMs finish together
    std::vector<int> order(n);
    for (int a = 0; a < n; a++) order[a] = a;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const double cx = (double)b->ctx[x]->prob.n_points * (n_to[x] - n_from[x] + 1);
        const double cy = (double)b->ctx[y]->prob.n_points * (n_to[y] - n_from[y] + 1);
        return cx > cy;
    });
    int q = 0;
    for (int k = 0; k < n; k++) {
        h[ctl_order(n) + k] = order[k];
        h[ctl_ord_off(n) + k] = q;
        q += 10 * (n_to[order[k]] - n_from[order[k]] + 1);
    }
    h[ctl_ord_off(n) + n] = q;
    h[0] = (int)fits;
    h[1] = (int)periods;
    h[2] = 0;
    if (!b->exec || fits > b->graph_fits || periods > b->graph_periods) {
        // keep (replayed) graphs for the largest size seen
        int rc = capture(b, std::max(fits, b->graph_fits), std::max(periods, b->graph_periods));
        if (rc) return rc;
    }
    PSB_BCUDA(cudaGraphLaunch(b->exec, launch));
    b->last = launch;
    psb::count_launch();
    psb::count_launch();
    *periods_out = periods;
    return PS_OK;
}

}  // namespace

extern "C" {

int ps_batch_open(ps_ctx* const* ctxs, int n, ps_batch** out) {
    if (!ctxs || n < 1 || !out) return psb::set_error(PS_ERR_ARG, "empty batch");
    *out = nullptr;
    ps_batch* b = new ps_batch();
    b->n = n;
    b->ctx.assign(ctxs, ctxs + n);
    const ps_ctx* c0 = ctxs[0];
    for (int a = 0; a < n; a++) {
        const ps_ctx* c = ctxs[a];
        std::string why;
        if (!c || c->host_only) why = "context without a device";
        else if (c->device != c0->device) why = "contexts on different devices";
        else if (c->form != c0->form) why = "contexts of different forms";
        else if (!c->rows_ready) why = "call ps_precalc or ps_set_conw_r on every context first";
        else if (c->dp.NCB != c0->dp.NCB || c->dp.F != c0->dp.F || c->dp.C != c0->dp.C || c->dp.ma != c0->dp.ma)
            why = "all asteroids of a batch need the same lmax, mmax and nrows";
        if (!why.empty()) {
            delete b;
            return psb::set_error(PS_ERR_ARG, why);
        }
    }
    b->device = c0->device;
    b->form = c0->form;
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    std::vector<psb::DevProblem> probs(n);
    std::vector<double> ndata(n);
    size_t best = 0;
    // Asteroids on the same facet grid (nrows, lmax, mmax) have identical
    // facet tables (normals, areas, Dsph, Legendre and Fourier factors);
    // their fits read one copy, which then stays in L2.
    std::vector<int> owners;
    for (int a = 0; a < n; a++) {
        probs[a] = ctxs[a]->dp;
        const psb::Problem& pa = ctxs[a]->prob;
        for (int o : owners) {
            const psb::Problem& po = ctxs[o]->prob;
            if (pa.lmax == po.lmax && pa.mmax == po.mmax && pa.nor == po.nor && pa.darea == po.darea &&
                pa.dsph == po.dsph && pa.pleg == po.pleg && pa.fc == po.fc && pa.fs == po.fs) {
                probs[a].fac = ctxs[o]->dp.fac;
                probs[a].fac32 = ctxs[o]->dp.fac32;
                probs[a].dsph = ctxs[o]->dp.dsph;
                probs[a].cpl = ctxs[o]->dp.cpl;
                probs[a].cfc = ctxs[o]->dp.cfc;
                probs[a].cfs = ctxs[o]->dp.cfs;
                break;
            }
        }
        if (probs[a].dsph == ctxs[a]->dp.dsph) owners.push_back(a);
        ndata[a] = ctxs[a]->dp.ndata_m3;
        b->stride = std::max(b->stride, b->form == PS_FORM_MIXED ? psb::mixed_scratch_doubles(ctxs[a]->dp)
                                                                 : (long long)(ctxs[a]->dp.ma + 1) * ctxs[a]->dp.npad);
        const size_t s = smem_of(b, probs[a]);
        if (s >= best) {
            best = s;
            b->head = probs[a];
        }
    }
    int threads = 0, sms = 0;
    const int per_sm = b->form == PS_FORM_MIXED  ? psb::mixed_max_blocks_per_sm(b->head, &threads)
                       : b->form == PS_FORM_FAST ? psb::fast_max_blocks_per_sm(b->head, &threads)
                                                 : psb::fp64_max_blocks_per_sm(b->head, &threads);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    b->grid = sms * per_sm;
    b->ctl_ints = (size_t)(6 + 5 * n);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_ctl, b->ctl_ints * sizeof(int));
    if (e == cudaSuccess) e = b->d_ctl.ensure(b->ctl_ints);
    if (e == cudaSuccess) e = b->d_probs.upload(probs, b->stream);
    if (e == cudaSuccess) e = b->d_ndata.upload(ndata, b->stream);
    if (e == cudaSuccess) e = b->d_scratch.ensure((size_t)b->stride * (b->grid > 0 ? b->grid : 1));
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess || b->grid <= 0) {
        ps_batch_close(b);
        return psb::set_error(e != cudaSuccess ? PS_ERR_CUDA : PS_ERR_LIMIT,
                              e != cudaSuccess ? cudaGetErrorString(e) : "fit kernel does not fit on the device");
    }
    *out = b;
    return PS_OK;
}

int ps_batch_scan_device(ps_batch* b, const int* n_from, const int* n_to, ps_record* d_out, void* stream) {
    if (!b || !n_from || !n_to || !d_out) return psb::set_error(PS_ERR_ARG, "null argument");
    PSB_BCUDA(cudaSetDevice(b->device));
    size_t periods = 0;
    cudaStream_t s = stream ? (cudaStream_t)stream : b->stream;
    int rc = run(b, n_from, n_to, &periods, s);
    if (rc) return rc;
    PSB_BCUDA(cudaMemcpyAsync(d_out, b->d_rec.p, periods * sizeof(ps_record), cudaMemcpyDeviceToDevice, s));
    return PS_OK;
}

int ps_batch_scan(ps_batch* b, const int* n_from, const int* n_to, ps_record* out) {
    if (!b || !n_from || !n_to || !out) return psb::set_error(PS_ERR_ARG, "null argument");
    PSB_BCUDA(cudaSetDevice(b->device));
    size_t periods = 0;
    int rc = run(b, n_from, n_to, &periods, b->stream);
    if (rc) return rc;
    PSB_BCUDA(cudaMemcpyAsync(out, b->d_rec.p, periods * sizeof(ps_record), cudaMemcpyDeviceToHost, b->stream));
    PSB_BCUDA(cudaStreamSynchronize(b->stream));
    return check_device_errors(b);
}

int ps_batch_fit_times(ps_batch* b, double* busy_ms, double* done_ms) {
    if (!b || !busy_ms || !done_ms) return psb::set_error(PS_ERR_ARG, "null argument");
    PSB_BCUDA(cudaSetDevice(b->device));
    PSB_BCUDA(cudaStreamSynchronize(b->stream));
    if (b->last) PSB_BCUDA(cudaStreamSynchronize(b->last));
    const int n = b->n;
    const size_t fits = (size_t)b->h_ctl[0];
    std::vector<psb::FitOut> f(fits);
    PSB_BCUDA(cudaMemcpy(f.data(), b->d_fits.p, fits * sizeof(psb::FitOut), cudaMemcpyDeviceToHost));
    // times relative to the first fit's end (32-bit microsecond stamps wrap
    // after 71 minutes; differences within a scan are well inside that)
    const unsigned int ref = fits ? f[0].end_us : 0;
    long long t0 = 0;  // the scan's first fit start
    for (size_t w = 0; w < fits; w++) {
        const long long start = (long long)(int)(f[w].end_us - ref) - (long long)f[w].dur_us;
        if (w == 0 || start < t0) t0 = start;
    }
    for (int a = 0; a < n; a++) {
        long long busy = 0, done = 0;
        for (int w = b->h_ctl[ctl_fit_off(n) + a]; w < b->h_ctl[ctl_fit_off(n) + a + 1]; w++) {
            busy += f[(size_t)w].dur_us;
            done = std::max(done, (long long)(int)(f[(size_t)w].end_us - ref) - t0);
        }
        busy_ms[a] = busy * 1e-3;
        done_ms[a] = done * 1e-3;
    }
    return PS_OK;
}

void ps_batch_close(ps_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->last) cudaStreamSynchronize(b->last);
    release_graph(b);
    b->d_probs.release();
    b->d_ctl.release();
    b->d_ndata.release();
    b->d_scratch.release();
    b->d_fits.release();
    b->d_rec.release();
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"

/* period_search_b200 — C ABI of the B200-native convex-inversion period scan.
 *
 * Drop-in for the GPU operator interface of the reference application
 * (ahorek/PeriodSearch, period_search_cuda/period_search/start_CUDA.h) and
 * for the scan loop of its CPU driver (period_search/period_search_BOINC.cpp).
 * Plain C types only: pointers, sizes, doubles and ints.  All arrays are
 * 0-based and dense, owned by the caller, and copied by the callee.
 *
 * Threading: a context (ps_ctx) belongs to one host thread at a time;
 * separate contexts are independent.  Errors are returned as status codes
 * (never exit()); ps_last_error() gives a message for the calling thread.
 */
#ifndef PERIOD_SEARCH_B200_H
#define PERIOD_SEARCH_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  PS_ERR_LIMIT (2) and PS_ERR_SINGULAR (4) carry the
 * reference's exit codes for the same conditions (period_search_BOINC.cpp
 * :326-327 etc. exit(2); ludcmp.c:23 exit(4)). */
enum {
    PS_OK = 0,
    PS_ERR_IO = 1,          /* input cannot be opened / output cannot be written */
    PS_ERR_LIMIT = 2,       /* malformed input or a size limit exceeded */
    PS_ERR_CUDA = 3,        /* CUDA runtime failure (message in ps_last_error) */
    PS_ERR_SINGULAR = 4,    /* singular ellipsoid-fit matrix (ludcmp) */
    PS_ERR_ARG = 5,         /* invalid argument */
    PS_ERR_DEVICE_LOOP = 6  /* a device loop hit its iteration guard: a bounded wait
                               of the tensor-core pipeline (PS_FORM_MIXED) gave up;
                               the fits it ended carry status -1 and the context
                               stays usable.  The environment variable
                               PS_B200_MAX_POLLS, read when a context opens,
                               sets that wait limit in polls (default 2^24; 0 makes
                               every such wait give up at once) */
};

/* Numerical form of the fit kernels. */
enum {
    PS_FORM_FP64 = 0, /* plain FP64, reference operation order (the drop-in) */
    PS_FORM_MIXED = 1, /* FP64 model/chi2/beta/solve, FP32 derivatives, shape block
                          of the Jacobian (split BF16) and alpha (split TF32) on
                          the tensor cores */
    PS_FORM_FAST = 2   /* FP64 throughout, derivative work rearranged and fused
                          (rounding-level differences to PS_FORM_FP64) */
};

/* One output record per trial period, the six values the reference prints
 * (period_search_BOINC.cpp:926-931), unrounded. */
typedef struct {
    double period_h;   /* 24 * best period [h] */
    double rms;        /* dev_best */
    double chi2;       /* dev_best^2 * (ndata - 3) */
    double dark_pct;   /* dark-facet percentage of the best pole */
    double lambda_deg; /* best pole longitude in [0, 360) */
    double beta_deg;   /* best pole latitude */
} ps_record;

/* One LM fit (one trial period, one initial pole). */
typedef struct {
    double dev;       /* final rms deviation */
    double dark;      /* |sum Area*Nor| of the accepted shape */
    double totarea;   /* sum of the last evaluated facet areas */
    double period_d;  /* 2 pi / omega [day] */
    double lambda_deg;
    double beta_deg;
    double chisq;
    int niter;
    int status;       /* 0, or the gauss_errc code that froze the fit */
} ps_fit_result;

/* Problem as the reference's host has it after parsing period_search_in
 * (period_search_BOINC.cpp:277-485), i.e. what CUDAPrepare/CUDAPrecalc/
 * CUDAStart receive plus the globals they read (l_curves, l_points, in_rel,
 * weight, l_max, m_max; period_search_cuda/.../period_search_BOINC.cpp
 * :141-155).  Vectors are already normalised, times already have jd_0
 * subtracted, sig is the per-lightcurve mean brightness. */
typedef struct {
    int n_points;            /* real data points (no convexity rows) */
    int n_lc;                /* lightcurves (no convexity pseudo-curve) */
    const int* lc_points;    /* [n_lc] points per lightcurve */
    const int* lc_relative;  /* [n_lc] 1 = relative (Inrel), 0 = calibrated */
    const double* tim;       /* [n_points] JD - jd_0 [day] */
    const double* ee;        /* [n_points*3] unit asteroid->Earth */
    const double* ee0;       /* [n_points*3] unit asteroid->Sun */
    const double* brightness;/* [n_points] */
    const double* sig;       /* [n_points] */
    const double* weight;    /* [n_points] */
    double per_start, per_step_coef, per_end; /* header line 1 */
    int ia_prd;
    double phi0_rad;         /* initial rotation angle [rad] */
    double conw;             /* convexity weight as given */
    int lmax, mmax, nrows;
    double par[3];           /* phase function a, d, k */
    int ia_par[3];
    double cl;               /* initial Lambert coefficient */
    int ia_cl;
    double stop_condition;
    int n_iter_min;
    double alamda_incr, alamda_start;
    double jd_min, jd_max;   /* data span (frequency step rule) */
    double escl;             /* initial size scale (shape guess) */
} ps_problem_desc;

typedef struct ps_ctx ps_ctx;

/* Parse a period_search_in file and do the host setup of the reference
 * (period_search_BOINC.cpp:277-485), then open a context on CUDA device
 * `device` (replaces the parse + CUDAPrepare, start_CUDA.h:2-4). */
int ps_open_file(const char* path, int device, int form, ps_ctx** out);
/* Same from in-memory arrays (replaces CUDAPrepare + the host globals). */
int ps_open(const ps_problem_desc* desc, int device, int form, ps_ctx** out);
/* Release the context (replaces CUDAUnprepare, start_CUDA.h:14).  Its
 * device buffers go back to a per-device cache (at most 512 buffers and
 * 4 GiB per device) from which later contexts and batches draw, so that
 * opening and closing a context per asteroid does not call cudaMalloc and
 * the device-synchronising cudaFree every time. */
void ps_close(ps_ctx* ctx);
/* Free the cached device buffers of every device.  No counterpart in the
 * reference (its buffers are static arrays). */
void ps_release_cached_memory(void);

/* Convexity-weight optimisation pre-pass (replaces CUDAPrecalc,
 * start_CUDA.h:9-10; period_search_BOINC.cpp:487-715), then the final setup
 * (:719-802).  Writes the resulting conw_r. */
int ps_precalc(ps_ctx* ctx, double* conw_r);
/* Resume path: use a conw_r from a checkpoint and skip the pre-pass
 * (period_search_cuda/.../period_search_BOINC.cpp:616-629). */
int ps_set_conw_r(ps_ctx* ctx, double conw_r);
/* Trial-period count, (int)((f_start - f_end)/f_step) + 1
 * (period_search_BOINC.cpp:807). */
int ps_n_periods(const ps_ctx* ctx);
/* Scan trial periods n_from..n_to (1-based, inclusive) and write one record
 * each to host memory (replaces CUDAStart, start_CUDA.h:6-7; the caller
 * formats the lines).  Requires ps_precalc or ps_set_conw_r first. */
int ps_scan(ps_ctx* ctx, int n_from, int n_to, ps_record* out);
/* Same, but the records stay on the device: d_out is a device pointer to
 * (n_to - n_from + 1) records; stream is a cudaStream_t (NULL = the
 * context's own stream, not the legacy default stream); asynchronous.  The
 * context's tables are complete on the device when ps_open* and
 * ps_precalc / ps_set_conw_r return, so any stream may scan afterwards.
 * Scans of one context share its work buffers: scans on different streams
 * must not overlap on the GPU.  ps_close waits for the last scan launched on
 * a caller's stream before it releases the context. */
int ps_scan_device(ps_ctx* ctx, int n_from, int n_to, ps_record* d_out, void* stream);

/* ps_scan_device without any device-memory allocation.  No counterpart in
 * the reference.  It is for callers that cannot allocate device memory while
 * they scan: a host that gives this library a fixed device-memory budget up
 * front, a plugin running inside a process whose allocator it does not own,
 * or a latency-sensitive service for which cudaMalloc/cudaFree are not
 * acceptable on the scan path (cudaFree waits for the whole device).  Set the
 * context up first (ps_open*, then ps_precalc or ps_set_conw_r, which
 * allocate the per-asteroid tables); this call then takes all scratch from
 * one 64 MiB device array that the library holds on every GPU it runs on
 * until exit, and rejects, with PS_ERR_LIMIT, a period range whose 72 bytes
 * per fit plus one CTA's Jacobian scratch do not fit in it.  Asynchronous on
 * `stream` (NULL = the context's stream).  All calls share the array and it
 * keeps the last call's contents: calls that overlap on the GPU race, so
 * serialise them.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture begins.  FP64 form only; that form has no bounded
 * device wait, so there is no device error word to check afterwards. */
int ps_scan_device_noalloc(ps_ctx* ctx, int n_from, int n_to, ps_record* d_out, void* stream);

/* Batched scans: many asteroids in one persistent launch, each fit pulling
 * from one device work queue (uneven point counts and per-fit LM
 * convergence do not stall one another), the steady state replayed from a
 * CUDA graph.  The reference runs one asteroid per process and, in its CUDA
 * port, one thread block per trial period of that asteroid
 * (period_search_cuda/period_search/start_CUDA.cu:654-776); a batch spans
 * asteroids.  The contexts must share the device, the form and lmax, mmax,
 * nrows, and have conw_r settled (ps_precalc / ps_set_conw_r).  The batch
 * borrows the contexts' tables: close the batch before its contexts.  In
 * the mixed form ps_batch_scan reports a bounded device wait that gave up
 * as PS_ERR_DEVICE_LOOP (the fits it ended carry status -1); the
 * asynchronous ps_batch_scan_device leaves that report to the next
 * ps_batch_scan. */
typedef struct ps_batch ps_batch;
int ps_batch_open(ps_ctx* const* ctxs, int n, ps_batch** out);
/* Scan periods n_from[a]..n_to[a] of every asteroid a; records are
 * concatenated in asteroid order (host memory). */
int ps_batch_scan(ps_batch* batch, const int* n_from, const int* n_to, ps_record* out);
/* Same into device memory, launched on `stream` (NULL = the batch's own
 * stream); asynchronous. */
int ps_batch_scan_device(ps_batch* batch, const int* n_from, const int* n_to, ps_record* d_out, void* stream);
/* Per asteroid of the last scan: busy_ms, the time its fits ran (summed
 * over its fits, each on its own CTA), and done_ms, the wall time from the
 * start of the scan's first fit to the end of the asteroid's last fit (its
 * latency inside the batch); from the GPU's global timer. */
int ps_batch_fit_times(ps_batch* batch, double* busy_ms, double* done_ms);
void ps_batch_close(ps_batch* batch);

/* One LM fit at trial frequency freq [1/day] from initial pole m (1..10)
 * (period_search_BOINC.cpp:817-920).  cg_out (may be NULL) receives the
 * final parameter vector (ma values). */
int ps_fit(ps_ctx* ctx, double freq, int pole, ps_fit_result* out, double* cg_out);
/* One model evaluation, the reference's mrqcof (mrqcof.c:16-148) at
 * parameter vector a (ma values): alpha [mfit*mfit], beta [mfit], chi2. */
int ps_mrqcof(ps_ctx* ctx, const double* a, double* alpha, double* beta, double* chisq);
/* Model rows after the relative-lightcurve normalisation:
 * ymod [n_points+3], dyda [(n_points+3)*ma] (row-major). */
int ps_model(ps_ctx* ctx, const double* a, double* ymod, double* dyda);

/* Sizes: [0] n_points, [1] n_lc (incl. convexity pseudo-curve),
 * [2] numfac, [3] ncoef, [4] ma, [5] mfit, [6] n_periods, [7] fits run by
 * the last ps_precalc (10 poles x up to 10 periods per pre-pass round).
 * Scalars: [0] escl, [1] conw_r, [2] freq_start, [3] freq_end,
 * [4] freq_step. */
int ps_info(const ps_ctx* ctx, int* ints, double* dbls);
/* Copy a host-setup array out (names as the oracle's pso_get_array:
 * "nor", "darea", "dsph", "cg_first", "ia", "tim", "ee", "ee0",
 * "brightness", "sig", "weight", "at", "af", "ifp").  Returns the element
 * count or -1. */
int ps_get_array(const ps_ctx* ctx, const char* name, double* out);

/* Parse + host setup only, no device: for host-side tests on machines
 * without a GPU.  The handle supports ps_info/ps_get_array/ps_close. */
int ps_open_host_only(const char* path, ps_ctx** out);

/* Format one record exactly as the reference prints it
 * ("%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n", period_search_BOINC.cpp:926-931);
 * when first_line is nonzero column 4 is conw_line instead of dark_pct.
 * Returns the number of characters written (excluding the NUL). */
int ps_format_record(const ps_record* r, int first_line, double conw_line, char* buf, int buflen);

/* Tile shapes: facets per staged chunk (fch, multiple of 4, 4..128) and
 * alpha rows per tile (rt, multiple of 4, 4..256) of the fast form, and the
 * number of points sorted together by viewing direction (sortseg, a power
 * of 2, 32..4096) in both FP64 forms.  No choice changes any result (the
 * sums keep their order); they change speed and shared memory.  Defaults
 * 40, 32, 1024.  PS_ERR_LIMIT if the layout does not fit.  No counterpart
 * in the reference (fixed array sizes there).
 * ps_autotune: time scans of trial periods 1..n (n = n_periods, at least
 * two waves of fits: 4 x SMs / 10 periods) under candidate
 * tiles (fch in {16, 32, 40, 48, 56, 64}, rt in {16, 32, 64}; sortseg in {256, 1024}; the
 * reference-order form only sortseg), keep the fastest; tiles[3] and
 * *seconds (its scan time) receive the choice. */
int ps_set_tiles(ps_ctx* ctx, int fch, int rt, int sortseg);
int ps_autotune(ps_ctx* ctx, int n_periods, int* tiles, double* seconds);

/* Matrix-free derivatives at parameters a[ma] (the adjoint form).  No
 * Jacobian is formed: one pass over the (point, facet) pairs evaluates the
 * model and the forward product, a second (thread per facet) applies J^T,
 * so a call costs O(N F + F C) instead of the N F C of mrqcof's explicit
 * dyda rows (mrqcof.c:16-148), with the same relative-lightcurve
 * normalisation and convexity rows.  FP64, fused arithmetic (the fast form's
 * rounding); deterministic.
 *
 * ps_chi2_grad: *chi2 and beta[mfit] = J^T W (y_obs - y) over the free
 * parameters, i.e. the chi2 gradient is -2 beta.  Replaces the beta/chisq
 * half of the reference's mrqcof (mrqcof.c:106-147) for callers that only
 * need the gradient.
 * ps_gn_product: out[mfit] = J^T W (J v) for v[mfit] over the free
 * parameters -- alpha v with alpha from ps_mrqcof, up to rounding.  No
 * counterpart in the reference (it forms alpha explicitly). */
int ps_chi2_grad(ps_ctx* ctx, const double* a, double* chi2, double* beta);
int ps_gn_product(ps_ctx* ctx, const double* a, const double* v, double* out);
/* One LM fit as ps_fit (period_search_BOINC.cpp:817-920; mrqmin.c:11-110
 * with gauss_errc's full pivoting), Jacobian-free: every model evaluation
 * runs the matrix-free kernels, alpha column by column from mfit
 * Gauss-Newton products with the free unit vectors, beta and chi2 from the
 * gradient pass, the trial points from the gradient pass alone, and the
 * solve on the host in FP64.  J is never formed (for shapes whose N x ma
 * Jacobian would not fit); each accepted step costs mfit + 1 matrix-free
 * passes over the whole GPU, so for shapes whose J fits, ps_fit and the
 * scans are far faster.  Same outputs as ps_fit, up to rounding. */
int ps_fit_jfree(ps_ctx* ctx, double freq, int pole, ps_fit_result* out, double* cg_out);

/* Message for the last error on the calling thread ("" if none). */
const char* ps_last_error(void);
/* Kernel launches issued by this process so far (all contexts). */
long long ps_kernel_launches(void);

/* Measured FP64 tensor-core throughput of `device` in TFLOP/s (m8n8k4 FP64
 * MMAs from registers on every SM, best of three ~0.1 s runs): the roofline
 * denominator for the FP64 forms.  No counterpart in the reference. */
int ps_fp64_tensor_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif

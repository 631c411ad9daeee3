/* CPU oracle for the period_search convex-inversion fit path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * CPU application (period_search/, ahorek/PeriodSearch) used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * The product (periodsearch_b200) never links, imports or calls it.
 *
 * Pinning: the restatement is compared bit-for-bit against the reference
 * itself, compiled in place from its own sources (oracle/Makefile, target
 * `ref`), on the reference's shipped input and on seeded synthetic inputs;
 * and against the reference's shipped golden output period_search_out and
 * the golden arrays of its unit tests (tests/golden/).
 *
 * Indexing: arrays passed across this API are 0-based and dense.
 */
#ifndef PS_ORACLE_H
#define PS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pso_problem pso_problem;

/* Per-period record, in the units the reference prints
 * (period_search_BOINC.cpp:926-931): period [h], rms, chi2 = rms^2 (ndata-3),
 * dark-facet [%], lambda [deg], beta [deg].  dark is always the dark-facet
 * value; the writer substitutes conw_r*escl^2 on the first line. */
typedef struct {
    double period_h, rms, chi2, dark, lambda_deg, beta_deg;
} pso_record;

/* Parse period_search_in and do everything the reference does before the
 * convexity-weight pre-pass (period_search_BOINC.cpp:277-485).  Returns NULL
 * and sets *status (2 = limit exceeded / malformed, -1 = cannot open). */
pso_problem* pso_load(const char* path, int* status);
void pso_free(pso_problem* p);

/* Convexity-weight optimisation pre-pass (period_search_BOINC.cpp:487-715)
 * followed by the final setup (:719-802).  Writes conw_r. */
int pso_prepass(pso_problem* p, double* conw_r);
/* Skip the pre-pass with a known conw_r (the value the pre-pass produced),
 * performing only the final setup (:719-802). */
int pso_set_conw_r(pso_problem* p, double conw_r);

/* Number of trial periods of the scan (period_search_BOINC.cpp:807). */
int pso_n_periods(const pso_problem* p);
/* Scan trial periods n_from..n_to (1-based, inclusive), one record each
 * (period_search_BOINC.cpp:807-945). */
int pso_scan(pso_problem* p, int n_from, int n_to, pso_record* out);

/* One LM fit at trial frequency freq [1/day] from initial pole m (1..10)
 * (period_search_BOINC.cpp:817-920).  out[0..8] = dev, dark (|chck|),
 * totarea, prd [day], lambda [deg], beta [deg], chisq, niter, alamda, status
 * (the first gauss_errc code of the fit, 0 if none; out has 10 slots);
 * cg_out (may be NULL) receives the final parameter vector (ma values). */
int pso_fit(pso_problem* p, double freq, int m, double* out, double* cg_out);

/* One model evaluation, mrqcof (mrqcof.c:16-148) at parameter vector a
 * (ma values).  alpha: mfit*mfit (symmetrised), beta: mfit.  Returns chi2. */
double pso_mrqcof(pso_problem* p, const double* a, double* alpha, double* beta);
/* The model and its derivatives for every row: ymod[ndata+3],
 * dyda[(ndata+3)*ma] after the relative-lightcurve normalisation. */
int pso_model(pso_problem* p, const double* a, double* ymod, double* dyda);

/* Gauss-Jordan elimination with full pivoting on a 0-based n x n matrix
 * (gauss_errc.c:9-73).  Returns 0, 1 or 2 like the reference. */
int pso_gauss_errc(double* a, int n, double* b);

/* Integer facts: [0] ndata (real points), [1] lcurves (incl. convexity
 * pseudo-curve), [2] numfac, [3] ncoef, [4] ma, [5] mfit, [6] n_periods,
 * [7] lmax, [8] mmax, [9] nrows, [10] onlyrel, [11] n_iter_min,
 * [12] ia_prd, [13] ia_cl.
 * Double facts: [0] escl, [1] conw_r, [2] freq_start, [3] freq_end,
 * [4] freq_step, [5] jd_0, [6] phi0 [rad], [7] alamda_start,
 * [8] alamda_incr, [9] stop_condition, [10] jd_min, [11] jd_max, [12] cl,
 * [13..15] par[1..3]. */
int pso_info(const pso_problem* p, int* ints, double* dbls);

/* Copy a named array out (0-based, dense).  Names: "nor" (F*3), "darea" (F),
 * "dsph" (F*C), "pleg" (F*(L+1)*(L+1), [f][l][m]), "fc" (F*(M+1)),
 * "fs" (F*(M+1)), "cg_first" (C), "ia" (ma), "tim" (N), "ee" (N*3),
 * "ee0" (N*3), "brightness" (N+3), "sig" (N+3), "weight" (N+3),
 * "lpoints" (lcurves), "inrel" (lcurves), "at" (F), "af" (F),
 * "ifp" (F*3), "alpha_phase" (N: acos(ee.ee0) per point).
 * Returns the element count, or -1 for an unknown name. */
int pso_get_array(const pso_problem* p, const char* name, double* out);

/* Geometry only (no data): the triangulated sphere of nrows rows, the
 * Laplace-series tables and the ellipsoid fit for axes a, b, c
 * (period_search_BOINC.cpp:729-782).  For the unit golden vectors. */
pso_problem* pso_geometry(int lmax, int mmax, int nrows, double a, double b, double c);
/* curv.c:10-38 at shape coefficients cg (ncoef values): area [F], dg [F*C]. */
void pso_curv(pso_problem* p, const double* cg, double* area, double* dg);

/* Stand-alone CLI entry: run the whole application in directory dir
 * (reads period_search_in, writes period_search_out and
 * period_search_out.full; honours period_search_state). */
int pso_run_app(const char* dir, int n_from, int n_to, double conw_r_given);

#ifdef __cplusplus
}
#endif
#endif

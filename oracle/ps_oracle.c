/* CPU oracle: plain-C restatement of the reference period_search fit path.
 *
 * TEST INFRASTRUCTURE ONLY -- used by tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / reference legs as the checker; the product
 * (periodsearch_b200) never links or calls it.
 *
 * Every routine follows the reference CPU application (ahorek/PeriodSearch,
 * directory period_search/) statement by statement, in the same arithmetic
 * order, so that when compiled with the same flags as the reference build
 * (-O3, no FMA contraction) it reproduces the reference bit for bit.  The
 * reference's process-global state (globals.h) becomes fields of
 * pso_problem; its 1-based arrays stay 1-based here so that every index can
 * be checked against the cited line.  Unlike the reference there are no
 * compile-time size limits (constants.h:1-7): arrays are sized from the
 * input, so large synthetic configurations run unchanged.
 *
 * Parity: pinned bit-exact against the reference compiled in place
 * (oracle/Makefile `ref`), see tests/test_oracle_pin.py.
 */
#include "ps_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PSO_PI M_PI                 /* constants.h:13 */
#define PSO_DEG2RAD (PSO_PI / 180)  /* constants.h:17 */
#define PSO_RAD2DEG (180 / PSO_PI)  /* constants.h:18 */
#define PSO_TINY 1e-8               /* constants.h:10 (mu, mu0 threshold) */
#define PSO_MAX_LM 10               /* constants.h:8 */
#define PSO_MAX_N_ITER 100          /* constants.h:6 */
#define PSO_N_POLES 10              /* constants.h:11 */
#define LM1 (PSO_MAX_LM + 1)

/* Perturbed builds for the chaotic-period triage (oracle/Makefile targets
   libps_oracle_sq.so / libps_oracle_fma.so / ps_oracle_sq / ps_oracle_fma):
   PSO_SQUARE_BY_MUL replaces pow(x, 2) on the fit path by x*x (it differs
   from glibc's pow in ~0.1 % of calls by one ulp).  The default build uses
   pow exactly like the reference. */
#ifdef PSO_SQUARE_BY_MUL
static double sq2(double x) { return x * x; }
#define PSO_SQ(x) sq2(x)
#else
#define PSO_SQ(x) pow((x), 2)
#endif

struct pso_problem {
    /* input header, period_search_BOINC.cpp:277-303 */
    double per_start, per_step_coef, per_end;
    int ia_prd;
    double jd_00, phi0, conw;
    int lmax, mmax, nrows;
    double par[4];
    int ia_par[4];
    double cl;
    int ia_cl;
    double stop_condition;
    int n_iter_min;
    double alamda_incr, alamda_start;
    /* lightcurves, :324-427 */
    int lcurves; /* incl. the convexity pseudo-curve once prepared */
    int *lpoints, *inrel;
    int ndata; /* real points */
    int ndata_tot; /* real points + 3 convexity rows */
    double *tim, *ee, *ee0; /* tim[1..N]; ee[np*4+k] k=1..3 */
    double *brightness, *sig, *weight; /* [1..N+3] */
    double jd_min, jd_max, jd_0, escl, conw_r;
    double a_axis, b_axis, c_axis;
    int onlyrel;
    /* geometry, :729-782 */
    int numfac, ndir, ncoef, nphpar, ma, mfit;
    double *t, *f, *at, *af;
    int* ifp; /* ifp[i*4+j] */
    double *nor, *darea, *fc, *fs, *tc, *ts, *pleg, *dsph;
    double* cg_first;
    int* ia;
    double freq_start, freq_end, freq_step;
    int geometry_ready;
    /* evaluation workspace (curv / bright / mrqcof) */
    double *area, *dg, *g;
    double blmat[4][4], dblm[3][4][4];
    double scale;
    int max_lpoints;
    double *ytemp, *dytemp, *dyda, *dave;
    int* incl;
    double *mu, *mu0, *s, *dbr, *dsmu, *dsmu0;
    /* LM state: the reference keeps these process-global (globals.h:5-6,
       mrqmin.c:17-19) and they carry from one fit to the next */
    double ochisq, chisq, alamda;
    int niter, lm_status;
    double *atry, *lm_beta, *da, *covar, *alpha, *cg;
};

/* index helpers (1-based, mirroring the reference's array shapes) */
#define NOR(p, i, j) ((p)->nor[(i)*4 + (j)])
#define PLEG(p, i, l, m) ((p)->pleg[((size_t)(i)*LM1 + (l)) * LM1 + (m)])
#define FC(p, i, m) ((p)->fc[(size_t)(i)*LM1 + (m)])
#define FS(p, i, m) ((p)->fs[(size_t)(i)*LM1 + (m)])
#define TC(p, i, m) ((p)->tc[(size_t)(i)*LM1 + (m)])
#define TS(p, i, m) ((p)->ts[(size_t)(i)*LM1 + (m)])
#define DSPH(p, i, k) ((p)->dsph[(size_t)(i) * ((p)->ncoef + 1) + (k)])
#define DG(p, i, k) ((p)->dg[(size_t)(i) * ((p)->ncoef + 1) + (k)])
#define MAT(m, n1, j, k) ((m)[(size_t)(j) * ((n1)) + (k)])

static void* xcalloc(size_t n, size_t sz) {
    void* q = calloc(n ? n : 1, sz);
    if (!q) {
        fprintf(stderr, "ps_oracle: out of memory\n");
        exit(3);
    }
    return q;
}

/* ---------------------------------------------------------------- setup */

/* trifac.c:10-82: vertex triplets of the standard triangulation. */
static void trifac(int nrows, int* ifp) {
    int rows = 2 * nrows + 1, cols = 4 * nrows + 1;
    int* nod = (int*)xcalloc((size_t)rows * cols, sizeof(int));
#define NOD(i, j) nod[(i)*cols + (j)]
    int nnod = 1, i, j, j0, j1, j2, j3, ntri;
    NOD(0, 0) = nnod;
    for (i = 1; i <= nrows; i++)
        for (j = 0; j <= 4 * i - 1; j++) {
            nnod++;
            NOD(i, j) = nnod;
            if (j == 0) NOD(i, 4 * i) = nnod;
        }
    for (i = nrows - 1; i >= 1; i--)
        for (j = 0; j <= 4 * i - 1; j++) {
            nnod++;
            NOD(2 * nrows - i, j) = nnod;
            if (j == 0) NOD(2 * nrows - i, 4 * i) = nnod;
        }
    NOD(2 * nrows, 0) = nnod + 1;
    ntri = 0;
    for (j1 = 1; j1 <= nrows; j1++)
        for (j3 = 1; j3 <= 4; j3++) {
            j0 = (j3 - 1) * j1;
            ntri++;
            ifp[ntri * 4 + 1] = NOD(j1 - 1, j0 - (j3 - 1));
            ifp[ntri * 4 + 2] = NOD(j1, j0);
            ifp[ntri * 4 + 3] = NOD(j1, j0 + 1);
            for (j2 = j0 + 1; j2 <= j0 + j1 - 1; j2++) {
                ntri++;
                ifp[ntri * 4 + 1] = NOD(j1, j2);
                ifp[ntri * 4 + 2] = NOD(j1 - 1, j2 - (j3 - 1));
                ifp[ntri * 4 + 3] = NOD(j1 - 1, j2 - 1 - (j3 - 1));
                ntri++;
                ifp[ntri * 4 + 1] = NOD(j1 - 1, j2 - (j3 - 1));
                ifp[ntri * 4 + 2] = NOD(j1, j2);
                ifp[ntri * 4 + 3] = NOD(j1, j2 + 1);
            }
        }
    for (j1 = nrows + 1; j1 <= 2 * nrows; j1++)
        for (j3 = 1; j3 <= 4; j3++) {
            j0 = (j3 - 1) * (2 * nrows - j1);
            ntri++;
            ifp[ntri * 4 + 1] = NOD(j1, j0);
            ifp[ntri * 4 + 2] = NOD(j1 - 1, j0 + 1 + (j3 - 1));
            ifp[ntri * 4 + 3] = NOD(j1 - 1, j0 + (j3 - 1));
            for (j2 = j0 + 1; j2 <= j0 + (2 * nrows - j1); j2++) {
                ntri++;
                ifp[ntri * 4 + 1] = NOD(j1, j2);
                ifp[ntri * 4 + 2] = NOD(j1 - 1, j2 + (j3 - 1));
                ifp[ntri * 4 + 3] = NOD(j1, j2 - 1);
                ntri++;
                ifp[ntri * 4 + 1] = NOD(j1, j2);
                ifp[ntri * 4 + 2] = NOD(j1 - 1, j2 + 1 + (j3 - 1));
                ifp[ntri * 4 + 3] = NOD(j1 - 1, j2 + (j3 - 1));
            }
        }
#undef NOD
    free(nod);
}

/* areanorm.c:10-60: unit-sphere facet areas, normals and normal angles. */
static void areanorm(pso_problem* p) {
    int ndir = p->ndir, nfac = p->numfac, i, j;
    double st, clen2, clen, c[4], vx[4], vy[4], vz[4];
    double* x = (double*)xcalloc(ndir + 1, sizeof(double));
    double* y = (double*)xcalloc(ndir + 1, sizeof(double));
    double* z = (double*)xcalloc(ndir + 1, sizeof(double));
    for (i = 1; i <= ndir; i++) {
        st = sin(p->t[i]);
        x[i] = st * cos(p->f[i]);
        y[i] = st * sin(p->f[i]);
        z[i] = cos(p->t[i]);
    }
    for (i = 1; i <= nfac; i++) {
        const int* v = &p->ifp[i * 4];
        for (j = 2; j <= 3; j++) {
            vx[j] = x[v[j]] - x[v[1]];
            vy[j] = y[v[j]] - y[v[1]];
            vz[j] = z[v[j]] - z[v[1]];
        }
        c[1] = vy[2] * vz[3] - vy[3] * vz[2];
        c[2] = vz[2] * vx[3] - vz[3] * vx[2];
        c[3] = vx[2] * vy[3] - vx[3] * vy[2];
        clen2 = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
        clen = sqrt(clen2);
        NOR(p, i, 1) = c[1] / clen;
        NOR(p, i, 2) = c[2] / clen;
        NOR(p, i, 3) = c[3] / clen;
        p->at[i] = acos(NOR(p, i, 3));
        p->af[i] = atan2(NOR(p, i, 2), NOR(p, i, 1));
        p->darea[i] = 0.5 * clen;
    }
    free(x);
    free(y);
    free(z);
}

/* sphfunc.c:11-87: unnormalised associated Legendre functions and the
   spherical-harmonic basis Dsph at every facet normal. */
static void sphfunc(pso_problem* p) {
    int ndir = p->numfac, Lmax = p->lmax, Mmax = p->mmax;
    int i, j, m, l, n, k, ibot;
    static double aleg[LM1][LM1][LM1];
    for (i = 1; i <= ndir; i++) {
        TS(p, i, 0) = 1;
        TC(p, i, 0) = 1;
        TS(p, i, 1) = sin(p->at[i]);
        TC(p, i, 1) = cos(p->at[i]);
        for (j = 2; j <= Lmax; j++) {
            TS(p, i, j) = TS(p, i, 1) * TS(p, i, j - 1);
            TC(p, i, j) = TC(p, i, 1) * TC(p, i, j - 1);
        }
        FS(p, i, 0) = 0;
        FC(p, i, 0) = 1;
        for (j = 1; j <= Mmax; j++) {
            FS(p, i, j) = sin(j * p->af[i]);
            FC(p, i, j) = cos(j * p->af[i]);
        }
    }
    for (m = 0; m <= Lmax; m++)
        for (l = 0; l <= Lmax; l++)
            for (n = 0; n <= Lmax; n++) aleg[n][l][m] = 0;
    aleg[0][0][0] = 1;
    aleg[1][1][0] = 1;
    for (l = 1; l <= Lmax; l++) aleg[0][l][l] = aleg[0][l - 1][l - 1] * (2 * l - 1);
    for (m = 0; m <= Mmax; m++)
        for (l = m + 1; l <= Lmax; l++) {
            if ((2 * ((l - m) / 2)) == (l - m)) {
                aleg[0][l][m] = -(l + m - 1) * aleg[0][l - 2][m] / (1 * (l - m));
                ibot = 2;
            } else
                ibot = 1;
            if (l != 1)
                for (n = ibot; n <= l - m; n = n + 2)
                    aleg[n][l][m] = ((2 * l - 1) * aleg[n - 1][l - 1][m] - (l + m - 1) * aleg[n][l - 2][m]) / (1 * (l - m));
        }
    for (i = 1; i <= ndir; i++) {
        k = 0;
        for (m = 0; m <= Mmax; m++)
            for (l = m; l <= Lmax; l++) {
                PLEG(p, i, l, m) = 0;
                if ((2 * ((l - m) / 2)) == (l - m))
                    ibot = 0;
                else
                    ibot = 1;
                for (n = ibot; n <= l - m; n = n + 2)
                    PLEG(p, i, l, m) = PLEG(p, i, l, m) + aleg[n][l][m] * TC(p, i, n) * TS(p, i, m);
                k++;
                DSPH(p, i, k) = FC(p, i, m) * PLEG(p, i, l, m);
                if (m != 0) {
                    k++;
                    DSPH(p, i, k) = FS(p, i, m) * PLEG(p, i, l, m);
                }
            }
    }
}

/* ludcmp.c:9-68 (Numerical Recipes LU with implicit pivoting); returns 4 on
   a singular matrix where the reference calls exit(4). */
static int ludcmp(double* a, int n, int* indx, double* d) {
    int i, imax = -999, j, k, n1 = n + 1;
    double big, dum, sum, temp;
    double* v = (double*)xcalloc(n + 1, sizeof(double));
    *d = 1.0;
    for (i = 1; i <= n; i++) {
        big = 0.0;
        for (j = 1; j <= n; j++)
            if ((temp = fabs(MAT(a, n1, i, j))) > big) big = temp;
        if (big == 0.0) {
            free(v);
            return 4;
        }
        v[i] = 1.0 / big;
    }
    for (j = 1; j <= n; j++) {
        for (i = 1; i < j; i++) {
            sum = MAT(a, n1, i, j);
            for (k = 1; k < i; k++) sum -= MAT(a, n1, i, k) * MAT(a, n1, k, j);
            MAT(a, n1, i, j) = sum;
        }
        big = 0.0;
        for (i = j; i <= n; i++) {
            sum = MAT(a, n1, i, j);
            for (k = 1; k < j; k++) sum -= MAT(a, n1, i, k) * MAT(a, n1, k, j);
            MAT(a, n1, i, j) = sum;
            if ((dum = v[i] * fabs(sum)) >= big) {
                big = dum;
                imax = i;
            }
        }
        if (j != imax) {
            for (k = 1; k <= n; k++) {
                dum = MAT(a, n1, imax, k);
                MAT(a, n1, imax, k) = MAT(a, n1, j, k);
                MAT(a, n1, j, k) = dum;
            }
            *d = -(*d);
            v[imax] = v[j];
        }
        indx[j] = imax;
        if (MAT(a, n1, j, j) == 0.0) MAT(a, n1, j, j) = 1.0e-20;
        if (j != n) {
            dum = 1.0 / (MAT(a, n1, j, j));
            for (i = j + 1; i <= n; i++) MAT(a, n1, i, j) *= dum;
        }
    }
    free(v);
    return 0;
}

/* lubksb.c:3-24 */
static void lubksb(const double* a, int n, const int* indx, double* b) {
    int i, ii = 0, ip, j, n1 = n + 1;
    double sum;
    for (i = 1; i <= n; i++) {
        ip = indx[i];
        sum = b[ip];
        b[ip] = b[i];
        if (ii)
            for (j = ii; j <= i - 1; j++) sum -= MAT(a, n1, i, j) * b[j];
        else if (sum)
            ii = i;
        b[i] = sum;
    }
    for (i = n; i >= 1; i--) {
        sum = b[i];
        for (j = i + 1; j <= n; j++) sum -= MAT(a, n1, i, j) * b[j];
        b[i] = sum / MAT(a, n1, i, i);
    }
}

/* ellfit.c:11-88: least-squares Laplace-series fit of the log curvature
   function of the a,b,c ellipsoid -> initial shape coefficients. */
static int ellfit(pso_problem* p, double* cg, double a, double b, double c) {
    int ndir = p->numfac, ncoef = p->ncoef, i, m, l, n, j, k, rc;
    int Lmax = p->lmax, Mmax = p->mmax, nc1 = ncoef + 1;
    double sum, st, d;
    int* indx = (int*)xcalloc(ncoef + 1, sizeof(int));
    double* fitvec = (double*)xcalloc(ncoef + 1, sizeof(double));
    double* er = (double*)xcalloc(ndir + 1, sizeof(double));
    double* fmat = (double*)xcalloc((size_t)(ndir + 1) * nc1, sizeof(double));
    double* fitmat = (double*)xcalloc((size_t)nc1 * nc1, sizeof(double));
    for (i = 1; i <= ndir; i++) {
        st = sin(p->at[i]);
        sum = pow(a * st * cos(p->af[i]), 2) + pow(b * st * sin(p->af[i]), 2) + pow(c * cos(p->at[i]), 2);
        er[i] = 2 * (log(a * b * c) - log(sum));
    }
    for (i = 1; i <= ndir; i++) {
        n = 0;
        for (m = 0; m <= Mmax; m++)
            for (l = m; l <= Lmax; l++) {
                n++;
                if (m != 0) {
                    MAT(fmat, nc1, i, n) = PLEG(p, i, l, m) * cos(m * p->af[i]);
                    n++;
                    MAT(fmat, nc1, i, n) = PLEG(p, i, l, m) * sin(m * p->af[i]);
                } else
                    MAT(fmat, nc1, i, n) = PLEG(p, i, l, m);
            }
    }
    for (i = 1; i <= ncoef; i++) {
        for (j = 1; j <= ncoef; j++) {
            MAT(fitmat, nc1, i, j) = 0;
            for (k = 1; k <= ndir; k++)
                MAT(fitmat, nc1, i, j) = MAT(fitmat, nc1, i, j) + MAT(fmat, nc1, k, i) * MAT(fmat, nc1, k, j);
        }
        fitvec[i] = 0;
        for (j = 1; j <= ndir; j++) fitvec[i] = fitvec[i] + MAT(fmat, nc1, j, i) * er[j];
    }
    rc = ludcmp(fitmat, ncoef, indx, &d);
    if (rc == 0) {
        lubksb(fitmat, ncoef, indx, fitvec);
        for (i = 1; i <= ncoef; i++) cg[i] = fitvec[i];
    }
    free(indx);
    free(fitvec);
    free(er);
    free(fmat);
    free(fitmat);
    return rc;
}

/* --------------------------------------------------------- forward model */

/* curv.c:10-38: facet areas Area = Darea*exp(sum Pleg*(c*Fc + s*Fs)) and
   Dg = g*Dsph. */
static void curv(pso_problem* p, const double* cg) {
    int i, m, n, l, k;
    double fsum;
    for (i = 1; i <= p->numfac; i++) {
        double gi = 0;
        n = 0;
        for (m = 0; m <= p->mmax; m++)
            for (l = m; l <= p->lmax; l++) {
                n++;
                fsum = cg[n] * FC(p, i, m);
                if (m != 0) {
                    n++;
                    fsum = fsum + cg[n] * FS(p, i, m);
                }
                gi = gi + PLEG(p, i, l, m) * fsum;
            }
        gi = exp(gi);
        p->g[i] = gi;
        p->area[i] = p->darea[i] * gi;
        for (k = 1; k <= n; k++) DG(p, i, k) = gi * DSPH(p, i, k);
    }
}

/* blmatrix.c:9-46: pole rotation and its derivatives. */
static void blmatrix(pso_problem* p, double bet, double lam) {
    double cb = cos(bet), sb = sin(bet), cl = cos(lam), sl = sin(lam);
    p->blmat[1][1] = cb * cl;
    p->blmat[1][2] = cb * sl;
    p->blmat[1][3] = -sb;
    p->blmat[2][1] = -sl;
    p->blmat[2][2] = cl;
    p->blmat[2][3] = 0;
    p->blmat[3][1] = sb * cl;
    p->blmat[3][2] = sb * sl;
    p->blmat[3][3] = cb;
    p->dblm[1][1][1] = -sb * cl;
    p->dblm[1][1][2] = -sb * sl;
    p->dblm[1][1][3] = -cb;
    p->dblm[1][2][1] = 0;
    p->dblm[1][2][2] = 0;
    p->dblm[1][2][3] = 0;
    p->dblm[1][3][1] = cb * cl;
    p->dblm[1][3][2] = cb * sl;
    p->dblm[1][3][3] = -sb;
    p->dblm[2][1][1] = -cb * sl;
    p->dblm[2][1][2] = cb * cl;
    p->dblm[2][1][3] = 0;
    p->dblm[2][2][1] = -cl;
    p->dblm[2][2][2] = -sl;
    p->dblm[2][2][3] = 0;
    p->dblm[2][3][1] = -sb * sl;
    p->dblm[2][3][2] = sb * cl;
    p->dblm[2][3][3] = 0;
}

/* matrix.c:11-58: spin rotation at time t and its derivatives. */
static void matrix(const pso_problem* p, double omg, double t, double tmat[][4], double dtm[][4][4]) {
    double f, cf, sf, dfm[4][4], fmat[4][4];
    int i, j, k;
    f = omg * t + p->phi0;
    f = fmod(f, 2 * PSO_PI);
    cf = cos(f);
    sf = sin(f);
    fmat[1][1] = cf;
    fmat[1][2] = sf;
    fmat[1][3] = 0;
    fmat[2][1] = -sf;
    fmat[2][2] = cf;
    fmat[2][3] = 0;
    fmat[3][1] = 0;
    fmat[3][2] = 0;
    fmat[3][3] = 1;
    dfm[1][1] = -t * sf;
    dfm[1][2] = t * cf;
    dfm[1][3] = 0;
    dfm[2][1] = -t * cf;
    dfm[2][2] = -t * sf;
    dfm[2][3] = 0;
    dfm[3][1] = 0;
    dfm[3][2] = 0;
    dfm[3][3] = 0;
    for (i = 1; i <= 3; i++)
        for (j = 1; j <= 3; j++) {
            tmat[i][j] = 0;
            dtm[1][i][j] = 0;
            dtm[2][i][j] = 0;
            dtm[3][i][j] = 0;
            for (k = 1; k <= 3; k++) {
                tmat[i][j] = tmat[i][j] + fmat[i][k] * p->blmat[k][j];
                dtm[1][i][j] = dtm[1][i][j] + fmat[i][k] * p->dblm[1][k][j];
                dtm[2][i][j] = dtm[2][i][j] + fmat[i][k] * p->dblm[2][k][j];
                dtm[3][i][j] = dtm[3][i][j] + dfm[i][k] * p->blmat[k][j];
            }
        }
}

/* phasec.c:11-24: exponential-linear phase function and its derivatives;
   sets Scale. */
static void phasec(pso_problem* p, double dcdp[], double alpha, const double pp[]) {
    double e, c;
    e = exp(-alpha / pp[2]);
    c = 1 + pp[1] * e + pp[3] * alpha;
    dcdp[1] = e;
    dcdp[2] = pp[1] * e * alpha / (pp[2] * pp[2]);
    dcdp[3] = alpha;
    p->scale = c;
}

static double dot3(const double a[4], const double b[4]) {
    /* dot_product.c:6-18 */
    return a[1] * b[1] + a[2] * b[2] + a[3] * b[3];
}

/* bright.c:14-126: disk-integrated Lambert + Lommel-Seeliger brightness of
   the visible and illuminated facets, and its derivatives. */
static double bright(pso_problem* p, const double ee[4], const double ee0[4], double t, const double* cg,
                     double* dyda, int ncoef) {
    int ncoef0, i, j, k, Numfac = p->numfac, Nphpar = p->nphpar;
    double cos_alpha, br, cl, cls, alpha, sum, sum0, dnom;
    double e[4], e0[4], php[6], dphp[6], de[4][4], de0[4][4], tmat[4][4], dtm[4][4][4];
    int* incl = p->incl;
    double *mu = p->mu, *mu0 = p->mu0, *s = p->s, *dbr = p->dbr, *dsmu = p->dsmu, *dsmu0 = p->dsmu0;

    ncoef0 = ncoef - 2 - Nphpar;
    cl = exp(cg[ncoef - 1]);
    cls = cg[ncoef];
    cos_alpha = dot3(ee, ee0);
    alpha = acos(cos_alpha);
    for (i = 1; i <= Nphpar; i++) php[i] = cg[ncoef0 + i];
    phasec(p, dphp, alpha, php);
    matrix(p, cg[ncoef0], t, tmat, dtm);
    br = 0;
    for (i = 1; i <= 3; i++) {
        e[i] = 0;
        e0[i] = 0;
        for (j = 1; j <= 3; j++) {
            e[i] = e[i] + tmat[i][j] * ee[j];
            e0[i] = e0[i] + tmat[i][j] * ee0[j];
            de[i][j] = 0;
            de0[i][j] = 0;
            for (k = 1; k <= 3; k++) {
                de[i][j] = de[i][j] + dtm[j][i][k] * ee[k];
                de0[i][j] = de0[i][j] + dtm[j][i][k] * ee0[k];
            }
        }
    }
    for (i = 1; i <= Numfac; i++) {
        incl[i] = 0;
        mu[i] = e[1] * NOR(p, i, 1) + e[2] * NOR(p, i, 2) + e[3] * NOR(p, i, 3);
        mu0[i] = e0[1] * NOR(p, i, 1) + e0[2] * NOR(p, i, 2) + e0[3] * NOR(p, i, 3);
        if ((mu[i] > PSO_TINY) && (mu0[i] > PSO_TINY)) {
            incl[i] = 1;
            dnom = mu[i] + mu0[i];
            s[i] = mu[i] * mu0[i] * (cl + cls / dnom);
            br = br + p->area[i] * s[i];
            dsmu[i] = cls * PSO_SQ(mu0[i] / dnom) + cl * mu0[i];
            dsmu0[i] = cls * PSO_SQ(mu[i] / dnom) + cl * mu[i];
            dbr[i] = p->darea[i] * s[i];
        }
    }
    for (i = 1; i <= ncoef0 - 3; i++) {
        dyda[i] = 0;
        for (j = 1; j <= Numfac; j++)
            if (incl[j] == 1) dyda[i] = dyda[i] + dbr[j] * DG(p, j, i);
        dyda[i] = p->scale * dyda[i];
    }
    for (k = 1; k <= 3; k++) {
        dyda[ncoef0 - 3 + k] = 0;
        for (i = 1; i <= Numfac; i++)
            if (incl[i] == 1) {
                sum = 0;
                sum0 = 0;
                for (j = 1; j <= 3; j++) {
                    sum = sum + NOR(p, i, j) * de[j][k];
                    sum0 = sum0 + NOR(p, i, j) * de0[j][k];
                }
                dyda[ncoef0 - 3 + k] = dyda[ncoef0 - 3 + k] + p->area[i] * (dsmu[i] * sum + dsmu0[i] * sum0);
            }
        dyda[ncoef0 - 3 + k] = p->scale * dyda[ncoef0 - 3 + k];
    }
    for (i = 1; i <= Nphpar; i++) dyda[ncoef0 + i] = br * dphp[i];
    dyda[ncoef - 1] = 0;
    dyda[ncoef] = 0;
    for (i = 1; i <= Numfac; i++)
        if (incl[i] == 1) {
            dyda[ncoef - 1] = dyda[ncoef - 1] + mu[i] * mu0[i] * p->area[i];
            dyda[ncoef] = dyda[ncoef] + p->area[i] * mu[i] * mu0[i] / (mu[i] + mu0[i]);
        }
    dyda[ncoef - 1] = p->scale * dyda[ncoef - 1] * cl;
    dyda[ncoef] = p->scale * dyda[ncoef];
    br *= p->scale;
    return br;
}

/* conv.c:12-29: convexity residual row nc and its shape derivatives. */
static double conv(pso_problem* p, int nc, double* dres, int ma) {
    int i, j;
    double res = 0;
    for (j = 1; j <= ma; j++) dres[j] = 0;
    for (i = 1; i <= p->numfac; i++) {
        res += p->area[i] * NOR(p, i, nc);
        for (j = 1; j <= p->ncoef; j++) dres[j] += p->darea[i] * DG(p, i, j) * NOR(p, i, nc);
    }
    return res;
}

/* mrqcof.c:16-148 (Lastcall == 0 branch, the only one the scan uses):
   model, Jacobian, relative-lightcurve normalisation, alpha = J^T W J,
   beta = J^T W r and chi2.  When model_y/model_dyda are given, the
   normalised rows are also stored there (0-based rows). */
static double mrqcof_impl(pso_problem* p, const double* a, double* alpha, double* beta, double* model_y,
                          double* model_dyda) {
    int ma = p->ma, mfit, i, j, k, l, m, np, np1, np2, jp, ic, m1;
    double xx1[4], xx2[4], dy, sig2i, wt, ymod, coef, ave = 0, trial_chisq, wght;
    double *dyda = p->dyda, *ytemp = p->ytemp, *dave = p->dave;
    size_t dstride = (size_t)ma + 1;
#define DYT(jp, l) p->dytemp[(size_t)(jp)*dstride + (l)]

    curv(p, a);
    blmatrix(p, a[ma - 4 - p->nphpar], a[ma - 3 - p->nphpar]);
    mfit = 0;
    for (j = 1; j <= ma; j++)
        if (p->ia[j]) mfit++;
    m1 = mfit + 1;
    for (j = 1; j <= mfit; j++) {
        for (k = 1; k <= j; k++) MAT(alpha, m1, j, k) = 0;
        beta[j] = 0;
    }
    trial_chisq = 0;
    np = 0;
    np1 = 0;
    np2 = 0;
    for (i = 1; i <= p->lcurves; i++) {
        if (p->inrel[i] == 1) {
            ave = 0;
            for (l = 1; l <= ma; l++) dave[l] = 0;
        }
        for (jp = 1; jp <= p->lpoints[i]; jp++) {
            np++;
            for (ic = 1; ic <= 3; ic++) {
                xx1[ic] = p->ee[np * 4 + ic];
                xx2[ic] = p->ee0[np * 4 + ic];
            }
            if (i < p->lcurves)
                ymod = bright(p, xx1, xx2, p->tim[np], a, dyda, ma);
            else
                ymod = conv(p, jp, dyda, ma);
            ytemp[jp] = ymod;
            if (p->inrel[i] == 1) ave = ave + ymod;
            for (l = 1; l <= ma; l++) {
                DYT(jp, l) = dyda[l];
                if (p->inrel[i] == 1) dave[l] = dave[l] + dyda[l];
            }
        }
        for (jp = 1; jp <= p->lpoints[i]; jp++) {
            np1++;
            if (p->inrel[i] == 1) {
                coef = p->sig[np1] * p->lpoints[i] / ave;
                for (l = 1; l <= ma; l++) DYT(jp, l) = coef * (DYT(jp, l) - ytemp[jp] * dave[l] / ave);
                ytemp[jp] = coef * ytemp[jp];
                DYT(jp, 1) = 0;
            }
        }
        for (jp = 1; jp <= p->lpoints[i]; jp++) {
            ymod = ytemp[jp];
            for (l = 1; l <= ma; l++) dyda[l] = DYT(jp, l);
            np2++;
            if (model_y) {
                model_y[np2 - 1] = ymod;
                for (l = 1; l <= ma; l++) model_dyda[(size_t)(np2 - 1) * ma + (l - 1)] = dyda[l];
            }
            sig2i = 1 / (p->sig[np2] * p->sig[np2]);
            wght = p->weight[np2];
            dy = p->brightness[np2] - ymod;
            j = 0;
            for (l = 1; l <= ma; l++) {
                if (p->ia[l]) {
                    j++;
                    wt = dyda[l] * sig2i * wght;
                    k = 0;
                    for (m = 1; m <= l; m++) {
                        if (p->ia[m]) {
                            k++;
                            MAT(alpha, m1, j, k) = MAT(alpha, m1, j, k) + wt * dyda[m];
                        }
                    }
                    beta[j] = beta[j] + dy * wt;
                }
            }
            trial_chisq = trial_chisq + dy * dy * sig2i * wght;
        }
    }
    for (j = 2; j <= mfit; j++)
        for (k = 1; k <= j - 1; k++) MAT(alpha, m1, k, j) = MAT(alpha, m1, j, k);
#undef DYT
    return trial_chisq;
}

/* gauss_errc.c:9-73 on a 1-based (n+1)x(n+1) matrix. */
static int gauss_errc1(double* a, int n, double* b) {
    int i, icol = 0, irow = 0, j, k, l, ll, n1 = n + 1;
    double big, dum, pivinv, temp;
    int* indxc = (int*)xcalloc(n + 1, sizeof(int));
    int* indxr = (int*)xcalloc(n + 1, sizeof(int));
    int* ipiv = (int*)xcalloc(n + 1, sizeof(int));
    int rc = 0;
    for (j = 1; j <= n; j++) ipiv[j] = 0;
    for (i = 1; i <= n; i++) {
        big = 0.0;
        for (j = 1; j <= n; j++)
            if (ipiv[j] != 1)
                for (k = 1; k <= n; k++) {
                    if (ipiv[k] == 0) {
                        if (fabs(MAT(a, n1, j, k)) >= big) {
                            big = fabs(MAT(a, n1, j, k));
                            irow = j;
                            icol = k;
                        }
                    } else if (ipiv[k] > 1) {
                        rc = 1;
                        goto done;
                    }
                }
        ++(ipiv[icol]);
        if (irow != icol) {
            for (l = 1; l <= n; l++) {
                temp = MAT(a, n1, irow, l);
                MAT(a, n1, irow, l) = MAT(a, n1, icol, l);
                MAT(a, n1, icol, l) = temp;
            }
            temp = b[irow];
            b[irow] = b[icol];
            b[icol] = temp;
        }
        indxr[i] = irow;
        indxc[i] = icol;
        if (MAT(a, n1, icol, icol) == 0.0) {
            rc = 2;
            goto done;
        }
        pivinv = 1.0 / MAT(a, n1, icol, icol);
        MAT(a, n1, icol, icol) = 1.0;
        for (l = 1; l <= n; l++) MAT(a, n1, icol, l) *= pivinv;
        b[icol] *= pivinv;
        for (ll = 1; ll <= n; ll++)
            if (ll != icol) {
                dum = MAT(a, n1, ll, icol);
                MAT(a, n1, ll, icol) = 0.0;
                for (l = 1; l <= n; l++) MAT(a, n1, ll, l) -= MAT(a, n1, icol, l) * dum;
                b[ll] -= b[icol] * dum;
            }
    }
    for (l = n; l >= 1; l--) {
        if (indxr[l] != indxc[l])
            for (k = 1; k <= n; k++) {
                temp = MAT(a, n1, k, indxr[l]);
                MAT(a, n1, k, indxr[l]) = MAT(a, n1, k, indxc[l]);
                MAT(a, n1, k, indxc[l]) = temp;
            }
    }
done:
    free(indxc);
    free(indxr);
    free(ipiv);
    return rc;
}

/* mrqmin.c:11-110 (Lastcall != 1 path).  alpha / covar are (mfit+1)^2. */
static int mrqmin(pso_problem* p, double* a) {
    int j, k, l, err_code, ma = p->ma, mfit = p->mfit, m1 = p->mfit + 1;
    double temp;
    if (p->alamda < 0) {
        p->alamda = p->alamda_start;
        temp = mrqcof_impl(p, a, p->alpha, p->lm_beta, NULL, NULL);
        p->ochisq = temp;
        for (j = 1; j <= ma; j++) p->atry[j] = a[j];
    }
    for (j = 1; j <= mfit; j++) {
        for (k = 1; k <= mfit; k++) MAT(p->covar, m1, j, k) = MAT(p->alpha, m1, j, k);
        MAT(p->covar, m1, j, j) = MAT(p->alpha, m1, j, j) * (1 + p->alamda);
        p->da[j] = p->lm_beta[j];
    }
    err_code = gauss_errc1(p->covar, mfit, p->da);
    if (err_code != 0) {
        if (p->lm_status == 0) p->lm_status = err_code;
        return err_code;
    }
    j = 0;
    for (l = 1; l <= ma; l++)
        if (p->ia[l]) {
            j++;
            p->atry[l] = a[l] + p->da[j];
        }
    temp = mrqcof_impl(p, p->atry, p->covar, p->da, NULL, NULL);
    p->chisq = temp;
    if (temp < p->ochisq) {
        p->alamda = p->alamda / p->alamda_incr;
        for (j = 1; j <= mfit; j++) {
            for (k = 1; k <= mfit; k++) MAT(p->alpha, m1, j, k) = MAT(p->covar, m1, j, k);
            p->lm_beta[j] = p->da[j];
        }
        for (l = 1; l <= ma; l++) a[l] = p->atry[l];
    } else {
        p->alamda = p->alamda_incr * p->alamda;
        p->chisq = p->ochisq;
    }
    return 0;
}

/* ----------------------------------------------------------- input file */

static void skip_line(FILE* fp) {
    int c;
    while ((c = fgetc(fp)) != EOF && c != '\n') {
    }
}

void pso_free(pso_problem* p) {
    if (!p) return;
    void* ptrs[] = {p->lpoints, p->inrel, p->tim, p->ee, p->ee0, p->brightness, p->sig, p->weight, p->t,
                    p->f, p->at, p->af, p->ifp, p->nor, p->darea, p->fc, p->fs, p->tc, p->ts, p->pleg,
                    p->dsph, p->cg_first, p->ia, p->area, p->dg, p->g, p->ytemp, p->dytemp, p->dyda,
                    p->dave, p->incl, p->mu, p->mu0, p->s, p->dbr, p->dsmu, p->dsmu0, p->atry,
                    p->lm_beta, p->da, p->covar, p->alpha, p->cg};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
    free(p);
}

/* period_search_BOINC.cpp:277-485: header, lightcurves, weights,
   normalisation, initial shape size, convexity pseudo-lightcurve. */
pso_problem* pso_load(const char* path, int* status) {
    FILE* fp = fopen(path, "r");
    int i, j, k, k2, i_temp, ial0, ial0_abs, lc_number, n_alloc;
    double ave, e0len, elen, cos_alpha, al0, al0_abs, e[4], e0[4], rfit;
    double* al;
    double* weight_lc;
    pso_problem* p;
    if (status) *status = 0;
    if (!fp) {
        if (status) *status = -1;
        return NULL;
    }
    p = (pso_problem*)xcalloc(1, sizeof(pso_problem));
#define RD(fmt, ...)                                     \
    do {                                                 \
        if (fscanf(fp, fmt, __VA_ARGS__) < 1) goto bad; \
        skip_line(fp);                                   \
    } while (0)
    RD("%lf %lf %lf %d", &p->per_start, &p->per_step_coef, &p->per_end, &p->ia_prd);
    RD("%lf", &p->jd_00);
    RD("%lf", &p->phi0);
    RD("%lf", &p->conw);
    RD("%d %d", &p->lmax, &p->mmax);
    RD("%d", &p->nrows);
    RD("%lf %d", &p->par[1], &p->ia_par[1]);
    RD("%lf %d", &p->par[2], &p->ia_par[2]);
    RD("%lf %d", &p->par[3], &p->ia_par[3]);
    RD("%lf %d", &p->cl, &p->ia_cl);
    RD("%lf", &p->stop_condition);
    RD("%d", &p->n_iter_min);
    RD("%lf", &p->alamda_incr);
    RD("%lf", &p->alamda_start);
#undef RD
    if (p->lmax < 0 || p->lmax > PSO_MAX_LM || p->mmax < 0 || p->mmax > p->lmax || p->nrows < 1) goto bad;
    if (fscanf(fp, "%d", &p->lcurves) != 1 || p->lcurves < 1) goto bad;
    /* +1 for the convexity pseudo-curve appended below */
    p->lpoints = (int*)xcalloc(p->lcurves + 2, sizeof(int));
    p->inrel = (int*)xcalloc(p->lcurves + 2, sizeof(int));
    al = (double*)xcalloc(p->lcurves + 1, sizeof(double));
    weight_lc = (double*)xcalloc(p->lcurves + 1, sizeof(double));
    n_alloc = 1024;
    p->tim = (double*)xcalloc(n_alloc + 1, sizeof(double));
    p->ee = (double*)xcalloc((size_t)(n_alloc + 1) * 4, sizeof(double));
    p->ee0 = (double*)xcalloc((size_t)(n_alloc + 1) * 4, sizeof(double));
    p->brightness = (double*)xcalloc(n_alloc + 4, sizeof(double));
    p->sig = (double*)xcalloc(n_alloc + 4, sizeof(double));
    p->ndata = 0;
    k2 = 0;
    al0 = al0_abs = PSO_PI;
    ial0 = ial0_abs = -1;
    p->jd_min = 1e20;
    p->jd_max = -1e40;
    p->onlyrel = 1;
    p->jd_0 = p->jd_00;
    p->a_axis = 1.05;
    p->b_axis = 1.00;
    p->c_axis = 0.95;
    for (i = 1; i <= p->lcurves; i++) {
        ave = 0;
        if (fscanf(fp, "%d %d", &p->lpoints[i], &i_temp) != 2 || p->lpoints[i] < 1) goto bad2;
        skip_line(fp);
        p->inrel[i] = 1 - i_temp;
        if (p->inrel[i] == 0) p->onlyrel = 0;
        if (p->lpoints[i] > p->max_lpoints) p->max_lpoints = p->lpoints[i];
        for (j = 1; j <= p->lpoints[i]; j++) {
            p->ndata++;
            if (p->ndata > n_alloc) {
                n_alloc *= 2;
                p->tim = (double*)realloc(p->tim, (n_alloc + 1) * sizeof(double));
                p->ee = (double*)realloc(p->ee, (size_t)(n_alloc + 1) * 4 * sizeof(double));
                p->ee0 = (double*)realloc(p->ee0, (size_t)(n_alloc + 1) * 4 * sizeof(double));
                p->brightness = (double*)realloc(p->brightness, (n_alloc + 4) * sizeof(double));
                p->sig = (double*)realloc(p->sig, (n_alloc + 4) * sizeof(double));
                if (!p->tim || !p->ee || !p->ee0 || !p->brightness || !p->sig) goto bad2;
            }
            if (fscanf(fp, "%lf %lf", &p->tim[p->ndata], &p->brightness[p->ndata]) != 2) goto bad2;
            if (fscanf(fp, "%lf %lf %lf", &e0[1], &e0[2], &e0[3]) != 3) goto bad2;
            if (fscanf(fp, "%lf %lf %lf", &e[1], &e[2], &e[3]) != 3) goto bad2;
            if (p->tim[p->ndata] < p->jd_min) p->jd_min = p->tim[p->ndata];
            if (p->tim[p->ndata] > p->jd_max) p->jd_max = p->tim[p->ndata];
            e0len = sqrt(e0[1] * e0[1] + e0[2] * e0[2] + e0[3] * e0[3]);
            elen = sqrt(e[1] * e[1] + e[2] * e[2] + e[3] * e[3]);
            ave += p->brightness[p->ndata];
            for (k = 1; k <= 3; k++) {
                p->ee[p->ndata * 4 + k] = e[k] / elen;
                p->ee0[p->ndata * 4 + k] = e0[k] / e0len;
            }
            if (j == 1) {
                cos_alpha = dot3(e, e0) / (elen * e0len);
                al[i] = acos(cos_alpha);
                if (al[i] < al0) {
                    al0 = al[i];
                    ial0 = p->ndata;
                }
                if ((al[i] < al0_abs) && (p->inrel[i] == 0)) {
                    al0_abs = al[i];
                    ial0_abs = p->ndata;
                }
            }
        }
        ave /= p->lpoints[i];
        for (j = 1; j <= p->lpoints[i]; j++) {
            k2++;
            p->sig[k2] = ave;
        }
    }
    /* weights: `lc weight` pairs to EOF (:420-427) */
    for (i = 1; i <= p->lcurves; i++) weight_lc[i] = -1;
    while (feof(fp) == 0) {
        double w;
        if (fscanf(fp, "%d", &lc_number) != 1) break;
        if (fscanf(fp, "%lf", &w) != 1) break;
        if (lc_number >= 1 && lc_number <= p->lcurves) weight_lc[lc_number] = w;
    }
    fclose(fp);
    fp = NULL;
    if (p->jd_0 <= 0) p->jd_0 = (int)p->jd_min;
    for (i = 1; i <= p->ndata; i++) p->tim[i] = p->tim[i] - p->jd_0;
    p->phi0 = p->phi0 * PSO_DEG2RAD;
    p->weight = (double*)xcalloc(p->ndata + 4, sizeof(double));
    k = 0;
    for (i = 1; i <= p->lcurves; i++)
        for (j = 1; j <= p->lpoints[i]; j++) {
            k++;
            if (weight_lc[i] == -1)
                p->weight[k] = 1;
            else
                p->weight[k] = weight_lc[i];
        }
    for (i = 1; i <= 3; i++) p->weight[k + i] = 1;
    if (p->onlyrel == 0) {
        al0 = al0_abs;
        ial0 = ial0_abs;
    }
    rfit = sqrt(2 * p->sig[ial0] / (0.5 * PSO_PI * (1 + cos(al0))));
    p->escl = rfit / sqrt((p->a_axis * p->b_axis + p->b_axis * p->c_axis + p->a_axis * p->c_axis) / 3);
    if (p->onlyrel == 0) p->escl *= 0.8;
    p->a_axis = p->a_axis * p->escl;
    p->b_axis = p->b_axis * p->escl;
    p->c_axis = p->c_axis * p->escl;
    p->lcurves = p->lcurves + 1;
    p->lpoints[p->lcurves] = 3;
    p->inrel[p->lcurves] = 0;
    if (p->max_lpoints < 3) p->max_lpoints = 3;
    p->conw_r = p->conw / p->escl / p->escl;
    p->ndata_tot = p->ndata; /* convexity rows appended by setup_rows() */
    free(al);
    free(weight_lc);
    return p;
bad2:
    free(al);
    free(weight_lc);
bad:
    if (fp) fclose(fp);
    pso_free(p);
    if (status) *status = 2;
    return NULL;
}

/* period_search_BOINC.cpp:491-496 / 719-726: append the three convexity
   rows (brightness 0, sigma 1/conw_r). */
static void setup_rows(pso_problem* p) {
    int j;
    p->ndata_tot = p->ndata;
    for (j = 1; j <= 3; j++) {
        p->ndata_tot++;
        p->brightness[p->ndata_tot] = 0;
        p->sig[p->ndata_tot] = 1 / p->conw_r;
    }
}

/* period_search_BOINC.cpp:497-556 / 728-802: Laplace-series ordering,
   vertex grid, triangulation, normals, SH tables, initial ellipsoid,
   frequency grid and the free-parameter mask. */
static int setup_geometry(pso_problem* p) {
    int i, j, k, m, l, nrows = p->nrows;
    double dth, dph;
    if (!p->geometry_ready) {
        p->ncoef = 0;
        for (m = 0; m <= p->mmax; m++)
            for (l = m; l <= p->lmax; l++) {
                p->ncoef++;
                if (m != 0) p->ncoef++;
            }
        p->numfac = 8 * nrows * nrows;
        p->ndir = 4 * nrows * nrows + 2;
        p->nphpar = 3;
        p->ma = p->ncoef + 5 + p->nphpar;
        int F = p->numfac, C = p->ncoef;
        p->t = (double*)xcalloc(p->ndir + 1, sizeof(double));
        p->f = (double*)xcalloc(p->ndir + 1, sizeof(double));
        p->at = (double*)xcalloc(F + 1, sizeof(double));
        p->af = (double*)xcalloc(F + 1, sizeof(double));
        p->ifp = (int*)xcalloc((size_t)(F + 1) * 4, sizeof(int));
        p->nor = (double*)xcalloc((size_t)(F + 1) * 4, sizeof(double));
        p->darea = (double*)xcalloc(F + 1, sizeof(double));
        p->fc = (double*)xcalloc((size_t)(F + 1) * LM1, sizeof(double));
        p->fs = (double*)xcalloc((size_t)(F + 1) * LM1, sizeof(double));
        p->tc = (double*)xcalloc((size_t)(F + 1) * LM1, sizeof(double));
        p->ts = (double*)xcalloc((size_t)(F + 1) * LM1, sizeof(double));
        p->pleg = (double*)xcalloc((size_t)(F + 1) * LM1 * LM1, sizeof(double));
        p->dsph = (double*)xcalloc((size_t)(F + 1) * (C + 1), sizeof(double));
        p->dg = (double*)xcalloc((size_t)(F + 1) * (C + 1), sizeof(double));
        p->area = (double*)xcalloc(F + 1, sizeof(double));
        p->g = (double*)xcalloc(F + 1, sizeof(double));
        p->cg_first = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->ia = (int*)xcalloc(p->ma + 1, sizeof(int));
        p->incl = (int*)xcalloc(F + 1, sizeof(int));
        p->mu = (double*)xcalloc(F + 1, sizeof(double));
        p->mu0 = (double*)xcalloc(F + 2, sizeof(double));
        p->s = (double*)xcalloc(F + 1, sizeof(double));
        p->dbr = (double*)xcalloc(F + 1, sizeof(double));
        p->dsmu = (double*)xcalloc(F + 1, sizeof(double));
        p->dsmu0 = (double*)xcalloc(F + 1, sizeof(double));
        p->ytemp = (double*)xcalloc(p->max_lpoints + 1, sizeof(double));
        p->dytemp = (double*)xcalloc((size_t)(p->max_lpoints + 1) * (p->ma + 1), sizeof(double));
        p->dyda = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->dave = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->atry = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->lm_beta = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->da = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->covar = (double*)xcalloc((size_t)(p->ma + 1) * (p->ma + 1), sizeof(double));
        p->alpha = (double*)xcalloc((size_t)(p->ma + 1) * (p->ma + 1), sizeof(double));
        p->cg = (double*)xcalloc(p->ma + 1, sizeof(double));
        p->geometry_ready = 1;
    }
    dth = PSO_PI / (2 * nrows);
    k = 1;
    p->t[1] = 0;
    p->f[1] = 0;
    for (i = 1; i <= nrows; i++) {
        dph = PSO_PI / (2 * i);
        for (j = 0; j <= 4 * i - 1; j++) {
            k++;
            p->t[k] = i * dth;
            p->f[k] = j * dph;
        }
    }
    for (i = nrows - 1; i >= 1; i--) {
        dph = PSO_PI / (2 * i);
        for (j = 0; j <= 4 * i - 1; j++) {
            k++;
            p->t[k] = PSO_PI - i * dth;
            p->f[k] = j * dph;
        }
    }
    p->ndir = k + 1;
    p->t[p->ndir] = PSO_PI;
    p->f[p->ndir] = 0;
    trifac(nrows, p->ifp);
    areanorm(p);
    sphfunc(p);
    if (ellfit(p, p->cg_first, p->a_axis, p->b_axis, p->c_axis) != 0) return 4;
    p->freq_start = 1 / p->per_start;
    p->freq_end = 1 / p->per_end;
    p->freq_step = 0.5 / (p->jd_max - p->jd_min) / 24 * p->per_step_coef;
    p->ia[p->ncoef + 1] = 1;
    p->ia[p->ncoef + 2] = 1;
    p->ia[p->ncoef + 3] = p->ia_prd;
    for (i = 1; i <= p->ncoef; i++) p->ia[i] = 1;
    if (p->onlyrel == 1) p->ia[1] = 0;
    p->ia[p->ncoef + 3 + p->nphpar + 1] = p->ia_cl;
    p->ia[p->ncoef + 3 + p->nphpar + 2] = 0;
    for (i = 1; i <= p->nphpar; i++) p->ia[p->ncoef + 3 + i] = p->ia_par[i];
    p->mfit = 0;
    for (j = 1; j <= p->ma; j++)
        if (p->ia[j]) p->mfit++;
    return 0;
}

int pso_n_periods(const pso_problem* p) {
    return (int)((p->freq_start - p->freq_end) / p->freq_step) + 1;
}

/* One fit, period_search_BOINC.cpp:819-920 (scan) / 610-694 (pre-pass). */
static void run_fit(pso_problem* p, double freq, int m, double* out) {
    static const double beta_pole[PSO_N_POLES + 1] = {0, 0, 0, 0, 0, 60, 60, 60, -60, -60, -60};
    static const double lambda_pole[PSO_N_POLES + 1] = {0, 0, 90, 180, 270, 60, 180, 300, 60, 180, 300};
    int i, j, n_iter_max, Ncoef = p->ncoef, Nphpar = p->nphpar, ma = p->ma;
    double prd, iter_diff_max, iter_diff, dev_old, dev_new, rchisq, chck[4] = {0, 0, 0, 0};
    double totarea, sum, dark;
    double* cg = p->cg;
    prd = 1 / freq;
    for (i = 1; i <= Ncoef; i++) cg[i] = p->cg_first[i];
    cg[Ncoef + 1] = beta_pole[m];
    cg[Ncoef + 2] = lambda_pole[m];
    cg[Ncoef + 1] = 90 - cg[Ncoef + 1];
    cg[Ncoef + 1] = PSO_DEG2RAD * cg[Ncoef + 1];
    cg[Ncoef + 2] = PSO_DEG2RAD * cg[Ncoef + 2];
    cg[Ncoef + 3] = 24 * 2 * PSO_PI / prd;
    for (i = 1; i <= Nphpar; i++) cg[Ncoef + 3 + i] = p->par[i];
    cg[Ncoef + 3 + Nphpar + 2] = 1;
    cg[Ncoef + 3 + Nphpar + 1] = log(p->cl);
    n_iter_max = 0;
    iter_diff_max = -1;
    rchisq = -1;
    if (p->stop_condition > 1) {
        n_iter_max = (int)p->stop_condition;
        iter_diff_max = 0;
        p->n_iter_min = 0; /* the reference overwrites its global here */
    }
    if (p->stop_condition < 1) {
        n_iter_max = PSO_MAX_N_ITER;
        iter_diff_max = p->stop_condition;
    }
    p->alamda = -1;
    p->niter = 0;
    p->lm_status = 0;
    iter_diff = 1e40;
    dev_old = 1e30;
    dev_new = 0;
    while (((p->niter < n_iter_max) && (iter_diff > iter_diff_max)) || (p->niter < p->n_iter_min)) {
        mrqmin(p, cg);
        p->niter++;
        if ((p->niter == 1) || (p->chisq < p->ochisq)) {
            p->ochisq = p->chisq;
            curv(p, cg);
            for (i = 1; i <= 3; i++) {
                chck[i] = 0;
                for (j = 1; j <= p->numfac; j++) chck[i] = chck[i] + p->area[j] * NOR(p, j, i);
            }
            rchisq = p->chisq - (PSO_SQ(chck[1]) + PSO_SQ(chck[2]) + PSO_SQ(chck[3])) * PSO_SQ(p->conw_r);
        }
        dev_new = sqrt(rchisq / (p->ndata_tot - 3));
        if (dev_old - dev_new > 1e-10) {
            iter_diff = dev_old - dev_new;
            dev_old = dev_new;
        }
    }
    /* Area[] now holds the last curv() evaluation (accepted or not), as in
       the reference (:900-902). */
    totarea = 0;
    for (i = 1; i <= p->numfac; i++) totarea = totarea + p->area[i];
    sum = PSO_SQ(chck[1]) + PSO_SQ(chck[2]) + PSO_SQ(chck[3]);
    dark = sqrt(sum);
    prd = 2 * PSO_PI / cg[Ncoef + 3];
    out[0] = dev_new;
    out[1] = dark;
    out[2] = totarea;
    out[3] = prd;
    out[4] = PSO_RAD2DEG * cg[Ncoef + 2];
    out[5] = 90 - PSO_RAD2DEG * cg[Ncoef + 1];
    out[6] = p->chisq;
    out[7] = p->niter;
    out[8] = p->alamda;
    out[9] = p->lm_status;
    (void)ma;
}

/* Best-of-poles record for trial period n (:811-924). */
static void run_period(pso_problem* p, int n, int prepass, pso_record* rec) {
    double freq = p->freq_start - (n - 1) * p->freq_step;
    double per_best = 0, dark_best = 0, la_best = 0, be_best = 0, dev_best = 1e40, out[10];
    int m;
    for (m = 1; m <= PSO_N_POLES; m++) {
        run_fit(p, freq, m, out);
        if (out[0] < dev_best) {
            dev_best = out[0];
            per_best = out[3];
            dark_best = out[1] / out[2] * 100;
            la_best = out[4];
            be_best = out[5];
        }
    }
    if (la_best < 0) la_best += 360;
    if (prepass && isnan(dark_best)) dark_best = 1.0;
    rec->period_h = 24 * per_best;
    rec->rms = dev_best;
    rec->chi2 = dev_best * dev_best * (p->ndata_tot - 3);
    rec->dark = dark_best;
    rec->lambda_deg = la_best;
    rec->beta_deg = be_best;
}

int pso_prepass(pso_problem* p, double* conw_r) {
    int new_conw = 0, n, max_test_periods, rc;
    double sum_dark_facet, ave_dark_facet;
    pso_record rec;
    while ((new_conw != 1) && ((p->conw_r * p->escl * p->escl) < 10.0)) {
        setup_rows(p);
        rc = setup_geometry(p);
        if (rc) return rc;
        max_test_periods = 10;
        sum_dark_facet = 0.0;
        n = pso_n_periods(p);
        if (n < max_test_periods) max_test_periods = n;
        for (n = 1; n <= max_test_periods; n++) {
            run_period(p, n, 1, &rec);
            sum_dark_facet = sum_dark_facet + rec.dark;
        }
        ave_dark_facet = sum_dark_facet / max_test_periods;
        if (ave_dark_facet < 1.0) new_conw = 1;
        if (ave_dark_facet >= 1.0) p->conw_r = p->conw_r * 2;
    }
    setup_rows(p);
    rc = setup_geometry(p);
    if (conw_r) *conw_r = p->conw_r;
    return rc;
}

int pso_set_conw_r(pso_problem* p, double conw_r) {
    p->conw_r = conw_r;
    setup_rows(p);
    return setup_geometry(p);
}

int pso_scan(pso_problem* p, int n_from, int n_to, pso_record* out) {
    int n;
    for (n = n_from; n <= n_to; n++) run_period(p, n, 0, &out[n - n_from]);
    return 0;
}

int pso_fit(pso_problem* p, double freq, int m, double* out, double* cg_out) {
    if (m < 1 || m > PSO_N_POLES) return 2;
    run_fit(p, freq, m, out);
    if (cg_out)
        for (int i = 1; i <= p->ma; i++) cg_out[i - 1] = p->cg[i];
    return 0;
}

double pso_mrqcof(pso_problem* p, const double* a, double* alpha, double* beta) {
    int ma = p->ma, mfit = p->mfit, j, k;
    double* a1 = (double*)xcalloc(ma + 1, sizeof(double));
    double* al1 = (double*)xcalloc((size_t)(mfit + 1) * (mfit + 1), sizeof(double));
    double* be1 = (double*)xcalloc(mfit + 1, sizeof(double));
    for (j = 1; j <= ma; j++) a1[j] = a[j - 1];
    double chi2 = mrqcof_impl(p, a1, al1, be1, NULL, NULL);
    for (j = 1; j <= mfit; j++) {
        if (beta) beta[j - 1] = be1[j];
        if (alpha)
            for (k = 1; k <= mfit; k++) alpha[(j - 1) * mfit + (k - 1)] = MAT(al1, mfit + 1, j, k);
    }
    free(a1);
    free(al1);
    free(be1);
    return chi2;
}

int pso_model(pso_problem* p, const double* a, double* ymod, double* dyda) {
    int ma = p->ma, mfit = p->mfit, j;
    double* a1 = (double*)xcalloc(ma + 1, sizeof(double));
    double* al1 = (double*)xcalloc((size_t)(mfit + 1) * (mfit + 1), sizeof(double));
    double* be1 = (double*)xcalloc(mfit + 1, sizeof(double));
    for (j = 1; j <= ma; j++) a1[j] = a[j - 1];
    mrqcof_impl(p, a1, al1, be1, ymod, dyda);
    free(a1);
    free(al1);
    free(be1);
    return 0;
}

int pso_gauss_errc(double* a, int n, double* b) {
    int n1 = n + 1, j, k, rc;
    double* a1 = (double*)xcalloc((size_t)n1 * n1, sizeof(double));
    double* b1 = (double*)xcalloc(n1, sizeof(double));
    for (j = 1; j <= n; j++) {
        b1[j] = b[j - 1];
        for (k = 1; k <= n; k++) MAT(a1, n1, j, k) = a[(j - 1) * n + (k - 1)];
    }
    rc = gauss_errc1(a1, n, b1);
    for (j = 1; j <= n; j++) {
        b[j - 1] = b1[j];
        for (k = 1; k <= n; k++) a[(j - 1) * n + (k - 1)] = MAT(a1, n1, j, k);
    }
    free(a1);
    free(b1);
    return rc;
}

pso_problem* pso_geometry(int lmax, int mmax, int nrows, double a, double b, double c) {
    pso_problem* p = (pso_problem*)xcalloc(1, sizeof(pso_problem));
    p->lmax = lmax;
    p->mmax = mmax;
    p->nrows = nrows;
    p->a_axis = a;
    p->b_axis = b;
    p->c_axis = c;
    p->per_start = 1;
    p->per_end = 2;
    p->per_step_coef = 1;
    p->jd_min = 0;
    p->jd_max = 1;
    p->max_lpoints = 3;
    p->lpoints = (int*)xcalloc(2, sizeof(int));
    p->inrel = (int*)xcalloc(2, sizeof(int));
    p->tim = (double*)xcalloc(1, sizeof(double));
    p->ee = (double*)xcalloc(4, sizeof(double));
    p->ee0 = (double*)xcalloc(4, sizeof(double));
    p->brightness = (double*)xcalloc(4, sizeof(double));
    p->sig = (double*)xcalloc(4, sizeof(double));
    p->weight = (double*)xcalloc(4, sizeof(double));
    if (setup_geometry(p) != 0) {
        pso_free(p);
        return NULL;
    }
    return p;
}

void pso_curv(pso_problem* p, const double* cg, double* area, double* dg) {
    int i, k;
    double* c1 = (double*)xcalloc(p->ma + 1, sizeof(double));
    for (i = 1; i <= p->ncoef; i++) c1[i] = cg[i - 1];
    curv(p, c1);
    for (i = 1; i <= p->numfac; i++) {
        area[i - 1] = p->area[i];
        for (k = 1; k <= p->ncoef; k++) dg[(size_t)(i - 1) * p->ncoef + (k - 1)] = DG(p, i, k);
    }
    free(c1);
}

int pso_info(const pso_problem* p, int* ints, double* dbls) {
    if (ints) {
        ints[0] = p->ndata;
        ints[1] = p->lcurves;
        ints[2] = p->numfac;
        ints[3] = p->ncoef;
        ints[4] = p->ma;
        ints[5] = p->mfit;
        ints[6] = p->geometry_ready ? pso_n_periods(p) : 0;
        ints[7] = p->lmax;
        ints[8] = p->mmax;
        ints[9] = p->nrows;
        ints[10] = p->onlyrel;
        ints[11] = p->n_iter_min;
        ints[12] = p->ia_prd;
        ints[13] = p->ia_cl;
    }
    if (dbls) {
        dbls[0] = p->escl;
        dbls[1] = p->conw_r;
        dbls[2] = p->freq_start;
        dbls[3] = p->freq_end;
        dbls[4] = p->freq_step;
        dbls[5] = p->jd_0;
        dbls[6] = p->phi0;
        dbls[7] = p->alamda_start;
        dbls[8] = p->alamda_incr;
        dbls[9] = p->stop_condition;
        dbls[10] = p->jd_min;
        dbls[11] = p->jd_max;
        dbls[12] = p->cl;
        dbls[13] = p->par[1];
        dbls[14] = p->par[2];
        dbls[15] = p->par[3];
    }
    return 0;
}

int pso_get_array(const pso_problem* p, const char* name, double* out) {
    int F = p->numfac, C = p->ncoef, N = p->ndata, i, j, l, m, n = 0;
#define NEED_GEOM \
    if (!p->geometry_ready) return -1
    if (!strcmp(name, "nor")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++)
            for (j = 1; j <= 3; j++) out[n++] = NOR(p, i, j);
    } else if (!strcmp(name, "darea")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++) out[n++] = p->darea[i];
    } else if (!strcmp(name, "at")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++) out[n++] = p->at[i];
    } else if (!strcmp(name, "af")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++) out[n++] = p->af[i];
    } else if (!strcmp(name, "ifp")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++)
            for (j = 1; j <= 3; j++) out[n++] = p->ifp[i * 4 + j];
    } else if (!strcmp(name, "dsph")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++)
            for (j = 1; j <= C; j++) out[n++] = DSPH(p, i, j);
    } else if (!strcmp(name, "pleg")) {
        NEED_GEOM;
        for (i = 1; i <= F; i++)
            for (l = 0; l <= p->lmax; l++)
                for (m = 0; m <= p->lmax; m++) out[n++] = PLEG(p, i, l, m);
    } else if (!strcmp(name, "fc") || !strcmp(name, "fs")) {
        NEED_GEOM;
        const double* src = name[1] == 'c' ? p->fc : p->fs;
        for (i = 1; i <= F; i++)
            for (m = 0; m <= p->mmax; m++) out[n++] = src[(size_t)i * LM1 + m];
    } else if (!strcmp(name, "cg_first")) {
        NEED_GEOM;
        for (i = 1; i <= C; i++) out[n++] = p->cg_first[i];
    } else if (!strcmp(name, "ia")) {
        NEED_GEOM;
        for (i = 1; i <= p->ma; i++) out[n++] = p->ia[i];
    } else if (!strcmp(name, "tim")) {
        for (i = 1; i <= N; i++) out[n++] = p->tim[i];
    } else if (!strcmp(name, "ee") || !strcmp(name, "ee0")) {
        const double* src = name[2] == '0' ? p->ee0 : p->ee;
        for (i = 1; i <= N; i++)
            for (j = 1; j <= 3; j++) out[n++] = src[i * 4 + j];
    } else if (!strcmp(name, "alpha_phase")) {
        for (i = 1; i <= N; i++) out[n++] = acos(dot3(&p->ee[i * 4], &p->ee0[i * 4]));
    } else if (!strcmp(name, "brightness") || !strcmp(name, "sig") || !strcmp(name, "weight")) {
        const double* src = name[0] == 'b' ? p->brightness : (name[0] == 's' ? p->sig : p->weight);
        for (i = 1; i <= p->ndata_tot; i++) out[n++] = src[i];
    } else if (!strcmp(name, "lpoints")) {
        for (i = 1; i <= p->lcurves; i++) out[n++] = p->lpoints[i];
    } else if (!strcmp(name, "inrel")) {
        for (i = 1; i <= p->lcurves; i++) out[n++] = p->inrel[i];
    } else {
        return -1;
    }
#undef NEED_GEOM
    return n;
}

/* The application body of period_search_BOINC.cpp:147-954 without BOINC:
   resume from period_search_state (:237-251), pre-pass, scan, output lines
   in the reference format plus a full-precision side file. */
int pso_run_app(const char* dir, int n_from, int n_to, double conw_r_given) {
    char path[4096];
    int status = 0, nlines, n_start_from = 1, n, n_max, rc;
    FILE *out, *full, *state;
    pso_problem* p;
    double conw_r;
    snprintf(path, sizeof path, "%s/period_search_in", dir);
    p = pso_load(path, &status);
    if (!p) return status;
    snprintf(path, sizeof path, "%s/period_search_state", dir);
    state = fopen(path, "r");
    int have_state = 0;
    if (state) {
        have_state = fscanf(state, "%d", &nlines) == 1;
        fclose(state);
    }
    if (have_state) n_start_from = nlines + 1;
    if (n_from > 0) n_start_from = n_from;
    snprintf(path, sizeof path, "%s/period_search_out", dir);
    out = fopen(path, have_state ? "a" : "w");
    snprintf(path, sizeof path, "%s/period_search_out.full", dir);
    full = fopen(path, have_state ? "a" : "w");
    if (!out || !full) {
        pso_free(p);
        return 1;
    }
    rc = conw_r_given > 0 ? pso_set_conw_r(p, conw_r_given) : pso_prepass(p, &conw_r);
    if (rc) {
        fclose(out);
        fclose(full);
        pso_free(p);
        return rc;
    }
    n_max = pso_n_periods(p);
    if (n_to > 0 && n_to < n_max) n_max = n_to;
    for (n = n_start_from; n <= n_max; n++) {
        pso_record r;
        run_period(p, n, 0, &r);
        double col4 = (n == 1) ? p->conw_r * p->escl * p->escl : r.dark;
        fprintf(out, "%.8f  %.6f  %.6f %4.1f %4.0f %4.0f\n", r.period_h, r.rms, r.chi2, col4, r.lambda_deg,
                r.beta_deg);
        fprintf(full, "%.17g %.17g %.17g %.17g %.17g %.17g\n", r.period_h, r.rms, r.chi2, col4, r.lambda_deg,
                r.beta_deg);
    }
    fclose(out);
    fclose(full);
    pso_free(p);
    return 0;
}

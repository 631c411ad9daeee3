// Host setup of the B200 period scan.  Each routine restates one reference
// routine (cited per function) in the same FP64 operation order; the
// compile flags (-O3 -ffp-contract=off) keep that order intact.
#include "ps_host.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

namespace psb {
namespace {

const double kPi = M_PI;               // constants.h:13
const double kDeg2Rad = kPi / 180;     // constants.h:17

void skip_line(FILE* fp) {
    int c;
    while ((c = std::fgetc(fp)) != EOF && c != '\n') {
    }
}

// trifac.c:10-82.  ifp gets 3 vertex ids (1-based) per facet.
void trifac(int nrows, std::vector<int>& ifp) {
    const int cols = 4 * nrows + 1;
    std::vector<int> nod((size_t)(2 * nrows + 1) * cols, 0);
    auto NOD = [&](int i, int j) -> int& { return nod[(size_t)i * cols + j]; };
    ifp.assign((size_t)8 * nrows * nrows * 3, 0);
    auto IFP = [&](int t, int j) -> int& { return ifp[(size_t)(t - 1) * 3 + (j - 1)]; };
    int nnod = 1, ntri = 0;
    NOD(0, 0) = nnod;
    for (int i = 1; i <= nrows; i++)
        for (int j = 0; j <= 4 * i - 1; j++) {
            nnod++;
            NOD(i, j) = nnod;
            if (j == 0) NOD(i, 4 * i) = nnod;
        }
    for (int i = nrows - 1; i >= 1; i--)
        for (int j = 0; j <= 4 * i - 1; j++) {
            nnod++;
            NOD(2 * nrows - i, j) = nnod;
            if (j == 0) NOD(2 * nrows - i, 4 * i) = nnod;
        }
    NOD(2 * nrows, 0) = nnod + 1;
    for (int j1 = 1; j1 <= nrows; j1++)
        for (int j3 = 1; j3 <= 4; j3++) {
            int j0 = (j3 - 1) * j1;
            ntri++;
            IFP(ntri, 1) = NOD(j1 - 1, j0 - (j3 - 1));
            IFP(ntri, 2) = NOD(j1, j0);
            IFP(ntri, 3) = NOD(j1, j0 + 1);
            for (int j2 = j0 + 1; j2 <= j0 + j1 - 1; j2++) {
                ntri++;
                IFP(ntri, 1) = NOD(j1, j2);
                IFP(ntri, 2) = NOD(j1 - 1, j2 - (j3 - 1));
                IFP(ntri, 3) = NOD(j1 - 1, j2 - 1 - (j3 - 1));
                ntri++;
                IFP(ntri, 1) = NOD(j1 - 1, j2 - (j3 - 1));
                IFP(ntri, 2) = NOD(j1, j2);
                IFP(ntri, 3) = NOD(j1, j2 + 1);
            }
        }
    for (int j1 = nrows + 1; j1 <= 2 * nrows; j1++)
        for (int j3 = 1; j3 <= 4; j3++) {
            int j0 = (j3 - 1) * (2 * nrows - j1);
            ntri++;
            IFP(ntri, 1) = NOD(j1, j0);
            IFP(ntri, 2) = NOD(j1 - 1, j0 + 1 + (j3 - 1));
            IFP(ntri, 3) = NOD(j1 - 1, j0 + (j3 - 1));
            for (int j2 = j0 + 1; j2 <= j0 + (2 * nrows - j1); j2++) {
                ntri++;
                IFP(ntri, 1) = NOD(j1, j2);
                IFP(ntri, 2) = NOD(j1 - 1, j2 + (j3 - 1));
                IFP(ntri, 3) = NOD(j1, j2 - 1);
                ntri++;
                IFP(ntri, 1) = NOD(j1, j2);
                IFP(ntri, 2) = NOD(j1 - 1, j2 + 1 + (j3 - 1));
                IFP(ntri, 3) = NOD(j1 - 1, j2 + (j3 - 1));
            }
        }
}

// areanorm.c:10-60 with the vertex grid of period_search_BOINC.cpp:739-770.
void areanorm(Problem& p) {
    const int nrows = p.nrows;
    std::vector<double> t(p.ndir + 1), f(p.ndir + 1);
    double dth = kPi / (2 * nrows);
    int k = 1;
    t[1] = 0;
    f[1] = 0;
    for (int i = 1; i <= nrows; i++) {
        double dph = kPi / (2 * i);
        for (int j = 0; j <= 4 * i - 1; j++) {
            k++;
            t[k] = i * dth;
            f[k] = j * dph;
        }
    }
    for (int i = nrows - 1; i >= 1; i--) {
        double dph = kPi / (2 * i);
        for (int j = 0; j <= 4 * i - 1; j++) {
            k++;
            t[k] = kPi - i * dth;
            f[k] = j * dph;
        }
    }
    t[k + 1] = kPi;
    f[k + 1] = 0;
    std::vector<double> x(p.ndir + 1), y(p.ndir + 1), z(p.ndir + 1);
    for (int i = 1; i <= p.ndir; i++) {
        double st = std::sin(t[i]);
        x[i] = st * std::cos(f[i]);
        y[i] = st * std::sin(f[i]);
        z[i] = std::cos(t[i]);
    }
    const int F = p.numfac;
    p.nor.assign((size_t)F * 3, 0);
    p.darea.assign(F, 0);
    p.at.assign(F, 0);
    p.af.assign(F, 0);
    for (int i = 0; i < F; i++) {
        const int* v = &p.ifp[(size_t)i * 3];
        double vx[4], vy[4], vz[4], c[4];
        for (int j = 2; j <= 3; j++) {
            vx[j] = x[v[j - 1]] - x[v[0]];
            vy[j] = y[v[j - 1]] - y[v[0]];
            vz[j] = z[v[j - 1]] - z[v[0]];
        }
        c[1] = vy[2] * vz[3] - vy[3] * vz[2];
        c[2] = vz[2] * vx[3] - vz[3] * vx[2];
        c[3] = vx[2] * vy[3] - vx[3] * vy[2];
        double clen2 = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
        double clen = std::sqrt(clen2);
        p.nor[(size_t)i * 3 + 0] = c[1] / clen;
        p.nor[(size_t)i * 3 + 1] = c[2] / clen;
        p.nor[(size_t)i * 3 + 2] = c[3] / clen;
        p.at[i] = std::acos(p.nor[(size_t)i * 3 + 2]);
        p.af[i] = std::atan2(p.nor[(size_t)i * 3 + 1], p.nor[(size_t)i * 3 + 0]);
        p.darea[i] = 0.5 * clen;
    }
}

// sphfunc.c:11-87: Legendre functions and the Dsph basis per facet normal.
void sphfunc(Problem& p) {
    const int F = p.numfac, L = p.lmax, M = p.mmax, L1 = L + 1;
    std::vector<double> ts((size_t)F * L1), tc((size_t)F * L1);
    p.fc.assign((size_t)F * (M + 1), 0);
    p.fs.assign((size_t)F * (M + 1), 0);
    for (int i = 0; i < F; i++) {
        double* Ts = &ts[(size_t)i * L1];
        double* Tc = &tc[(size_t)i * L1];
        Ts[0] = 1;
        Tc[0] = 1;
        if (L >= 1) {
            Ts[1] = std::sin(p.at[i]);
            Tc[1] = std::cos(p.at[i]);
        }
        for (int j = 2; j <= L; j++) {
            Ts[j] = Ts[1] * Ts[j - 1];
            Tc[j] = Tc[1] * Tc[j - 1];
        }
        p.fs[(size_t)i * (M + 1)] = 0;
        p.fc[(size_t)i * (M + 1)] = 1;
        for (int j = 1; j <= M; j++) {
            p.fs[(size_t)i * (M + 1) + j] = std::sin(j * p.af[i]);
            p.fc[(size_t)i * (M + 1) + j] = std::cos(j * p.af[i]);
        }
    }
    // aleg[n][l][m], n,l,m in 0..L (sphfunc.c:44-70)
    std::vector<double> aleg((size_t)L1 * L1 * L1, 0.0);
    auto A = [&](int n, int l, int m) -> double& { return aleg[((size_t)n * L1 + l) * L1 + m]; };
    A(0, 0, 0) = 1;
    if (L >= 1) A(1, 1, 0) = 1;
    for (int l = 1; l <= L; l++) A(0, l, l) = A(0, l - 1, l - 1) * (2 * l - 1);
    for (int m = 0; m <= M; m++)
        for (int l = m + 1; l <= L; l++) {
            int ibot;
            if ((2 * ((l - m) / 2)) == (l - m)) {
                A(0, l, m) = -(l + m - 1) * A(0, l - 2, m) / (1 * (l - m));
                ibot = 2;
            } else {
                ibot = 1;
            }
            if (l != 1)
                for (int n = ibot; n <= l - m; n = n + 2)
                    A(n, l, m) = ((2 * l - 1) * A(n - 1, l - 1, m) - (l + m - 1) * A(n, l - 2, m)) / (1 * (l - m));
        }
    p.pleg.assign((size_t)F * L1 * L1, 0.0);
    p.dsph.assign((size_t)F * p.ncoef, 0.0);
    for (int i = 0; i < F; i++) {
        const double* Ts = &ts[(size_t)i * L1];
        const double* Tc = &tc[(size_t)i * L1];
        int k = 0;
        for (int m = 0; m <= M; m++)
            for (int l = m; l <= L; l++) {
                double& P = p.pleg[((size_t)i * L1 + l) * L1 + m];
                P = 0;
                int ibot = ((2 * ((l - m) / 2)) == (l - m)) ? 0 : 1;
                for (int n = ibot; n <= l - m; n = n + 2) P = P + A(n, l, m) * Tc[n] * Ts[m];
                p.dsph[(size_t)i * p.ncoef + k] = p.fc[(size_t)i * (M + 1) + m] * P;
                k++;
                if (m != 0) {
                    p.dsph[(size_t)i * p.ncoef + k] = p.fs[(size_t)i * (M + 1) + m] * P;
                    k++;
                }
            }
    }
}

// Dense LU solve of the ellipsoid fit's normal equations, the role of the
// reference's ludcmp/lubksb (ludcmp.c:9-68, lubksb.c:3-24), written from the
// algorithm: Crout's LU factorisation P A = L U with implicit row scaling and
// partial pivoting, then forward and back substitution.  The result must
// carry the reference's bits (cg_first seeds every fit), so the choices that
// decide rounding are the reference's: columns are processed left to right,
// each entry's dot product is subtracted term by term in index order, the
// pivot of a column is the row maximising |entry| / (largest |entry| of its
// original row), the last such row on ties, rows are exchanged whole, a zero
// pivot becomes 1e-20, the multipliers below the pivot are formed with the
// pivot's reciprocal, and forward substitution starts at the first nonzero
// right-hand-side entry.
struct LuSolver {
    int n = 0;
    std::vector<double> m;   // row-major; L below the diagonal (unit), U on and above
    std::vector<int> swap;   // row exchanged with row j at column j
    std::vector<double> rinv;  // 1 / (largest |entry| of each row), permuted with the rows

    // Returns 4 (the reference's exit code) when a row is entirely zero.
    int factor(const std::vector<double>& a, int size) {
        n = size;
        m = a;
        swap.assign(n, 0);
        rinv.assign(n, 0.0);
        for (int r = 0; r < n; r++) {
            double largest = 0.0;
            for (int c = 0; c < n; c++) {
                const double v = std::fabs(at(r, c));
                if (v > largest) largest = v;
            }
            if (largest == 0.0) return 4;
            rinv[r] = 1.0 / largest;
        }
        int pivot_row = -1;  // kept across columns, as a column of NaNs leaves it
        for (int col = 0; col < n; col++) {
            for (int r = 0; r < col; r++) at(r, col) = reduced(r, col, r);
            double best = 0.0;
            for (int r = col; r < n; r++) {
                const double v = reduced(r, col, col);
                at(r, col) = v;
                const double score = rinv[r] * std::fabs(v);
                if (score >= best) {
                    best = score;
                    pivot_row = r;
                }
            }
            if (pivot_row != col) {
                for (int c = 0; c < n; c++) std::swap(at(pivot_row, c), at(col, c));
                rinv[pivot_row] = rinv[col];
            }
            swap[col] = pivot_row;
            if (at(col, col) == 0.0) at(col, col) = 1.0e-20;
            if (col + 1 < n) {
                const double inv = 1.0 / at(col, col);
                for (int r = col + 1; r < n; r++) at(r, col) *= inv;
            }
        }
        return 0;
    }

    // Solves A x = rhs in place (rhs has n entries).
    void solve(std::vector<double>& rhs) const {
        int first = -1;  // first row with a nonzero right-hand side after the exchanges
        for (int r = 0; r < n; r++) {
            double v = rhs[swap[r]];
            rhs[swap[r]] = rhs[r];
            if (first >= 0) {
                for (int c = first; c < r; c++) v -= get(r, c) * rhs[c];
            } else if (v != 0.0) {
                first = r;
            }
            rhs[r] = v;
        }
        for (int r = n - 1; r >= 0; r--) {
            double v = rhs[r];
            for (int c = r + 1; c < n; c++) v -= get(r, c) * rhs[c];
            rhs[r] = v / get(r, r);
        }
    }

  private:
    double& at(int r, int c) { return m[(size_t)r * n + c]; }
    double get(int r, int c) const { return m[(size_t)r * n + c]; }
    // entry (r, c) minus the dot product of row r of L and column c of U over
    // the first `terms` indices, subtracted term by term
    double reduced(int r, int c, int terms) const {
        double v = get(r, c);
        for (int k = 0; k < terms; k++) v -= get(r, k) * get(k, c);
        return v;
    }
};

// ellfit.c:11-88: Laplace-series coefficients of the ellipsoid's log
// curvature function (normal equations + LU solve).  The spherical-function
// matrix, its normal matrix and that matrix's LU factors depend on the facet
// grid alone (nrows, lmax, mmax): EllfitGrid holds them, built once per grid
// and shared by every asteroid on it; per asteroid only the ellipsoid's log
// radii, the right-hand side and the substitutions remain.  Every value is
// formed by the same operations in the same order as in one pass, so the
// coefficients are the same bits.
struct EllfitGrid {
    std::vector<double> fmat;  // [F][C]
    LuSolver lu;
    int rc = 0;  // 4: the normal matrix is singular (the reference's exit code)
};

std::shared_ptr<const EllfitGrid> ellfit_grid(const Problem& p) {
    const int F = p.numfac, C = p.ncoef, L1 = p.lmax + 1;
    auto eg = std::make_shared<EllfitGrid>();
    std::vector<double>& fmat = eg->fmat;
    fmat.assign((size_t)F * C, 0.0);
    for (int i = 0; i < F; i++) {
        int n = 0;
        for (int m = 0; m <= p.mmax; m++)
            for (int l = m; l <= p.lmax; l++) {
                double P = p.pleg[((size_t)i * L1 + l) * L1 + m];
                if (m != 0) {
                    fmat[(size_t)i * C + n] = P * std::cos(m * p.af[i]);
                    n++;
                    fmat[(size_t)i * C + n] = P * std::sin(m * p.af[i]);
                    n++;
                } else {
                    fmat[(size_t)i * C + n] = P;
                    n++;
                }
            }
    }
    std::vector<double> fitmat((size_t)C * C);
    for (int i = 0; i < C; i++)
        for (int j = 0; j < C; j++) {
            double s = 0;
            for (int k = 0; k < F; k++) s = s + fmat[(size_t)k * C + i] * fmat[(size_t)k * C + j];
            fitmat[(size_t)i * C + j] = s;
        }
    eg->rc = eg->lu.factor(fitmat, C);
    return eg;
}

int ellfit(Problem& p, const EllfitGrid& eg) {
    const int F = p.numfac, C = p.ncoef;
    const double a = p.a_axis, b = p.b_axis, c = p.c_axis;
    std::vector<double> er(F);
    for (int i = 0; i < F; i++) {
        double st = std::sin(p.at[i]);
        double sum = std::pow(a * st * std::cos(p.af[i]), 2) + std::pow(b * st * std::sin(p.af[i]), 2) +
                     std::pow(c * std::cos(p.at[i]), 2);
        er[i] = 2 * (std::log(a * b * c) - std::log(sum));
    }
    if (eg.rc != 0) return 4;
    std::vector<double> fitvec(C);
    for (int i = 0; i < C; i++) {
        double s = 0;
        for (int j = 0; j < F; j++) s = s + eg.fmat[(size_t)j * C + i] * er[j];
        fitvec[i] = s;
    }
    eg.lu.solve(fitvec);
    p.cg_first = fitvec;
    return 0;
}

}  // namespace

int parse_input(const char* path, Problem& p, std::string& err) {
    FILE* fp = std::fopen(path, "r");
    if (!fp) {
        err = std::string("cannot open input file ") + path;
        return -1;
    }
    int rc = 2;
    std::vector<double> al;
    auto bad = [&](const char* what) {
        err = std::string("malformed input: ") + what;
        return 2;
    };
#define PSB_RD(n, ...)                                                         \
    if (std::fscanf(fp, __VA_ARGS__) < (n)) { rc = bad("header"); goto done; } \
    skip_line(fp);
    PSB_RD(4, "%lf %lf %lf %d", &p.per_start, &p.per_step_coef, &p.per_end, &p.ia_prd)
    PSB_RD(1, "%lf", &p.jd_00)
    PSB_RD(1, "%lf", &p.phi0)
    PSB_RD(1, "%lf", &p.conw)
    PSB_RD(2, "%d %d", &p.lmax, &p.mmax)
    PSB_RD(1, "%d", &p.nrows)
    PSB_RD(2, "%lf %d", &p.par[1], &p.ia_par[1])
    PSB_RD(2, "%lf %d", &p.par[2], &p.ia_par[2])
    PSB_RD(2, "%lf %d", &p.par[3], &p.ia_par[3])
    PSB_RD(2, "%lf %d", &p.cl, &p.ia_cl)
    PSB_RD(1, "%lf", &p.stop_condition)
    PSB_RD(1, "%d", &p.n_iter_min)
    PSB_RD(1, "%lf", &p.alamda_incr)
    PSB_RD(1, "%lf", &p.alamda_start)
#undef PSB_RD
    {
        int nlc = 0;
        if (std::fscanf(fp, "%d", &nlc) != 1 || nlc < 1) {
            rc = bad("number of lightcurves");
            goto done;
        }
        p.lc_points.assign(nlc, 0);
        p.lc_rel.assign(nlc, 0);
        for (int i = 0; i < nlc; i++) {
            int np = 0, flag = 0;
            if (std::fscanf(fp, "%d %d", &np, &flag) != 2 || np < 1) {
                rc = bad("lightcurve header");
                goto done;
            }
            skip_line(fp);
            p.lc_points[i] = np;
            p.lc_rel[i] = 1 - flag;
            for (int j = 0; j < np; j++) {
                double t, b, e0[3], e[3];
                if (std::fscanf(fp, "%lf %lf", &t, &b) != 2 ||
                    std::fscanf(fp, "%lf %lf %lf", &e0[0], &e0[1], &e0[2]) != 3 ||
                    std::fscanf(fp, "%lf %lf %lf", &e[0], &e[1], &e[2]) != 3) {
                    rc = bad("data point");
                    goto done;
                }
                p.tim.push_back(t);
                p.brightness.push_back(b);
                // raw (unnormalised) vectors; finish_raw() normalises
                for (int k = 0; k < 3; k++) p.ee.push_back(e[k]);
                for (int k = 0; k < 3; k++) p.ee0.push_back(e0[k]);
            }
        }
        // weights: `lc weight` pairs to EOF (period_search_BOINC.cpp:420-427)
        std::vector<double> wlc(nlc + 1, -1.0);
        while (std::feof(fp) == 0) {
            int lc = 0;
            double w = 0;
            if (std::fscanf(fp, "%d", &lc) != 1) break;
            if (std::fscanf(fp, "%lf", &w) != 1) break;
            if (lc >= 1 && lc <= nlc) wlc[lc] = w;
        }
        p.n_points = (int)p.tim.size();
        p.weight.assign(p.n_points, 1.0);
        int k = 0;
        for (int i = 0; i < nlc; i++)
            for (int j = 0; j < p.lc_points[i]; j++, k++) p.weight[k] = (wlc[i + 1] == -1) ? 1 : wlc[i + 1];
        // normalise vectors, lightcurve means, phase angles of first points
        // (period_search_BOINC.cpp:343-414)
        double al0 = kPi, al0_abs = kPi;
        int ial0 = -1, ial0_abs = -1;
        p.jd_min = 1e20;
        p.jd_max = -1e40;
        p.onlyrel = 1;
        p.sig.assign(p.n_points, 0);
        int np = 0;
        for (int i = 0; i < nlc; i++) {
            double ave = 0;
            if (p.lc_rel[i] == 0) p.onlyrel = 0;
            for (int j = 0; j < p.lc_points[i]; j++, np++) {
                if (p.tim[np] < p.jd_min) p.jd_min = p.tim[np];
                if (p.tim[np] > p.jd_max) p.jd_max = p.tim[np];
                double* e = &p.ee[(size_t)np * 3];
                double* e0 = &p.ee0[(size_t)np * 3];
                double e0len = std::sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
                double elen = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
                ave += p.brightness[np];
                if (j == 0) {
                    double cos_alpha = (e[0] * e0[0] + e[1] * e0[1] + e[2] * e0[2]) / (elen * e0len);
                    double a = std::acos(cos_alpha);
                    if (a < al0) {
                        al0 = a;
                        ial0 = np;
                    }
                    if ((a < al0_abs) && (p.lc_rel[i] == 0)) {
                        al0_abs = a;
                        ial0_abs = np;
                    }
                }
                for (int c = 0; c < 3; c++) {
                    e[c] = e[c] / elen;
                    e0[c] = e0[c] / e0len;
                }
            }
            ave /= p.lc_points[i];
            for (int j = np - p.lc_points[i]; j < np; j++) p.sig[j] = ave;
        }
        p.jd_0 = p.jd_00;
        if (p.jd_0 <= 0) p.jd_0 = (int)p.jd_min;
        for (int i = 0; i < p.n_points; i++) p.tim[i] = p.tim[i] - p.jd_0;
        p.phi0 = p.phi0 * kDeg2Rad;
        if (p.onlyrel == 0) {
            al0 = al0_abs;
            ial0 = ial0_abs;
        }
        double a = 1.05, b = 1.00, c = 0.95;
        double rfit = std::sqrt(2 * p.sig[ial0] / (0.5 * kPi * (1 + std::cos(al0))));
        p.escl = rfit / std::sqrt((a * b + b * c + a * c) / 3);
        if (p.onlyrel == 0) p.escl *= 0.8;
        rc = finish_from_arrays(p, err);
    }
done:
    std::fclose(fp);
    return rc;
}

int finish_from_arrays(Problem& p, std::string& err) {
    if (p.lmax < 0 || p.lmax > kMaxLm || p.mmax < 0 || p.mmax > p.lmax || p.nrows < 1 || p.nrows > 64) {
        err = "degree/order or number of rows out of range";
        return 2;
    }
    if (p.n_points < 1 || p.per_start <= 0 || p.per_end <= 0 || p.per_step_coef <= 0) {
        err = "empty data or invalid period range";
        return 2;
    }
    p.onlyrel = 1;
    for (int r : p.lc_rel)
        if (r == 0) p.onlyrel = 0;
    p.a_axis = 1.05 * p.escl;
    p.b_axis = 1.00 * p.escl;
    p.c_axis = 0.95 * p.escl;
    p.conw_r = p.conw / p.escl / p.escl;
    return 0;
}

// The facet grid and its spherical-harmonic tables (trifac, areanorm,
// sphfunc) depend only on (nrows, lmax, mmax): computed once per process and
// copied for every further asteroid on the same grid.
std::shared_ptr<const EllfitGrid> grid_tables(Problem& p) {
    struct Tables {
        std::vector<int> ifp;
        std::vector<double> nor, darea, at, af, pleg, dsph, fc, fs;
        std::shared_ptr<const EllfitGrid> ell;
    };
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, Tables> cache;
    const auto key = std::make_tuple(p.nrows, p.lmax, p.mmax);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            const Tables& t = it->second;
            p.ifp = t.ifp;
            p.nor = t.nor;
            p.darea = t.darea;
            p.at = t.at;
            p.af = t.af;
            p.pleg = t.pleg;
            p.dsph = t.dsph;
            p.fc = t.fc;
            p.fs = t.fs;
            return t.ell;
        }
    }
    trifac(p.nrows, p.ifp);
    areanorm(p);
    sphfunc(p);
    auto ell = ellfit_grid(p);
    std::lock_guard<std::mutex> lock(mu);
    if (cache.size() < 16)
        cache.emplace(key, Tables{p.ifp, p.nor, p.darea, p.at, p.af, p.pleg, p.dsph, p.fc, p.fs, ell});
    return ell;
}

int setup_geometry(Problem& p, std::string& err) {
    p.ncoef = 0;
    for (int m = 0; m <= p.mmax; m++)
        for (int l = m; l <= p.lmax; l++) {
            p.ncoef++;
            if (m != 0) p.ncoef++;
        }
    p.numfac = 8 * p.nrows * p.nrows;
    p.ndir = 4 * p.nrows * p.nrows + 2;
    p.nphpar = 3;
    p.ma = p.ncoef + 5 + p.nphpar;
    const std::shared_ptr<const EllfitGrid> ell = grid_tables(p);
    if (ellfit(p, *ell) != 0) {
        err = "singular matrix in the ellipsoid fit (ludcmp)";
        return 4;
    }
    p.freq_start = 1 / p.per_start;
    p.freq_end = 1 / p.per_end;
    p.freq_step = 0.5 / (p.jd_max - p.jd_min) / 24 * p.per_step_coef;
    // free-parameter mask (period_search_BOINC.cpp:789-802, 839)
    const int C = p.ncoef;
    p.ia.assign(p.ma, 0);
    p.ia[C + 0] = 1;  // beta pole
    p.ia[C + 1] = 1;  // lambda pole
    p.ia[C + 2] = p.ia_prd;
    for (int i = 0; i < C; i++) p.ia[i] = 1;
    if (p.onlyrel == 1) p.ia[0] = 0;
    for (int i = 1; i <= p.nphpar; i++) p.ia[C + 2 + i] = p.ia_par[i];
    p.ia[C + 3 + p.nphpar] = p.ia_cl;
    p.ia[C + 4 + p.nphpar] = 0;  // Lommel-Seeliger coefficient fixed
    p.mfit = 0;
    for (int v : p.ia) p.mfit += v ? 1 : 0;
    p.geometry_ready = true;
    return 0;
}

void initial_parameters(const Problem& p, double freq, int m, double* cg) {
    // initial poles (period_search_BOINC.cpp:197-206)
    static const double beta_pole[kNPoles + 1] = {0, 0, 0, 0, 0, 60, 60, 60, -60, -60, -60};
    static const double lambda_pole[kNPoles + 1] = {0, 0, 90, 180, 270, 60, 180, 300, 60, 180, 300};
    const int C = p.ncoef;
    double prd = 1 / freq;
    for (int i = 0; i < C; i++) cg[i] = p.cg_first[i];
    double b = beta_pole[m], l = lambda_pole[m];
    b = 90 - b;
    cg[C + 0] = kDeg2Rad * b;
    cg[C + 1] = kDeg2Rad * l;
    cg[C + 2] = 24 * 2 * kPi / prd;
    for (int i = 1; i <= p.nphpar; i++) cg[C + 2 + i] = p.par[i];
    cg[C + 4 + p.nphpar] = 1;
    cg[C + 3 + p.nphpar] = std::log(p.cl);
}

}  // namespace psb

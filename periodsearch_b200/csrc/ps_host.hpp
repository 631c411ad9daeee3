// Host-side problem description and setup precompute of the B200 period
// scan: what the reference application computes on the host before its fit
// loop (period_search/period_search_BOINC.cpp:277-802): input parsing, data
// normalisation, the triangulated Gaussian sphere, the spherical-harmonic
// tables and the initial ellipsoid.  All of it runs once per asteroid, in
// FP64, in the reference's arithmetic order so that every table the device
// receives equals the reference's bit for bit.
#pragma once

#include <string>
#include <vector>

namespace psb {

constexpr int kMaxLm = 10;      // constants.h:8 (degree/order of the series)
constexpr int kNPoles = 10;     // constants.h:11
constexpr int kMaxNIter = 100;  // constants.h:6
constexpr double kTiny = 1e-8;  // constants.h:10

struct Problem {
    // header (period_search_BOINC.cpp:277-303)
    double per_start = 0, per_step_coef = 0, per_end = 0;
    int ia_prd = 1;
    double jd_00 = 0, phi0 = 0 /* rad */, conw = 0;
    int lmax = 0, mmax = 0, nrows = 0;
    double par[4] = {0, 0, 0, 0};
    int ia_par[4] = {0, 0, 0, 0};
    double cl = 0;
    int ia_cl = 0;
    double stop_condition = 0;
    int n_iter_min = 0;
    double alamda_incr = 0, alamda_start = 0;

    // data (0-based; real lightcurves only, the convexity pseudo-curve is
    // implicit: 3 rows after the last point)
    int n_points = 0;
    std::vector<int> lc_points, lc_rel;
    std::vector<double> tim, ee, ee0, brightness, sig, weight;  // ee: 3 per point
    double jd_min = 0, jd_max = 0, jd_0 = 0, escl = 0;
    double a_axis = 0, b_axis = 0, c_axis = 0;
    int onlyrel = 1;

    // geometry (period_search_BOINC.cpp:497-556)
    int numfac = 0, ndir = 0, ncoef = 0, nphpar = 3, ma = 0, mfit = 0;
    std::vector<double> nor, darea, at, af;  // nor: 3 per facet
    std::vector<int> ifp;                    // 3 per facet, 1-based vertex ids
    std::vector<double> pleg;                // [f][l][m], (lmax+1)^2 per facet
    std::vector<double> fc, fs;              // [f][m], mmax+1 per facet
    std::vector<double> dsph;                // [f][k], ncoef per facet
    std::vector<double> cg_first;            // ncoef
    std::vector<int> ia;                     // ma free/fixed flags
    double freq_start = 0, freq_end = 0, freq_step = 0;
    double conw_r = 0;
    bool geometry_ready = false;

    int n_periods() const { return (int)((freq_start - freq_end) / freq_step) + 1; }
    int n_lc() const { return (int)lc_points.size(); }
};

// Parse period_search_in (period_search_BOINC.cpp:277-485).  Returns 0,
// -1 (cannot open) or 2 (malformed / out of range); err gets a message.
int parse_input(const char* path, Problem& p, std::string& err);

// Fill the derived quantities of a problem given as arrays (everything but
// the geometry).  Returns 0 or 2.
int finish_from_arrays(Problem& p, std::string& err);

// Geometry and parameter mask (period_search_BOINC.cpp:497-556/728-802).
// Returns 0, or 4 when the ellipsoid normal matrix is singular.
int setup_geometry(Problem& p, std::string& err);

// Initial parameter vector of pole m (1..10) at trial frequency freq
// (period_search_BOINC.cpp:819-844); cg has ma entries (0-based).
void initial_parameters(const Problem& p, double freq, int m, double* cg);

}  // namespace psb

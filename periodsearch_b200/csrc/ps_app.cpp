// period_search_b200: drop-in executable for the reference application's
// process contract (period_search/period_search_BOINC.cpp:81-251, 807-945;
// period_search_cuda/period_search/period_search_BOINC.cpp:96-112,579-629).
//
//   period_search_b200 [--device N] [--dir DIR] [--chunk PERIODS]
//
// Reads DIR/period_search_in, writes DIR/period_search_out in the
// reference's 6-column format and checkpoints to DIR/period_search_state
// after every chunk of trial periods ("nlines newConw conw_r", the CUDA
// application's 3-field form; a 1-field CPU-style state is also accepted,
// which re-runs the convexity pre-pass like the CPU application does, and
// the 5-field "nlines newConw conw_r sum_dark_facet ntestperiods" form of the
// pure-CPU and OpenCL applications
// (period_search_pure_cpu_win/period_search/period_search_BOINC.cpp:91,257)
// is read by its first three fields: a pre-pass it interrupted (newConw 0)
// runs again from the start, which ends at the same conw_r).  On restart the
// scan resumes at nlines + 1 and the output is appended.
// Exit codes follow the reference: -1 missing input, 1 output cannot be
// opened, 2 limit exceeded / malformed input, 4 singular ellipsoid fit.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/period_search_b200.h"

static int write_state(const std::string& dir, int nlines, int new_conw, double conw_r) {
    const std::string tmp = dir + "/period_search_state.tmp";
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return 1;
    std::fprintf(f, "%d %d %.17g", nlines, new_conw, conw_r);
    std::fclose(f);
    return std::rename(tmp.c_str(), (dir + "/period_search_state").c_str()) ? 1 : 0;
}

int main(int argc, char** argv) {
    int device = 0, chunk = 0;
    std::string dir = ".";
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc)
            device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--dir") && i + 1 < argc)
            dir = argv[++i];
        else if (!std::strcmp(argv[i], "--chunk") && i + 1 < argc)
            chunk = std::atoi(argv[++i]);
        else {
            std::fprintf(stderr, "usage: %s [--device N] [--dir DIR] [--chunk PERIODS]\n", argv[0]);
            return 2;
        }
    }
    const std::string in = dir + "/period_search_in";
    const std::string outp = dir + "/period_search_out";
    ps_ctx* ctx = nullptr;
    int rc = ps_open_file(in.c_str(), device, PS_FORM_FP64, &ctx);
    if (rc) {
        std::fprintf(stderr, "period_search_b200: %s\n", ps_last_error());
        return rc == PS_ERR_IO ? -1 : rc;
    }
    int nlines = 0, new_conw = 0, have_state = 0;
    double conw_r = 0;
    if (FILE* st = std::fopen((dir + "/period_search_state").c_str(), "r")) {
        int n = std::fscanf(st, "%d %d %lf", &nlines, &new_conw, &conw_r);
        std::fclose(st);
        have_state = n >= 1;
        if (n < 3) new_conw = 0;
    }
    FILE* out = std::fopen(outp.c_str(), have_state ? "a" : "w");
    if (!out) {
        std::fprintf(stderr, "period_search_b200: cannot open %s\n", outp.c_str());
        ps_close(ctx);
        return 1;
    }
    if (have_state && new_conw == 1 && conw_r > 0)
        rc = ps_set_conw_r(ctx, conw_r);
    else
        rc = ps_precalc(ctx, &conw_r);
    if (rc) {
        std::fprintf(stderr, "period_search_b200: %s\n", ps_last_error());
        std::fclose(out);
        ps_close(ctx);
        return rc;
    }
    int ints[8];
    double dbls[8];
    ps_info(ctx, ints, dbls);
    const double escl = dbls[0];
    const int n_max = ps_n_periods(ctx);
    if (chunk <= 0) chunk = 2048;
    std::vector<ps_record> rec;
    char line[256];
    for (int n0 = (have_state ? nlines : 0) + 1; n0 <= n_max; n0 += chunk) {
        const int n1 = n0 + chunk - 1 < n_max ? n0 + chunk - 1 : n_max;
        rec.resize((size_t)(n1 - n0 + 1));
        rc = ps_scan(ctx, n0, n1, rec.data());
        if (rc) {
            std::fprintf(stderr, "period_search_b200: %s\n", ps_last_error());
            std::fclose(out);
            ps_close(ctx);
            return rc;
        }
        for (int n = n0; n <= n1; n++) {
            ps_format_record(&rec[(size_t)(n - n0)], n == 1, conw_r * escl * escl, line, sizeof line);
            std::fputs(line, out);
        }
        std::fflush(out);
        if (write_state(dir, n1, 1, conw_r)) {
            std::fprintf(stderr, "period_search_b200: checkpoint failed\n");
            std::fclose(out);
            ps_close(ctx);
            return 1;
        }
    }
    std::fclose(out);
    ps_close(ctx);
    return 0;
}

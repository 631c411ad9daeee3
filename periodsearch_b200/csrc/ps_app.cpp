// period_search_b200: drop-in executable for the reference application's
// process contract (period_search/period_search_BOINC.cpp:81-251, 807-945;
// period_search_cuda/period_search/period_search_BOINC.cpp:96-112,579-629).
//
//   period_search_b200 [--device N] [--dir DIR] [--chunk PERIODS]
//   period_search_b200 --shard K/N [--device D] [--dir DIR] [--chunk PERIODS]
//   period_search_b200 --merge N [--dir DIR]
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
//
// Sharding (one process per GPU, README.md:12 of the reference: the period
// interval can be divided into smaller parts; its CUDA host strides the range
// by grid, period_search_cuda/period_search/start_CUDA.cu:654).  --shard K/N
// scans the blocks of CHUNK consecutive trial periods whose index b (0-based)
// has b % N == K, after running the convexity pre-pass itself (every shard
// computes the same conw_r), and writes DIR/period_search_out.shard_K_of_N:
// a header line "# shard K N n_periods conw_r escl" and one line per trial
// period "n period_h rms chi2 dark_pct lambda_deg beta_deg" at full
// precision; it checkpoints to DIR/period_search_state.shard_K_of_N
// ("blocks_done 1 conw_r") after every block and resumes from there.
// --merge N joins the N shard files into the single-process
// DIR/period_search_out (the reference's format, the first line carrying
// conw_r escl^2) and DIR/period_search_state ("n_periods 1 conw_r"), the
// same files an unsharded run leaves behind; every period must come from
// exactly one shard and the shards must agree on n_periods, conw_r and escl.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/period_search_b200.h"

static int write_state(const std::string& dir, int nlines, int new_conw, double conw_r,
                       const std::string& suffix = "") {
    const std::string tmp = dir + "/period_search_state" + suffix + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "w");
    if (!f) return 1;
    std::fprintf(f, "%d %d %.17g", nlines, new_conw, conw_r);
    std::fclose(f);
    return std::rename(tmp.c_str(), (dir + "/period_search_state" + suffix).c_str()) ? 1 : 0;
}

static std::string shard_suffix(int k, int n) { return ".shard_" + std::to_string(k) + "_of_" + std::to_string(n); }

// --merge: join the shard files of an N-way sharded scan.
static int merge_shards(const std::string& dir, int nshard) {
    int n_max = -1;
    double conw_r = 0, escl = 0;
    std::map<int, ps_record> recs;
    std::map<int, int> owner;  // period -> shard (a block re-scanned after a resume repeats its lines)
    for (int k = 0; k < nshard; k++) {
        const std::string path = dir + "/period_search_out" + shard_suffix(k, nshard);
        FILE* f = std::fopen(path.c_str(), "r");
        if (!f) {
            std::fprintf(stderr, "period_search_b200: missing shard file %s\n", path.c_str());
            return -1;
        }
        int hk = -1, hn = -1, hmax = -1;
        double hc = 0, he = 0;
        if (std::fscanf(f, " # shard %d %d %d %lf %lf", &hk, &hn, &hmax, &hc, &he) != 5 || hk != k || hn != nshard) {
            std::fprintf(stderr, "period_search_b200: %s: bad shard header\n", path.c_str());
            std::fclose(f);
            return 2;
        }
        if (n_max < 0) {
            n_max = hmax;
            conw_r = hc;
            escl = he;
        } else if (hmax != n_max || hc != conw_r || he != escl) {
            std::fprintf(stderr, "period_search_b200: %s: shards disagree on n_periods/conw_r/escl\n", path.c_str());
            std::fclose(f);
            return 2;
        }
        int n;
        ps_record r;
        while (std::fscanf(f, "%d %lf %lf %lf %lf %lf %lf", &n, &r.period_h, &r.rms, &r.chi2, &r.dark_pct,
                           &r.lambda_deg, &r.beta_deg) == 7) {
            auto it = owner.find(n);
            if (n < 1 || n > n_max || (it != owner.end() && it->second != k)) {
                std::fprintf(stderr, "period_search_b200: %s: period %d out of range or in two shards\n",
                             path.c_str(), n);
                std::fclose(f);
                return 2;
            }
            owner[n] = k;
            recs[n] = r;
        }
        std::fclose(f);
    }
    if ((int)recs.size() != n_max) {
        std::fprintf(stderr, "period_search_b200: shards hold %d of %d periods (unfinished shard?)\n",
                     (int)recs.size(), n_max);
        return 2;
    }
    FILE* out = std::fopen((dir + "/period_search_out").c_str(), "w");
    if (!out) return 1;
    char line[256];
    for (const auto& kv : recs) {
        ps_format_record(&kv.second, kv.first == 1, conw_r * escl * escl, line, sizeof line);
        std::fputs(line, out);
    }
    std::fclose(out);
    return write_state(dir, n_max, 1, conw_r);
}

int main(int argc, char** argv) {
    int device = 0, chunk = 0, shard_k = -1, shard_n = 0, merge_n = 0;
    std::string dir = ".";
    for (int i = 1; i < argc; i++) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc)
            device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--dir") && i + 1 < argc)
            dir = argv[++i];
        else if (!std::strcmp(argv[i], "--chunk") && i + 1 < argc)
            chunk = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--shard") && i + 1 < argc &&
                 std::sscanf(argv[i + 1], "%d/%d", &shard_k, &shard_n) == 2 && shard_n >= 1 && shard_k >= 0 &&
                 shard_k < shard_n)
            i++;
        else if (!std::strcmp(argv[i], "--merge") && i + 1 < argc && (merge_n = std::atoi(argv[i + 1])) >= 1)
            i++;
        else {
            std::fprintf(stderr,
                         "usage: %s [--device N] [--dir DIR] [--chunk PERIODS] [--shard K/N]\n"
                         "       %s --merge N [--dir DIR]\n",
                         argv[0], argv[0]);
            return 2;
        }
    }
    if (merge_n) return merge_shards(dir, merge_n);
    const bool sharded = shard_n > 0;
    const std::string sfx = sharded ? shard_suffix(shard_k, shard_n) : "";
    const std::string in = dir + "/period_search_in";
    const std::string outp = dir + "/period_search_out" + sfx;
    const std::string statep = dir + "/period_search_state" + sfx;
    ps_ctx* ctx = nullptr;
    int rc = ps_open_file(in.c_str(), device, PS_FORM_FP64, &ctx);
    if (rc) {
        std::fprintf(stderr, "period_search_b200: %s\n", ps_last_error());
        return rc == PS_ERR_IO ? -1 : rc;
    }
    int nlines = 0, new_conw = 0, have_state = 0;
    double conw_r = 0;
    if (FILE* st = std::fopen(statep.c_str(), "r")) {
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
    if (sharded) {
        // blocks b = shard_k, shard_k + shard_n, ...; nlines counts the blocks done
        if (!have_state) std::fprintf(out, "# shard %d %d %d %.17g %.17g\n", shard_k, shard_n, n_max, conw_r, escl);
        int done = have_state ? nlines : 0;
        for (long long b = shard_k + (long long)done * shard_n; b * chunk < n_max; b += shard_n) {
            const int n0 = (int)(b * chunk) + 1;
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
                const ps_record& r = rec[(size_t)(n - n0)];
                std::fprintf(out, "%d %.17g %.17g %.17g %.17g %.17g %.17g\n", n, r.period_h, r.rms, r.chi2,
                             r.dark_pct, r.lambda_deg, r.beta_deg);
            }
            std::fflush(out);
            done++;
            if (write_state(dir, done, 1, conw_r, sfx)) {
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

/* A plain C client of the library, as the reference's driver would call it
 * (period_search_BOINC.cpp after parsing period_search_in): open from the
 * input file, run the convexity-weight pre-pass, scan every trial period and
 * print the records in the reference's output format.
 *
 *   scan_client INPUT FORM   (FORM 0 = reference-order FP64, 2 = fast FP64)
 */
#include <stdio.h>
#include <stdlib.h>

#include "period_search_b200.h"

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s INPUT FORM\n", argv[0]);
        return 2;
    }
    ps_ctx* ctx = NULL;
    int rc = ps_open_file(argv[1], 0, atoi(argv[2]), &ctx);
    if (rc != PS_OK) {
        fprintf(stderr, "ps_open_file: %d %s\n", rc, ps_last_error());
        return 1;
    }
    double conw_r = 0;
    rc = ps_precalc(ctx, &conw_r);
    if (rc != PS_OK) {
        fprintf(stderr, "ps_precalc: %d %s\n", rc, ps_last_error());
        ps_close(ctx);
        return 1;
    }
    int ints[16];
    double dbls[16];
    ps_info(ctx, ints, dbls);
    const int n = ps_n_periods(ctx);
    ps_record* rec = (ps_record*)malloc(sizeof(ps_record) * (size_t)n);
    rc = ps_scan(ctx, 1, n, rec);
    if (rc != PS_OK) {
        fprintf(stderr, "ps_scan: %d %s\n", rc, ps_last_error());
        free(rec);
        ps_close(ctx);
        return 1;
    }
    char line[256];
    const double escl = dbls[0];
    for (int i = 0; i < n; i++) {
        ps_format_record(&rec[i], i == 0, conw_r * escl * escl, line, (int)sizeof(line));
        fputs(line, stdout);
    }
    free(rec);
    ps_close(ctx);
    return 0;
}

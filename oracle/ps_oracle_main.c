/* CLI for the CPU oracle (test infrastructure only).
 *
 *   ps_oracle [dir] [n_from n_to [conw_r]]
 *
 * Runs the restated application in dir (default "."): reads
 * period_search_in, writes period_search_out (reference format) and
 * period_search_out.full (the same six values at %.17g).  With n_from/n_to
 * only that slice of trial periods is scanned; with conw_r > 0 the
 * convexity-weight pre-pass is skipped and that value is used, which is how
 * bench.py and the fixture scripts split a scan across host cores.
 */
#include <stdio.h>
#include <stdlib.h>

#include "ps_oracle.h"

int main(int argc, char** argv) {
    const char* dir = argc > 1 ? argv[1] : ".";
    int n_from = argc > 3 ? atoi(argv[2]) : 0;
    int n_to = argc > 3 ? atoi(argv[3]) : 0;
    double conw_r = argc > 4 ? atof(argv[4]) : 0.0;
    int rc = pso_run_app(dir, n_from, n_to, conw_r);
    if (rc) fprintf(stderr, "ps_oracle: exit status %d\n", rc);
    return rc;
}

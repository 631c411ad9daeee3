/* Stand-in for BOINC's MFILE (buffered output file) used to compile the
 * reference period_search application unchanged.
 *
 * Besides writing the formatted text exactly like the original, printf()
 * also records every double argument at full precision ("%.17g") into a
 * side file <output>.full, one line per record.  The reference's own output
 * format (period_search_BOINC.cpp:926-931, "%.8f  %.6f  %.6f %4.1f %4.0f
 * %4.0f") passes six doubles, so the side file carries the same six values
 * unrounded: 24*per_best, dev_best, dev_best^2*(ndata-3), dark (or conw on
 * line 1), lambda, beta.  This is how parity is checked at 1e-9 instead of at
 * the printed digits.
 *
 * Test infrastructure: built into oracle/_ref/, never shipped.
 */
#ifndef PS_REF_SHIM_MFILE_H
#define PS_REF_SHIM_MFILE_H

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

class MFILE {
    FILE* f_ = nullptr;
    FILE* full_ = nullptr;

public:
    int open(const char* path, const char* mode) {
        f_ = std::fopen(path, mode);
        if (!f_) return -1;
        std::string side = std::string(path) + ".full";
        full_ = std::fopen(side.c_str(), mode);
        return full_ ? 0 : -1;
    }
    int printf(const char* fmt, ...) {
        va_list ap;
        va_start(ap, fmt);
        va_list ap2;
        va_copy(ap2, ap);
        int n = std::vfprintf(f_, fmt, ap);
        va_end(ap);
        /* count conversions; every conversion in the reference's record
           format is a floating-point one (%f). */
        int nconv = 0;
        for (const char* p = fmt; *p; ++p) {
            if (*p != '%') continue;
            if (p[1] == '%') { ++p; continue; }
            ++nconv;
        }
        for (int i = 0; i < nconv; ++i) {
            double v = va_arg(ap2, double);
            std::fprintf(full_, i ? " %.17g" : "%.17g", v);
        }
        std::fprintf(full_, "\n");
        va_end(ap2);
        return n;
    }
    int flush() {
        std::fflush(f_);
        std::fflush(full_);
        return 0;
    }
    int close() {
        if (f_) std::fclose(f_);
        if (full_) std::fclose(full_);
        f_ = full_ = nullptr;
        return 0;
    }
};

#endif

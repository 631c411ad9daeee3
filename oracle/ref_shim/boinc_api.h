/* Minimal stand-in for the BOINC client API, used only to compile the
 * reference period_search application (period_search/period_search_BOINC.cpp)
 * unchanged as a standalone oracle binary.  Nothing here touches arithmetic:
 * the reference calls these for file-name resolution, progress and
 * checkpoint timing only (period_search_BOINC.cpp:220-251, 806-810, 932-936).
 *
 * Test infrastructure: built into oracle/_ref/, never shipped.
 */
#ifndef PS_REF_SHIM_BOINC_API_H
#define PS_REF_SHIM_BOINC_API_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

inline int boinc_init() { return 0; }
inline int boinc_is_standalone() { return 0; }
inline int boinc_resolve_filename(const char* name, char* out, int len) {
    std::snprintf(out, (size_t)len, "%s", name);
    return 0;
}
inline int boinc_resolve_filename_s(const char* name, std::string& out) {
    out = name;
    return 0;
}
inline FILE* boinc_fopen(const char* path, const char* mode) { return std::fopen(path, mode); }
inline int boinc_rename(const char* from, const char* to) { return std::rename(from, to); }
inline int boinc_fraction_done(double) { return 0; }
/* Never checkpoint: the oracle run is one uninterrupted scan. */
inline int boinc_time_to_checkpoint() { return 0; }
inline int boinc_checkpoint_completed() { return 0; }
inline int boinc_finish(int status) { std::exit(status); return status; }
inline char* boinc_msg_prefix(char* buf, int len) {
    if (len > 0) buf[0] = 0;
    return buf;
}

#endif

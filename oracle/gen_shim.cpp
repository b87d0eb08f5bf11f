// Support for a standalone build of the workload generator
// (adabool_b200/csrc/abf_gen.cpp) into oracle/libwgen.so. TEST AND BASELINE
// INFRASTRUCTURE ONLY: the reference's CPU timing leg of bench.py generates
// the same seeded workload through this library, so that its process loads
// no library of the product. The generator source is shared, not copied;
// this file supplies the two helpers it takes from the product library.
#include <string>
#include <thread>

#include "../adabool_b200/csrc/abf_internal.h"

namespace {
thread_local std::string g_err;
}

namespace abf {
abf_status fail(abf_status s, const std::string& msg) {
    g_err = msg;
    return s;
}
int resolve_threads(int n) {
    if (n > 0) return n;
    const unsigned hc = std::thread::hardware_concurrency();
    return hc ? int(hc) : 1;
}
}  // namespace abf

extern "C" const char* wgen_last_error_string(void) { return g_err.c_str(); }

// Status strings, version and per-thread error text of the s1b C ABI.
#include <cstdio>
#include <cstring>

#include "s1b.h"
#include "s1b_internal.h"

namespace {
thread_local char g_last_error[512] = "";
}

int s1b_fail(int status, const char *msg) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
  return status;
}

extern "C" const char *s1b_last_error(void) { return g_last_error; }

extern "C" int s1b_version(void) { return 100; }

extern "C" size_t s1b_sizeof_burst_plan(void) { return sizeof(s1b_burst_plan_t); }
extern "C" size_t s1b_sizeof_orbit_poly(void) { return sizeof(s1b_orbit_poly_t); }

extern "C" const char *s1b_status_string(int status) {
  switch (status) {
    case S1B_OK: return "ok";
    case S1B_ERR_INVALID_ARGUMENT: return "invalid argument";
    case S1B_ERR_CUDA: return "CUDA error";
    case S1B_ERR_TOO_LARGE: return "size exceeds a supported maximum";
    case S1B_ERR_EMPTY: return "empty region: nothing to compute";
    case S1B_ERR_NO_DEVICE: return "no CUDA device";
    case S1B_ERR_UNSUPPORTED: return "unsupported parameter";
    default: return "unknown status";
  }
}

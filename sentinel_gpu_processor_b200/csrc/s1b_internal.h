// Internal helpers shared by the host planner and the CUDA kernels.
#ifndef S1B_INTERNAL_H
#define S1B_INTERNAL_H

#include <stdint.h>

#include "s1b.h"

#ifdef __CUDACC__
#define S1B_HD __host__ __device__ __forceinline__
#else
#define S1B_HD inline
#endif

// Record a failure message for s1b_last_error() and return `status`.
int s1b_fail(int status, const char *msg);

// Window index (1..n_win) of the orbit polynomial used at time t: the
// reference's truncating selector int((t - t0) / dt) clamped to [1, n-3]
// (csrc/src/orbit.cu:229-232).
S1B_HD int s1b_orbit_window(const s1b_orbit_poly_t &p, double t) {
  double q = (t - p.t0) * p.inv_dt;
  // clamp before the conversion so that huge |q| (or NaN) cannot overflow int
  if (!(q >= 1.0)) q = 1.0;
  if (q > (double)p.n_win) q = (double)p.n_win;
  return (int)q;
}

#endif

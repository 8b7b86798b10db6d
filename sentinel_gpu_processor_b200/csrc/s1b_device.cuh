// Device helpers: error plumbing, phase wrapping, orbit polynomial evaluation.
#ifndef S1B_DEVICE_CUH
#define S1B_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "s1b.h"
#include "s1b_internal.h"

#define S1B_CUDA_TRY(expr)                                           \
  do {                                                               \
    cudaError_t e_ = (expr);                                         \
    if (e_ != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

// Check the launch that was just issued.
inline int s1b_launch_status() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  return S1B_OK;
}

constexpr double kPiD = 3.14159265358979323846;
constexpr double kSolD = 299792458.0;

// Reduce an FP64 phase to [-pi, pi] and return it as float.
// Cody-Waite reduction (W. J. Cody, W. Waite, "Software Manual for the
// Elementary Functions", 1980): 2 pi is split into HI + MID + LO where HI
// and MID carry 27 significant bits, so k*HI and k*MID are exact for
// |k| < 2^26 (phases up to ~4e8 rad); the constants were generated from
// pi evaluated to 60 decimal digits with Machin's formula.
__device__ __forceinline__ float wrap_phase(double x) {
  const double k = rint(x * 0x1.45f306dc9c883p-3);  // 1 / (2 pi)
  double r = fma(-k, 0x1.921fb54000000p+2, x);
  r = fma(-k, 0x1.10b4610000000p-28, r);
  r = fma(-k, 0x1.a62633145c06ep-56, r);
  return (float)r;
}

// Unit phasor exp(i x) of an FP64 phase.
__device__ __forceinline__ float2 phasor(double x) {
  float s, c;
  sincosf(wrap_phase(x), &s, &c);
  return make_float2(c, s);
}

// Unit phasor exp(i pi h) of an FP64 phase h given in half-cycles (units of
// pi rad).  h - 2 rint(h / 2) is exact in FP64 for |h| < 2^52, so the only
// rounding is the final float conversion of a value in [-1, 1] (<= 6e-8).
__device__ __forceinline__ float2 phasor_pi(double h) {
  const double r = fma(-2.0, rint(0.5 * h), h);
  float s, c;
  sincospif((float)r, &s, &c);
  return make_float2(c, s);
}

// exp(i pi h) as phasor_pi, rotated with the hardware sine/cosine
// approximations (__sincosf: absolute error ~4e-7 on [-pi, pi]).  For
// per-pixel phases that are not accumulated further.
__device__ __forceinline__ float2 phasor_pi_fast(double h) {
  const double r = fma(-2.0, rint(0.5 * h), h);
  float s, c;
  __sincosf((float)r * 3.14159265f, &s, &c);
  return make_float2(c, s);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Position, velocity and acceleration of the orbit at time t from the
// window polynomial: Horner's scheme carrying the first two derivatives.
struct OrbitState {
  double x[3], v[3], a[3];
};

__device__ __forceinline__ void orbit_eval(const s1b_orbit_poly_t &P, double t, OrbitState &s) {
  const int w = s1b_orbit_window(P, t) - 1;
  const double tau = t - P.tc[w];
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const double *c = P.c[w][comp];
    double f = c[7], d = 0.0, dd = 0.0;
#pragma unroll
    for (int k = 6; k >= 0; --k) {
      dd = fma(dd, tau, d);
      d = fma(d, tau, f);
      f = fma(f, tau, c[k]);
    }
    s.x[comp] = f;
    s.v[comp] = d;
    s.a[comp] = 2.0 * dd;
  }
}

// Zero-Doppler time of ECEF point p: Newton on f(t) = (p - X(t)) . V(t)
// with the exact derivative f' = -|V|^2 + (p - X) . A.  The reference
// iterates with f' ~ -|V|^2 (csrc/src/orbit.cu:259-274), which converges
// linearly (7-11 steps from the burst centre); both stop once a step is
// below `tol` and solve the same equation, so the roots agree to far below
// the 5e-9 s tolerance.  Returns the number of steps taken; dr = p - X(t).
__device__ __forceinline__ int zero_doppler(const s1b_orbit_poly_t &P, const double p[3],
                                            double &t, OrbitState &s, double dr[3],
                                            int max_iter = 51, double tol = 5.0e-9) {
  int it = 0;
  for (; it < max_iter; ++it) {
    double fn = 0.0, fp = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      dr[i] = p[i] - s.x[i];
      fn = fma(dr[i], s.v[i], fn);
      fp = fma(dr[i], s.a[i], fp);
      fp = fma(-s.v[i], s.v[i], fp);
    }
    const double step = fn / fp;
    t -= step;
    if (fabs(step) < tol) {
      // last correction is below tolerance: move the state to the new time
      // to first order instead of re-evaluating the polynomial
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        s.x[i] = fma(-step, s.v[i], s.x[i]);
        dr[i] = p[i] - s.x[i];
      }
      return it + 1;
    }
    orbit_eval(P, t, s);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) dr[i] = p[i] - s.x[i];
  return it;
}

// Cubic expansion of the orbit about t0 (position, velocity, acceleration,
// jerk of the window polynomial).  A column walk solves its first pixel on
// the polynomial and the following ones on the expansion: over a segment of
// 16 lines (|t - t0| <= ~0.035 s) the dropped fourth-order term is
// snap |dt|^4 / 24 < 1e-12 m for an orbit (snap ~ omega^4 r ~ 1e-5 m/s^4),
// and each Newton step costs 18 FMA instead of a 54-FMA polynomial pass.
struct OrbitCubic {
  double t0, x[3], v[3], a[3], j[3];
};

// Position and the first three derivatives of the window polynomial at t.
__device__ __forceinline__ void orbit_cubic(const s1b_orbit_poly_t &P, double t, OrbitCubic &o) {
  const int w = s1b_orbit_window(P, t) - 1;
  const double tau = t - P.tc[w];
  o.t0 = t;
#pragma unroll
  for (int comp = 0; comp < 3; ++comp) {
    const double *c = P.c[w][comp];
    double f = c[7], d = 0.0, dd = 0.0, ddd = 0.0;
#pragma unroll
    for (int k = 6; k >= 0; --k) {
      ddd = fma(ddd, tau, dd);
      dd = fma(dd, tau, d);
      d = fma(d, tau, f);
      f = fma(f, tau, c[k]);
    }
    o.x[comp] = f;
    o.v[comp] = d;
    o.a[comp] = 2.0 * dd;
    o.j[comp] = 6.0 * ddd;
  }
}

// Zero-Doppler Newton (same iteration and stopping rule as zero_doppler)
// with the orbit state taken from the cubic expansion.
__device__ __forceinline__ void zero_doppler_cubic(const OrbitCubic &o, const double p[3], double &t, double dr[3]) {
  for (int it = 0; it < 51; ++it) {
    const double h = t - o.t0;
    double fn = 0.0, fp = 0.0, v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double a = fma(o.j[i], h, o.a[i]);
      v[i] = fma(fma(0.5 * o.j[i], h, o.a[i]), h, o.v[i]);
      const double x = fma(fma(fma(o.j[i] * (1.0 / 6.0), h, 0.5 * o.a[i]), h, o.v[i]), h, o.x[i]);
      dr[i] = p[i] - x;
      fn = fma(dr[i], v[i], fn);
      fp = fma(dr[i], a, fp);
      fp = fma(-v[i], v[i], fp);
    }
    const double step = fn / fp;
    t -= step;
    if (fabs(step) < 5.0e-9) {
#pragma unroll
      for (int i = 0; i < 3; ++i) dr[i] = fma(step, v[i], dr[i]);
      return;
    }
  }
}

// zero_doppler_cubic with a fixed reciprocal derivative (chord Newton).
__device__ __forceinline__ void zero_doppler_cubic_chord(const OrbitCubic &o, const double p[3], double &t,
                                                         double dr[3], double inv_fp) {
  for (int it = 0; it < 51; ++it) {
    const double h = t - o.t0;
    double fn = 0.0, v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      v[i] = fma(fma(0.5 * o.j[i], h, o.a[i]), h, o.v[i]);
      const double x = fma(fma(fma(o.j[i] * (1.0 / 6.0), h, 0.5 * o.a[i]), h, o.v[i]), h, o.x[i]);
      dr[i] = p[i] - x;
      fn = fma(dr[i], v[i], fn);
    }
    const double step = fn * inv_fp;
    t -= step;
    if (fabs(step) < 5.0e-9) {
#pragma unroll
      for (int i = 0; i < 3; ++i) dr[i] = fma(step, v[i], dr[i]);
      return;
    }
  }
}

#endif

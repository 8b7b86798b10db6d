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

// int -> double from an integer add and an FP64 add: adding x to the bit
// pattern of 1.5 * 2^52 adds it to the value (exact for |x| < 2^51), and
// subtracting 1.5 * 2^52 leaves x exactly.  The same value as (double)x.
__device__ __forceinline__ double i32_to_f64(int x) {
  return __longlong_as_double(0x4338000000000000LL + (long long)x) - 6755399441055744.0;
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

// Zero-Doppler model of a patch of ground points about t0, from the cubic
// orbit expansion (x, v, a, j at t0) and u(h) = v h + a h^2/2 + j h^3/6:
//   f(h) = (p - x(t0 + h)) . v(t0 + h) = d.u'(h) - (1/2) d|u|^2/dh,  d = p - x
//        = c0 + c1 h + c2 h^2 + c3 h^3 + O(h^4)
//   c0 = d.v,  c1 = d.a - |v|^2,  c2 = d.j/2 - (3/2) v.a,
//   c3 = -(|a|^2/2 + (2/3) v.j)  (the same for every point),
// and, since d|p - x|^2/dh = -2 f,
//   |p - x(t0 + h)|^2 = |d|^2 - h (2 c0 + h (c1 + h ((2/3) c2 + h c3 / 2))).
// The dropped h^4 term of f is (5/12)(a.j) h^4 < 5e-5 for |h| < 0.2 s
// (a time error below 1e-12 s).  A point costs four dot products of d; each
// Newton step three FMA.
struct ZeroDopplerPatch {
  double t0, x[3], v[3], a[3], jh[3];  // jh = j / 2
  double vv, k2, c3;                   // |v|^2, (3/2) v.a, c3
  double inv_c1;                       // 1 / f'(0) at the patch's own centre point (chord slope)
};

__device__ __forceinline__ void zero_doppler_patch(const OrbitCubic &o, ZeroDopplerPatch &z) {
  z.t0 = o.t0;
  double vv = 0.0, va = 0.0, aa = 0.0, vj = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    z.x[i] = o.x[i];
    z.v[i] = o.v[i];
    z.a[i] = o.a[i];
    z.jh[i] = 0.5 * o.j[i];
    vv = fma(o.v[i], o.v[i], vv);
    va = fma(o.v[i], o.a[i], va);
    aa = fma(o.a[i], o.a[i], aa);
    vj = fma(o.v[i], o.j[i], vj);
  }
  z.vv = vv;
  z.k2 = 1.5 * va;
  z.c3 = -(0.5 * aa + (2.0 / 3.0) * vj);
}

// Per-point coefficients of the patch model: c0, c1, c2 and |d|^2.
struct ZeroDopplerPoint {
  double c0, c1, c2, dd;
};

__device__ __forceinline__ ZeroDopplerPoint zero_doppler_point(const ZeroDopplerPatch &z, const double p[3]) {
  const double d0 = p[0] - z.x[0], d1 = p[1] - z.x[1], d2 = p[2] - z.x[2];
  ZeroDopplerPoint q;
  q.c0 = fma(d0, z.v[0], fma(d1, z.v[1], d2 * z.v[2]));
  q.c1 = fma(d0, z.a[0], fma(d1, z.a[1], fma(d2, z.a[2], -z.vv)));
  q.c2 = fma(d0, z.jh[0], fma(d1, z.jh[1], fma(d2, z.jh[2], -z.k2)));
  q.dd = fma(d0, d0, fma(d1, d1, d2 * d2));
  return q;
}

// Chord Newton on f(h) = 0 from the seed h with the fixed reciprocal slope
// inv_c1 (= 1 / f'(0)); stops as the reference's iteration does, once a step
// is below 5e-9 s (csrc/src/orbit.cu:259-274).  Returns the squared range.
__device__ __forceinline__ double zero_doppler_solve(const ZeroDopplerPoint &q, double c3, double inv_c1,
                                                     double &h) {
  for (int it = 0; it < 51; ++it) {
    const double f = fma(fma(fma(c3, h, q.c2), h, q.c1), h, q.c0);
    const double step = f * inv_c1;
    h -= step;
    if (fabs(step) < 5.0e-9) break;
  }
  return fma(-h, fma(fma(fma(0.5 * c3, h, (2.0 / 3.0) * q.c2), h, q.c1), h, 2.0 * q.c0), q.dd);
}

// zero_doppler_solve as straight-line code: two chord-Newton steps from the
// seed, then the same stopping test (|step| < 5e-9 s), with further steps
// only when the second step is not yet below it and `more` is set.  From a
// seed within ~1e-6 s of the root and a slope within 1e-3 of f' the second
// step is below 1e-9 s, so the common path has no data-dependent branch and
// independent solves (the two bursts of a pair) interleave.  Returns the
// squared range.
__device__ __forceinline__ double zero_doppler_solve2(const ZeroDopplerPoint &q, double c3, double inv_c1,
                                                      double &h, bool more) {
  double f = fma(fma(fma(c3, h, q.c2), h, q.c1), h, q.c0);
  double step = f * inv_c1;
  h -= step;
  f = fma(fma(fma(c3, h, q.c2), h, q.c1), h, q.c0);
  step = f * inv_c1;
  h -= step;
  if (more && fabs(step) >= 5.0e-9) {
    for (int it = 2; it < 51; ++it) {
      f = fma(fma(fma(c3, h, q.c2), h, q.c1), h, q.c0);
      step = f * inv_c1;
      h -= step;
      if (fabs(step) < 5.0e-9) break;
    }
  }
  return fma(-h, fma(fma(fma(0.5 * c3, h, (2.0 / 3.0) * q.c2), h, q.c1), h, 2.0 * q.c0), q.dd);
}

// exp(i pi x) of an FP32 phase in half-cycles (|x| < 2^22): the reduction
// x - 2 rint(x / 2) is exact, then the hardware sine and cosine of the
// reduced angle (absolute error ~4e-7 on [-pi, pi]).
__device__ __forceinline__ float2 phasor_pi_f(float x) {
  const float r = fmaf(-2.f, rintf(0.5f * x), x);
  float s, c;
  __sincosf(r * 3.14159265f, &s, &c);
  return make_float2(c, s);
}

// exp(i pi x) for the small rotations between neighbouring burst columns
// (|pi x| <= 0.1: Taylor series of cos and sin to the fourth and fifth
// order, truncation error < 1e-7), larger angles through phasor_pi_f.
__device__ __forceinline__ float2 rotation_pi_f(float x) {
  const float a = x * 3.14159265f;
  if (fabsf(a) > 0.1f) return phasor_pi_f(x);
  const float a2 = a * a;
  return make_float2(fmaf(a2, fmaf(a2, 1.f / 24.f, -0.5f), 1.f), a * fmaf(a2, -1.f / 6.f, 1.f));
}

// sqrt(s) for normal s in float range, to FP64 accuracy: Heron's method
// (Newton on r^2 = s) from the FP32 estimate y ~ 1/sqrt(s) with y held fixed,
// r <- r + (s - r^2) y / 2.  With y = (1 + e)/sqrt(s), r = s y has relative
// error e, the first step leaves 1.5 e^2 and the second 1.5 e^3 (e < 3e-7:
// below 1e-19), so the result is within an ulp of the rounded square root.
__device__ __forceinline__ double sqrt_heron(double s) {
  const float y = rsqrtf((float)s);
  const double hy = 0.5 * (double)y;
  double r = s * (double)y;
  r = fma(fma(-r, r, s), hy, r);
  return fma(fma(-r, r, s), hy, r);
}

// 1 / x for normal x in float range, to FP64 accuracy: Newton's iteration
// r <- r + r (1 - x r) from an FP32 estimate; each step squares the relative
// error (3e-7 -> 1e-13 -> 1e-26).
__device__ __forceinline__ double rcp_newton(double x) {
  double r = (double)__fdividef(1.0f, (float)x);
  r = fma(r, fma(-x, r, 1.0), r);
  return fma(r, fma(-x, r, 1.0), r);
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

// One full-resolution pixel pair into the multilook sums of crossmul:
// conj(r) * s (sario.cu:207-208) and both powers, each added in one
// expression so that every kernel summing them rounds alike.
__device__ __forceinline__ void xm_accumulate(float2 r, float2 s, float &ir, float &ii, float &p1, float &p2) {
  ir += r.x * s.x + r.y * s.y;
  ii += -r.y * s.x + r.x * s.y;
  p1 += r.x * r.x + r.y * r.y;
  p2 += s.x * s.x + s.y * s.y;
}

#endif

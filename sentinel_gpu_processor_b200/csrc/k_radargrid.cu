// Radar-grid coregistration on sm_100a: secondary sample offsets from
// float64 lat/lon/height rasters of the reference grid, TOPS-aware resampling
// of the secondary onto the reference grid (8-tap windowed sinc or
// bilinear), and boxcar coherence at full resolution (a register row walk
// for windows up to 5 x 5, TMA-staged halo tiles for 7 x 7 and 9 x 9).
//
// The reference geocodes every SLC onto a lat/lon grid instead
// (csrc/src/geo2rdr.cu:170-248); this mode has no reference counterpart.  It
// reuses the reference's geometry (orbit interpolant, zero-Doppler
// condition, range/azimuth sample formulas geo2rdr.cu:205-207) and its TOPS
// phase (geo2rdr.cu:151-152, 210-219).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <mutex>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_internal.h"

namespace {

constexpr double kRaD = 6378137.0;
constexpr double kRe2D = 0.00669437999015;

// -------------------------------------------------------------- offsets
// Same column walk as the geocoding kernel: thread = reference column, 16
// rows per thread; the first row solves on the window polynomial from the
// burst centre, the others on the cubic expansion there (OrbitCubic).
constexpr int O_TX = 128, O_RY = 16;

// ECEF position of a geodetic point and the geodetic up vector dp/dh.
__device__ __forceinline__ void llh_ecef(double lat_deg, double lon_deg, double h, double p[3], double up[3]) {
  double sl, cl, so, co;
  sincospi(lat_deg * (1.0 / 180.0), &sl, &cl);
  sincospi(lon_deg * (1.0 / 180.0), &so, &co);
  const double re = kRaD * rsqrt(1. - kRe2D * sl * sl);  // orbit.cu:27-30
  p[0] = (re + h) * cl * co;
  p[1] = (re + h) * cl * so;
  p[2] = (re * (1 - kRe2D) + h) * sl;
  up[0] = cl * co;
  up[1] = cl * so;
  up[2] = sl;
}

// Height sensitivity of the secondary offsets of a reference-grid pixel.  A
// height error moves the ground point along the reference's zero-Doppler
// iso-range circle: dp = (rhat_r x V_r) / (up . (rhat_r x V_r)) per metre
// (range to and Doppler of the reference unchanged, geodetic height +1).
// The secondary then sees f(t, p) = (p - X(t)).V(t) = 0 move by dt/dh =
// (V.dp) / (|V|^2 - dr.A) and its range by rhat.(dp - V dt/dh).
__device__ __forceinline__ void height_sensitivity(const OrbitCubic &o, double t, const double dr[3],
                                                   const double up[3], const double rr[3], const double vr[3],
                                                   double &dt_dh, double &dR_dh) {
  // c = dr_ref x V_ref (the unit of dr_ref cancels in the ratio)
  const double c0 = rr[1] * vr[2] - rr[2] * vr[1];
  const double c1 = rr[2] * vr[0] - rr[0] * vr[2];
  const double c2 = rr[0] * vr[1] - rr[1] * vr[0];
  const double inv = 1.0 / (up[0] * c0 + up[1] * c1 + up[2] * c2);
  const double dp[3] = {c0 * inv, c1 * inv, c2 * inv};
  const double h = t - o.t0;
  double v[3], a[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    a[i] = fma(o.j[i], h, o.a[i]);
    v[i] = fma(fma(0.5 * o.j[i], h, o.a[i]), h, o.v[i]);
  }
  const double vn = v[0] * dp[0] + v[1] * dp[1] + v[2] * dp[2];
  const double den = (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - (dr[0] * a[0] + dr[1] * a[1] + dr[2] * a[2]);
  dt_dh = vn / den;
  const double inv_r = rsqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
  dR_dh = inv_r * (dr[0] * (dp[0] - v[0] * dt_dh) + dr[1] * (dp[1] - v[1] * dt_dh) + dr[2] * (dp[2] - v[2] * dt_dh));
}

// Reference satellite state for the sensitivities: the reference pixel
// (row, col) is the reference's own sample, so its zero-Doppler time is
// tstart + row dtaz and no Newton is needed.
struct RefOrbit {
  s1b_orbit_poly_t orbit;
  double tstart, dtaz;
};

template <bool kSens>
__global__ __launch_bounds__(O_TX) void offsets_kernel(const __grid_constant__ s1b_burst_plan_t P,
                                                       const __grid_constant__ RefOrbit R,
                                                       const double *__restrict__ lat,
                                                       const double *__restrict__ lon,
                                                       const double *__restrict__ hgt, int L, int S,
                                                       float *__restrict__ az_off,
                                                       float *__restrict__ rg_off,
                                                       float *__restrict__ daz_dh,
                                                       float *__restrict__ drg_dh) {
  const int col = blockIdx.x * O_TX + threadIdx.x;
  const int row0 = blockIdx.y * O_RY;
  if (col >= S) return;
  const double inv_dmrg = 1.0 / P.dmrg, prf = 1.0 / P.dtaz;
  const int rmax = min(O_RY, L - row0);
  size_t i = (size_t)row0 * S + col;
  double la = __ldcs(lat + i), lo = __ldcs(lon + i), h = __ldcs(hgt + i);
  double p[3], dr[3], up[3];
  // first row: from the burst centre on the window polynomial
  double t = P.tmid;
  {
    OrbitState st;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      st.x[k] = P.xmid[k];
      st.v[k] = P.vmid[k];
      st.a[k] = P.amid[k];
    }
    llh_ecef(la, lo, h, p, up);
    zero_doppler(P.orbit, p, t, st, dr);
  }
  OrbitCubic o;
  orbit_cubic(P.orbit, t, o);
  double tprev = t - P.dtaz;
  // the next row's inputs are loaded one row ahead
  if (rmax > 1) {
    la = __ldcs(lat + i + S);
    lo = __ldcs(lon + i + S);
    h = __ldcs(hgt + i + S);
  }
  for (int r = 0;;) {
    const double rng = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    // residuals relative to the pixel index keep float32 at ~1e-5 px
    __stcs(az_off + i, (float)((t - P.tstart) * prf - (row0 + r)));
    __stcs(rg_off + i, (float)((rng - P.rngstart) * inv_dmrg - col));
    if (kSens) {
      OrbitState rs;
      orbit_eval(R.orbit, R.tstart + (row0 + r) * R.dtaz, rs);
      const double rr[3] = {p[0] - rs.x[0], p[1] - rs.x[1], p[2] - rs.x[2]};
      double dt_dh, dR_dh;
      height_sensitivity(o, t, dr, up, rr, rs.v, dt_dh, dR_dh);
      __stcs(daz_dh + i, (float)(dt_dh * prf));
      __stcs(drg_dh + i, (float)(dR_dh * inv_dmrg));
    }
    if (++r >= rmax) break;
    i += S;
    llh_ecef(la, lo, h, p, up);
    if (r + 1 < rmax) {
      la = __ldcs(lat + i + S);
      lo = __ldcs(lon + i + S);
      h = __ldcs(hgt + i + S);
    }
    // seed: linear extrapolation down the column
    const double tn = 2.0 * t - tprev;
    tprev = t;
    t = tn;
    zero_doppler_cubic(o, p, t, dr);
  }
}

// ------------------------------------------------ TMA / mbarrier helpers
// Bounded wait: try_wait suspends for a hardware time slice per call; after
// kSpinLimit calls the caller treats the copy as lost.
constexpr uint32_t kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit = kSpinLimit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ------------------------------------------------------------- resample
// Output tile 64 columns x 16 rows; 256 threads = 64 columns x 4 row groups
// of 4 rows.  The tile's secondary window (its sample coordinates plus the
// kernel support) is staged deramped in shared memory.  A thread whose four
// outputs sit on consecutive secondary lines of one column range (the usual
// case: offsets vary slowly) reads each of the 11 tap rows once for all four
// outputs; others, and tiles whose window exceeds the stage, take the
// per-output path.  Complex x real multiply-adds use the paired FP32 FMA.
constexpr int R_TX = 64, R_TY = 4, R_RPT = 4;  // columns, row groups, rows per thread
constexpr int R_TH = R_TY * R_RPT;             // 16 tile rows
constexpr int R_WROWS = 32, R_WCOLS = 96;
constexpr int SINC_BINS = 1024;

// Normalised 8-tap windowed-sinc weights at SINC_BINS + 1 fractions f = b /
// SINC_BINS (taps k = -3..4 at distance k - f: sinc(k - f) (0.5 + 0.5
// cos(pi (k - f) / 4)), divided by their sum); evaluated by the host in
// double precision, read with linear interpolation in the fraction.
__device__ __align__(16) float g_sinc_table[(SINC_BINS + 1) * 8];
std::mutex g_sinc_mu;
bool g_sinc_ready[64] = {};

int ensure_sinc_table() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_resample: device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_sinc_mu);
  if (g_sinc_ready[dev]) return S1B_OK;
  static float host[(SINC_BINS + 1) * 8];
  for (int b = 0; b <= SINC_BINS; ++b) {
    const double f = (double)b / SINC_BINS;
    double w[8], sum = 0.0;
    for (int k = 0; k < 8; ++k) {
      const double x = (k - 3) - f;
      const double sc = x == 0.0 ? 1.0 : sin(kPiD * x) / (kPiD * x);
      w[k] = sc * (0.5 + 0.5 * cos(kPiD * x / 4.0));
      sum += w[k];
    }
    for (int k = 0; k < 8; ++k) host[b * 8 + k] = (float)(w[k] / sum);
  }
  e = cudaMemcpyToSymbol(g_sinc_table, host, sizeof(host));
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  g_sinc_ready[dev] = true;
  return S1B_OK;
}

__device__ __forceinline__ void sinc8_weights(float f, float w[8]) {
  const float pos = f * SINC_BINS;
  const int b = min((int)pos, SINC_BINS - 1);
  const float t = pos - (float)b;
  const float4 *T = reinterpret_cast<const float4 *>(g_sinc_table) + 2 * b;
  const float4 a0 = __ldg(T), a1 = __ldg(T + 1), b0 = __ldg(T + 2), b1 = __ldg(T + 3);
  w[0] = fmaf(t, b0.x - a0.x, a0.x);
  w[1] = fmaf(t, b0.y - a0.y, a0.y);
  w[2] = fmaf(t, b0.z - a0.z, a0.z);
  w[3] = fmaf(t, b0.w - a0.w, a0.w);
  w[4] = fmaf(t, b1.x - a1.x, a1.x);
  w[5] = fmaf(t, b1.y - a1.y, a1.y);
  w[6] = fmaf(t, b1.z - a1.z, a1.z);
  w[7] = fmaf(t, b1.w - a1.w, a1.w);
}

// TOPS coefficients at a continuous range sample, the phase in half-cycles
// (units of pi rad): -kt, so that the deramp phase is pi (-kt) (eta -
// etaref)^2, and etaref (geo2rdr.cu:533-541 with the sample index
// fractional).  One division serves kt = ka ks / (ka - ks) and fnc / ka.
__device__ __forceinline__ void tops_range(const s1b_burst_plan_t &P, double rs, double &mkt, double &etaref) {
  const double tr = P.slant_range_time + rs / P.range_sampling_rate;
  double dt = tr - P.fm[0];
  const double ka = P.fm[1] + dt * (P.fm[2] + P.fm[3] * dt);
  dt = tr - P.dc[0];
  const double fnc = P.dc[1] + dt * (P.dc[2] + P.dc[3] * dt);
  const double kmk = ka - P.ks;
  const double inv = 1.0 / (ka * kmk);
  mkt = -(ka * P.ks * (ka * inv));
  etaref = -fnc * (kmk * inv) - P.etac0;
}

__device__ __forceinline__ float2 deramped_tap(const s1b_burst_plan_t &P, const float2 *sec, int r, int c) {
  const float2 v = __ldg(sec + (size_t)r * P.samples + c);
  double mkt, etaref;
  tops_range(P, (double)c, mkt, etaref);
  const double d = (-P.lines * P.ati / 2. + r * P.ati) - etaref;
  return cmul(v, phasor_pi(mkt * d * d));
}

__device__ __forceinline__ float2 fma2(float w, float2 v, float2 acc) {
  return __ffma2_rn(make_float2(w, w), v, acc);
}

// Secondary sample coordinate of one output pixel: the integer sample (na,
// nr) at or below it, the fractions in [0, 1), and whether the kernel
// support [n - lo, n + hi] lies inside the secondary burst.
struct Coord {
  int na, nr;
  float fa, fr;
  bool ok;
};

__device__ __forceinline__ Coord coord_of(const s1b_burst_plan_t &P, const float *az_off, const float *rg_off,
                                          int row, int col, int S, int lo, int hi) {
  Coord k;
  const size_t i = (size_t)row * S + col;
  const float a = __ldg(az_off + i), r = __ldg(rg_off + i);
  // offsets of 2^20 samples or more (and NaN) leave any burst
  k.ok = fabsf(a) < 0x1p20f && fabsf(r) < 0x1p20f;
  const float fla = k.ok ? floorf(a) : 0.f, flr = k.ok ? floorf(r) : 0.f;
  k.na = row + (int)fla;
  k.nr = col + (int)flr;
  // a - floor(a) is exact for a >= 0; for a small negative a it can round
  // to 1.0f, which would put a sinc tap at distance 0 from the wrong sample
  k.fa = fminf(a - fla, 0x1.fffffep-1f);
  k.fr = fminf(r - flr, 0x1.fffffep-1f);
  k.ok = k.ok && k.na - lo >= 0 && k.na + hi < P.lines && k.nr - lo >= 0 && k.nr + hi < P.samples;
  return k;
}

// Restore the secondary's TOPS phase at the fractional position (az lines).
// eta0 = -lines ati / 2 (line 0 from the burst centre), formed once per
// thread: converting the plan's line count per pixel costs issue slots on the
// conversion pipe.
__device__ __forceinline__ float2 reramp(const s1b_burst_plan_t &P, float2 v, double mkt, double eref, double az,
                                         double eta0) {
  const double d = fma(az, P.ati, eta0) - eref;
  return cmul(v, phasor_pi_fast(-(mkt * d * d)));
}

__global__ __launch_bounds__(R_TX *R_TY, 2) void resample_kernel(const __grid_constant__ s1b_burst_plan_t P,
                                                              const float2 *__restrict__ sec,
                                                              const float *__restrict__ az_off,
                                                              const float *__restrict__ rg_off, int L, int S,
                                                              int sinc, float2 *__restrict__ out) {
  __shared__ float2 win[R_WROWS][R_WCOLS];
  __shared__ double s_mkt[R_WCOLS], s_eref[R_WCOLS];
  __shared__ int s_red[4];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * R_TX + tx;
  const int col = blockIdx.x * R_TX + tx;
  const int rowb = blockIdx.y * R_TH + ty * R_RPT;
  const int lo = sinc ? 3 : 0, hi = sinc ? 4 : 1;
  const double eta0 = -P.lines * P.ati / 2.;  // line 0 from the burst centre
  if (tid == 0) {
    s_red[0] = INT_MAX;
    s_red[1] = INT_MIN;
    s_red[2] = INT_MAX;
    s_red[3] = INT_MIN;
  }
  Coord k[R_RPT];
  int mna = INT_MAX, xna = INT_MIN, mnr = INT_MAX, xnr = INT_MIN;
#pragma unroll
  for (int q = 0; q < R_RPT; ++q) {
    const int row = rowb + q;
    if (row < L && col < S) {
      k[q] = coord_of(P, az_off, rg_off, row, col, S, lo, hi);
    } else {
      k[q] = Coord{0, 0, 0.f, 0.f, false};
    }
    if (k[q].ok) {
      mna = min(mna, k[q].na);
      xna = max(xna, k[q].na);
      mnr = min(mnr, k[q].nr);
      xnr = max(xnr, k[q].nr);
    }
  }
  __syncthreads();
  if (mna <= xna) {
    atomicMin(&s_red[0], mna);
    atomicMax(&s_red[1], xna);
    atomicMin(&s_red[2], mnr);
    atomicMax(&s_red[3], xnr);
  }
  __syncthreads();
  const int wa0 = s_red[0] - lo, wr0 = s_red[2] - lo;
  const int nwr = s_red[1] + hi - wa0 + 1, nwc = s_red[3] + hi - wr0 + 1;
  const bool any = s_red[0] <= s_red[1];
  const bool staged = any && nwr <= R_WROWS && nwc <= R_WCOLS;  // block-uniform
  if (staged) {
    // Deramp the window while staging it (the phase of geo2rdr.cu:151-152 at
    // every sample).  Threads own window columns and walk down row segments:
    // along a column phi(r) = mkt (eta0 + r ati - etaref)^2 has increments
    // that grow by the constant 2 mkt ati^2, so after one exact float64 start
    // per segment the rotation is carried by two float32 phasor recurrences
    // (drift ~1e-6 rad over a segment).
    for (int c = tid; c < nwc; c += R_TX * R_TY) tops_range(P, (double)(wr0 + c), s_mkt[c], s_eref[c]);
    __syncthreads();
    const int groups = max(1, (R_TX * R_TY) / nwc);
    const int seg = (nwr + groups - 1) / groups;
    const int g = tid / nwc, c = tid - g * nwc;
    if (g < groups) {
      const int r0 = g * seg, r1 = min(nwr, r0 + seg);
      if (r0 < r1) {
        const double mkt = s_mkt[c], eref = s_eref[c];
        const double u = fma((double)(wa0 + r0), P.ati, -P.lines * P.ati / 2.) - eref;
        float2 ph = phasor_pi(mkt * u * u);
        float2 step = phasor_pi(mkt * P.ati * (2.0 * u + P.ati));
        const float2 dstep = phasor_pi(2.0 * mkt * P.ati * P.ati);
        const float2 *src = sec + (size_t)(wa0 + r0) * P.samples + (wr0 + c);
#pragma unroll 4
        for (int r = r0; r < r1; ++r) {
          const float2 v = __ldg(src);
          src += P.samples;
          win[r][c] = cmul(v, ph);
          ph = cmul(ph, step);
          step = cmul(step, dstep);
        }
      }
    }
    __syncthreads();
  }
  const bool block4 = staged && sinc && k[0].ok && k[1].ok && k[2].ok && k[3].ok && k[1].na == k[0].na + 1 &&
                      k[2].na == k[0].na + 2 && k[3].na == k[0].na + 3 && k[1].nr == k[0].nr &&
                      k[2].nr == k[0].nr && k[3].nr == k[0].nr;
  if (block4) {
    // four outputs on consecutive lines of one range sample: each of the 11
    // tap rows is read once for all four
    float2 acc[R_RPT];
    float wr[R_RPT][8], wa[R_RPT][8];
#pragma unroll
    for (int q = 0; q < R_RPT; ++q) {
      acc[q] = make_float2(0.f, 0.f);
      sinc8_weights(k[q].fr, wr[q]);
      sinc8_weights(k[q].fa, wa[q]);
    }
    const float2 *base = &win[k[0].na - 3 - wa0][k[0].nr - 3 - wr0];
#pragma unroll
    for (int rr = 0; rr < 8 + R_RPT - 1; ++rr) {
      float2 tap[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) tap[j] = base[rr * R_WCOLS + j];
#pragma unroll
      for (int q = 0; q < R_RPT; ++q) {
        const int ka = rr - q;  // tap row of output q
        if (ka < 0 || ka > 7) continue;
        float2 rs = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 8; ++j) rs = fma2(wr[q][j], tap[j], rs);
        acc[q] = fma2(wa[q][ka], rs, acc[q]);
      }
    }
    // -kt and etaref at the fractional sample from the staged per-column
    // values (smooth in range: linear interpolation is exact to ~1e-7 rad)
    const int c = k[0].nr - wr0;
    const double m0 = s_mkt[c], dm = s_mkt[c + 1] - m0, e0 = s_eref[c], de = s_eref[c + 1] - e0;
#pragma unroll
    for (int q = 0; q < R_RPT; ++q) {
      const double t = k[q].fr;
      const float2 v = reramp(P, acc[q], fma(t, dm, m0), fma(t, de, e0), i32_to_f64(k[q].na) + (double)k[q].fa, eta0);
      __stcs(out + (size_t)(rowb + q) * S + col, v);
    }
    return;
  }
  // Any other thread: one output at a time, its coordinate re-read (L1 hit)
  // so that no per-output array is indexed by a loop variable.
#pragma unroll 1
  for (int q = 0; q < R_RPT; ++q) {
    const int row = rowb + q;
    if (row >= L || col >= S) break;
    const Coord kq = coord_of(P, az_off, rg_off, row, col, S, lo, hi);
    float2 v = make_float2(0.f, 0.f);
    if (kq.ok) {
      float2 acc = make_float2(0.f, 0.f);
      if (sinc) {
        float wr[8], wa[8];
        sinc8_weights(kq.fr, wr);
        sinc8_weights(kq.fa, wa);
        if (staged) {
          const float2 *base = &win[kq.na - 3 - wa0][kq.nr - 3 - wr0];
#pragma unroll
          for (int ka = 0; ka < 8; ++ka) {
            float2 rs = make_float2(0.f, 0.f);
#pragma unroll
            for (int kr = 0; kr < 8; ++kr) rs = fma2(wr[kr], base[ka * R_WCOLS + kr], rs);
            acc = fma2(wa[ka], rs, acc);
          }
        } else {
          for (int ka = 0; ka < 8; ++ka) {
            float2 rs = make_float2(0.f, 0.f);
            for (int kr = 0; kr < 8; ++kr) rs = fma2(wr[kr], deramped_tap(P, sec, kq.na + ka - 3, kq.nr + kr - 3), rs);
            acc = fma2(wa[ka], rs, acc);
          }
        }
      } else {
        float2 b[4];
        if (staged) {
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = win[kq.na + (j >> 1) - wa0][kq.nr + (j & 1) - wr0];
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = deramped_tap(P, sec, kq.na + (j >> 1), kq.nr + (j & 1));
        }
        const float fr = kq.fr, fa = kq.fa;
        const float2 c1 = make_float2(fmaf(fr, b[1].x - b[0].x, b[0].x), fmaf(fr, b[1].y - b[0].y, b[0].y));
        const float2 c2 = make_float2(fmaf(fr, b[3].x - b[2].x, b[2].x), fmaf(fr, b[3].y - b[2].y, b[2].y));
        acc = make_float2(fmaf(fa, c2.x - c1.x, c1.x), fmaf(fa, c2.y - c1.y, c1.y));
      }
      double mkt, eref;
      if (staged) {
        const int c = kq.nr - wr0;
        const double t = kq.fr;
        mkt = fma(t, s_mkt[c + 1] - s_mkt[c], s_mkt[c]);
        eref = fma(t, s_eref[c + 1] - s_eref[c], s_eref[c]);
      } else {
        tops_range(P, (double)kq.nr + (double)kq.fr, mkt, eref);
      }
      v = reramp(P, acc, mkt, eref, i32_to_f64(kq.na) + (double)kq.fa, eta0);
    }
    __stcs(out + (size_t)row * S + col, v);
  }
}

// ------------------------------------------------- resample, TMA pipeline
// Persistent form of the resampler (one CTA per half SM, tiles of 64
// columns x 16 rows taken round-robin) for rasters a tensor map can describe.
// Everything a tile reads comes through shared memory by TMA
// (cp.async.bulk.tensor, completion on an mbarrier):
//   offsets  - the tile's az/rg offset blocks, issued two tiles ahead into
//              one of three stages;
//   window   - the raw secondary window of the tile, box RT_WC x RT_WR at an
//              even column (16-byte rule), issued one tile ahead into one of
//              two stages as soon as the tile's coordinate range is known;
//   sinc LUT - copied once per CTA.
// Per tile the CTA (1) reduces the next tile's coordinate range and issues
// its window, (2) deramps the current window in place, (3) interpolates,
// reramps and stores.  Waits are bounded; a wait that runs out sets *status,
// lets the copies in flight land (again bounded) and ends the block.
constexpr int RT_THREADS = R_TX * R_TY;           // 256: 64 columns x 4 row groups of 4 rows
constexpr int RT_WR = 32, RT_WC = 96;             // window box rows x columns
constexpr int RT_OFF_BYTES = 2 * R_TH * R_TX * 4; // az + rg blocks of one tile
constexpr int RT_WIN_BYTES = RT_WR * RT_WC * 8;

struct RtSmem {
  float2 win[2][RT_WR][RT_WC];
  float offs[3][2][R_TH][R_TX];
  float lut[(SINC_BINS + 1) * 8];
  double mkt[2][RT_WC], eref[2][RT_WC];  // per window stage
  int red[RT_THREADS / 32][4];
  uint64_t bar_off[3], bar_win[2];
};

__device__ __forceinline__ void sinc8_weights_lut(const float *lut, float f, float w[8]) {
  const float pos = f * SINC_BINS;
  const int b = min((int)pos, SINC_BINS - 1);
  const float t = pos - (float)b;
  const float4 *T = reinterpret_cast<const float4 *>(lut) + 2 * b;
  const float4 a0 = T[0], a1 = T[1], b0 = T[2], b1 = T[3];
  const float2 tt = make_float2(t, t), m1 = make_float2(-1.f, -1.f);
  const float2 w01 = __ffma2_rn(tt, __ffma2_rn(m1, make_float2(a0.x, a0.y), make_float2(b0.x, b0.y)), make_float2(a0.x, a0.y));
  const float2 w23 = __ffma2_rn(tt, __ffma2_rn(m1, make_float2(a0.z, a0.w), make_float2(b0.z, b0.w)), make_float2(a0.z, a0.w));
  const float2 w45 = __ffma2_rn(tt, __ffma2_rn(m1, make_float2(a1.x, a1.y), make_float2(b1.x, b1.y)), make_float2(a1.x, a1.y));
  const float2 w67 = __ffma2_rn(tt, __ffma2_rn(m1, make_float2(a1.z, a1.w), make_float2(b1.z, b1.w)), make_float2(a1.z, a1.w));
  w[0] = w01.x; w[1] = w01.y; w[2] = w23.x; w[3] = w23.y;
  w[4] = w45.x; w[5] = w45.y; w[6] = w67.x; w[7] = w67.y;
}

// Coordinate of one output from its offsets (as coord_of, values given).
__device__ __forceinline__ Coord coord_from(const s1b_burst_plan_t &P, float a, float r, int row, int col, bool in,
                                            int lo, int hi) {
  Coord k;
  k.ok = in && fabsf(a) < 0x1p20f && fabsf(r) < 0x1p20f;
  const float fla = k.ok ? floorf(a) : 0.f, flr = k.ok ? floorf(r) : 0.f;
  k.na = row + (int)fla;
  k.nr = col + (int)flr;
  k.fa = fminf(a - fla, 0x1.fffffep-1f);
  k.fr = fminf(r - flr, 0x1.fffffep-1f);
  k.ok = k.ok && k.na - lo >= 0 && k.na + hi < P.lines && k.nr - lo >= 0 && k.nr + hi < P.samples;
  return k;
}

// Secondary window of a tile: origin (row wa0, even column wr0) and extent.
struct Window {
  int wa0, wr0, nwr, nwc;
  bool staged;
};

__device__ __forceinline__ void mbar_init(uint64_t *b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(b)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap &m, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(&m)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

__global__ __launch_bounds__(RT_THREADS, 2) void resample_tma_kernel(
    const __grid_constant__ s1b_burst_plan_t P, const __grid_constant__ CUtensorMap tsec,
    const __grid_constant__ CUtensorMap taz, const __grid_constant__ CUtensorMap trg, const float2 *__restrict__ sec,
    int L, int S, int sinc, int ntx, int ntiles, float2 *__restrict__ out, int *__restrict__ status,
    uint32_t poll_limit) {
  extern __shared__ __align__(1024) unsigned char rt_raw[];
  RtSmem &sm = *reinterpret_cast<RtSmem *>(rt_raw);
  const int tid = threadIdx.x, tx = tid % R_TX, ty = tid / R_TX, lane = tid % 32, warp = tid / 32;
  const int lo = sinc ? 3 : 0, hi = sinc ? 4 : 1;
  const double eta0 = -P.lines * P.ati / 2.;  // line 0 from the burst centre
  const int n = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  if (n == 0) return;
  {
    const float4 *g = reinterpret_cast<const float4 *>(g_sinc_table);
    float4 *s = reinterpret_cast<float4 *>(sm.lut);
    for (int i = tid; i < (SINC_BINS + 1) * 2; i += RT_THREADS) s[i] = g[i];
  }
  if (tid == 0) {
    for (int i = 0; i < 3; ++i) mbar_init(&sm.bar_off[i]);
    for (int i = 0; i < 2; ++i) mbar_init(&sm.bar_win[i]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // copies in flight, tracked by thread 0 (bits 0-2 offsets, 3-4 windows),
  // with the phase parity each offsets stage is waiting on
  uint32_t pending = 0, opar = 0, wphase = 0;
  auto tile_origin = [&](int j, int &row0, int &col0) {
    const int t = blockIdx.x + j * gridDim.x;
    row0 = (t / ntx) * R_TH;
    col0 = (t % ntx) * R_TX;
  };
  auto issue_offsets = [&](int j) {  // thread 0 only
    int row0, col0;
    tile_origin(j, row0, col0);
    const int s = j % 3;
    mbar_expect(&sm.bar_off[s], RT_OFF_BYTES);
    tma_load_2d(&sm.offs[s][0][0][0], taz, col0, row0, &sm.bar_off[s]);
    tma_load_2d(&sm.offs[s][1][0][0], trg, col0, row0, &sm.bar_off[s]);
    pending |= 1u << s;
    opar = (opar & ~(1u << s)) | ((uint32_t)((j / 3) & 1) << s);
  };
  // Drain what thread 0 issued (bounded) and flag the failure.
  auto abort_block = [&]() {
    if (tid == 0) {
      atomicExch(status, 1);
      for (int s = 0; s < 3; ++s)
        if (pending & (1u << s)) mbar_wait(smem_addr(&sm.bar_off[s]), (opar >> s) & 1);
      for (int s = 0; s < 2; ++s)
        if (pending & (8u << s)) mbar_wait(smem_addr(&sm.bar_win[s]), (wphase >> s) & 1);
    }
  };
  // Coordinates of this thread's outputs of local tile j from its offsets stage.
  auto coords = [&](int j, Coord k[R_RPT]) {
    int row0, col0;
    tile_origin(j, row0, col0);
    const int s = j % 3, col = col0 + tx;
#pragma unroll
    for (int q = 0; q < R_RPT; ++q) {
      const int r = ty * R_RPT + q, row = row0 + r;
      k[q] = coord_from(P, sm.offs[s][0][r][tx], sm.offs[s][1][r][tx], row, col, row < L && col < S, lo, hi);
    }
  };
  // Step b for local tile j: wait its offsets, reduce its coordinate range,
  // issue its window and the offsets of tile j + 1.  Returns false on a
  // failed wait (uniform over the block).
  auto prepare = [&](int j, Window &w) -> bool {
    const bool ok_wait = mbar_wait(smem_addr(&sm.bar_off[j % 3]), (j / 3) & 1, poll_limit);
    if (tid == 0 && ok_wait) pending &= ~(1u << (j % 3));
    int mna = INT_MAX, xna = INT_MIN, mnr = INT_MAX, xnr = INT_MIN;
    if (ok_wait) {
      Coord k[R_RPT];
      coords(j, k);
#pragma unroll
      for (int q = 0; q < R_RPT; ++q)
        if (k[q].ok) {
          mna = min(mna, k[q].na);
          xna = max(xna, k[q].na);
          mnr = min(mnr, k[q].nr);
          xnr = max(xnr, k[q].nr);
        }
    }
    mna = __reduce_min_sync(0xffffffffu, mna);
    xna = __reduce_max_sync(0xffffffffu, xna);
    mnr = __reduce_min_sync(0xffffffffu, mnr);
    xnr = __reduce_max_sync(0xffffffffu, xnr);
    if (lane == 0) {
      sm.red[warp][0] = mna;
      sm.red[warp][1] = xna;
      sm.red[warp][2] = mnr;
      sm.red[warp][3] = xnr;
    }
    // generic-proxy writes to the stages that the copies below overwrite are
    // ordered before them by this fence and the barrier
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (__syncthreads_or(!ok_wait)) return false;
#pragma unroll
    for (int i = 0; i < RT_THREADS / 32; ++i) {
      mna = min(mna, sm.red[i][0]);
      xna = max(xna, sm.red[i][1]);
      mnr = min(mnr, sm.red[i][2]);
      xnr = max(xnr, sm.red[i][3]);
    }
    w = Window{0, 0, 0, 0, false};
    if (mna <= xna) {
      w.wa0 = mna - lo;
      w.wr0 = (mnr - lo) & ~1;
      w.nwr = xna + hi - w.wa0 + 1;
      w.nwc = xnr + hi - w.wr0 + 1;
      w.staged = w.nwr <= RT_WR && w.nwc <= RT_WC;
    }
    if (tid == 0) {
      if (w.staged) {
        const int s = j & 1;
        mbar_expect(&sm.bar_win[s], RT_WIN_BYTES);
        tma_load_2d(&sm.win[s][0][0], tsec, w.wr0, w.wa0, &sm.bar_win[s]);
        pending |= 8u << s;
      }
      if (j + 1 < n) issue_offsets(j + 1);
    }
    return true;
  };

  if (tid == 0) issue_offsets(0);
  Window cur, nxt;
  if (!prepare(0, cur)) {
    abort_block();
    return;
  }
  for (int i = 0; i < n; ++i) {
    if (i + 1 < n && !prepare(i + 1, nxt)) {
      abort_block();
      return;
    }
    const int s = i & 1;
    bool ok_wait = true;
    if (cur.staged) {
      ok_wait = mbar_wait(smem_addr(&sm.bar_win[s]), (wphase >> s) & 1, poll_limit);
      if (ok_wait) {
        wphase ^= 1u << s;
        if (tid == 0) pending &= ~(8u << s);
      }
    }
    if (cur.staged && ok_wait) {
      // deramp the window in place: threads own columns and walk row
      // segments with the phasor recurrence of the direct kernel
      // tid / nwc and RT_THREADS / nwc by a float reciprocal: every quotient
      // (i + 0.5) / nwc with i <= 256, nwc <= 96 is >= 0.005 from an integer
      const float rn = __frcp_rn((float)cur.nwc);
      const int groups = max(1, __float2int_rz((RT_THREADS + 0.5f) * rn));
      const int seg = (cur.nwr + groups - 1) / groups;
      const int g = __float2int_rz((tid + 0.5f) * rn), c = tid - g * cur.nwc;
      if (g < groups) {
        double mkt, eref;
        tops_range(P, (double)(cur.wr0 + c), mkt, eref);
        if (g == 0) {
          sm.mkt[s][c] = mkt;
          sm.eref[s][c] = eref;
        }
        const int r0 = g * seg, r1 = min(cur.nwr, r0 + seg);
        if (r0 < r1) {
          const double u = fma((double)(cur.wa0 + r0), P.ati, -P.lines * P.ati / 2.) - eref;
          float2 ph = phasor_pi(mkt * u * u);
          float2 step = phasor_pi(mkt * P.ati * (2.0 * u + P.ati));
          const float2 dstep = phasor_pi(2.0 * mkt * P.ati * P.ati);
#pragma unroll 4
          for (int r = r0; r < r1; ++r) {
            sm.win[s][r][c] = cmul(sm.win[s][r][c], ph);
            ph = cmul(ph, step);
            step = cmul(step, dstep);
          }
        }
      }
    }
    if (__syncthreads_or(!ok_wait)) {
      abort_block();
      return;
    }
    // interpolate, reramp and store tile i
    int row0, col0;
    tile_origin(i, row0, col0);
    const int col = col0 + tx, rowb = row0 + ty * R_RPT;
    Coord k[R_RPT];
    coords(i, k);
    const bool block4 = cur.staged && sinc && k[0].ok && k[1].ok && k[2].ok && k[3].ok &&
                        k[1].na == k[0].na + 1 && k[2].na == k[0].na + 2 && k[3].na == k[0].na + 3 &&
                        k[1].nr == k[0].nr && k[2].nr == k[0].nr && k[3].nr == k[0].nr;
    if (block4) {
      float2 acc[R_RPT];
      float wr[R_RPT][8], wa[R_RPT][8];
#pragma unroll
      for (int q = 0; q < R_RPT; ++q) {
        acc[q] = make_float2(0.f, 0.f);
        sinc8_weights_lut(sm.lut, k[q].fr, wr[q]);
        sinc8_weights_lut(sm.lut, k[q].fa, wa[q]);
      }
      const float2 *base = &sm.win[s][k[0].na - 3 - cur.wa0][k[0].nr - 3 - cur.wr0];
#pragma unroll
      for (int rr = 0; rr < 8 + R_RPT - 1; ++rr) {
        float2 tap[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) tap[j] = base[rr * RT_WC + j];
#pragma unroll
        for (int q = 0; q < R_RPT; ++q) {
          const int ka = rr - q;
          if (ka < 0 || ka > 7) continue;
          float2 rs = make_float2(0.f, 0.f);
#pragma unroll
          for (int j = 0; j < 8; ++j) rs = fma2(wr[q][j], tap[j], rs);
          acc[q] = fma2(wa[q][ka], rs, acc[q]);
        }
      }
      const int c = k[0].nr - cur.wr0;
      const double m0 = sm.mkt[s][c], dm = sm.mkt[s][c + 1] - m0, e0 = sm.eref[s][c], de = sm.eref[s][c + 1] - e0;
#pragma unroll
      for (int q = 0; q < R_RPT; ++q) {
        const double t = k[q].fr;
        const float2 v = reramp(P, acc[q], fma(t, dm, m0), fma(t, de, e0), i32_to_f64(k[q].na) + (double)k[q].fa, eta0);
        __stcs(out + (size_t)(rowb + q) * S + col, v);
      }
    } else {
#pragma unroll 1
      for (int q = 0; q < R_RPT; ++q) {
        const int row = rowb + q;
        if (row >= L || col >= S) break;
        const int r = ty * R_RPT + q;
        const Coord kq = coord_from(P, sm.offs[i % 3][0][r][tx], sm.offs[i % 3][1][r][tx], row, col, true, lo, hi);
        float2 v = make_float2(0.f, 0.f);
        if (kq.ok) {
          float2 acc = make_float2(0.f, 0.f);
          if (sinc) {
            float wr[8], wa[8];
            sinc8_weights_lut(sm.lut, kq.fr, wr);
            sinc8_weights_lut(sm.lut, kq.fa, wa);
            if (cur.staged) {
              const float2 *base = &sm.win[s][kq.na - 3 - cur.wa0][kq.nr - 3 - cur.wr0];
#pragma unroll
              for (int ka = 0; ka < 8; ++ka) {
                float2 rs = make_float2(0.f, 0.f);
#pragma unroll
                for (int kr = 0; kr < 8; ++kr) rs = fma2(wr[kr], base[ka * RT_WC + kr], rs);
                acc = fma2(wa[ka], rs, acc);
              }
            } else {
              for (int ka = 0; ka < 8; ++ka) {
                float2 rs = make_float2(0.f, 0.f);
                for (int kr = 0; kr < 8; ++kr)
                  rs = fma2(wr[kr], deramped_tap(P, sec, kq.na + ka - 3, kq.nr + kr - 3), rs);
                acc = fma2(wa[ka], rs, acc);
              }
            }
          } else {
            float2 b[4];
            if (cur.staged) {
#pragma unroll
              for (int j = 0; j < 4; ++j) b[j] = sm.win[s][kq.na + (j >> 1) - cur.wa0][kq.nr + (j & 1) - cur.wr0];
            } else {
#pragma unroll
              for (int j = 0; j < 4; ++j) b[j] = deramped_tap(P, sec, kq.na + (j >> 1), kq.nr + (j & 1));
            }
            const float fr = kq.fr, fa = kq.fa;
            const float2 c1 = make_float2(fmaf(fr, b[1].x - b[0].x, b[0].x), fmaf(fr, b[1].y - b[0].y, b[0].y));
            const float2 c2 = make_float2(fmaf(fr, b[3].x - b[2].x, b[2].x), fmaf(fr, b[3].y - b[2].y, b[2].y));
            acc = make_float2(fmaf(fa, c2.x - c1.x, c1.x), fmaf(fa, c2.y - c1.y, c1.y));
          }
          double mkt, eref;
          if (cur.staged) {
            const int c = kq.nr - cur.wr0;
            const double t = kq.fr;
            mkt = fma(t, sm.mkt[s][c + 1] - sm.mkt[s][c], sm.mkt[s][c]);
            eref = fma(t, sm.eref[s][c + 1] - sm.eref[s][c], sm.eref[s][c]);
          } else {
            tops_range(P, (double)kq.nr + (double)kq.fr, mkt, eref);
          }
          v = reramp(P, acc, mkt, eref, i32_to_f64(kq.na) + (double)kq.fa, eta0);
        }
        __stcs(out + (size_t)row * S + col, v);
      }
    }
    cur = nxt;
  }
}

// ------------------------------------------------------- box coherence
// Windows of 7 x 7 and 9 x 9 (5 x 5 and smaller use the row walk below).
// Persistent kernel, one CTA of 512 threads per SM, output tiles of 128
// columns x 32 rows taken round-robin.  Both SLC tiles plus a halo are
// brought into shared memory by TMA (cp.async.bulk.tensor, zero fill outside
// the raster) through a two-stage pipeline: the next tile streams in while
// the current one is reduced.  The conj product and both powers are formed
// once per staged pixel in place, two pixels per 16-byte access.  Each thread
// then slides the windows of two adjacent columns down 4 output rows:
// horizontal sums per row from 16-byte reads (the taps the two windows share
// summed once), a ring of the last `win` of them, and the vertical sums.  The
// vertical sum of the complex channel slides (add the entering row, subtract
// the leaving one) with Kahan compensation, re and im in paired FP32; the
// power sums, of non-negative terms, are summed directly.  Without a tensor
// map (odd width, unaligned base) tiles are staged by plain loads.
constexpr int C_TW = 128, C_TH = 32, C_HX = 4;  // halo columns (even, >= half window)
constexpr int C_IW = C_TW + 2 * C_HX;            // 136 staged columns
constexpr int C_MAXH = 4;                        // half window <= 4 (win <= 9)
constexpr int C_IH = C_TH + 2 * C_MAXH;          // 40 staged rows
// 512 threads: 64 column pairs x 8 parts of 4 output rows
constexpr int C_THREADS = 512, C_PAIRS = C_TW / 2, C_PARTS = C_THREADS / C_PAIRS, C_ROWS = C_TH / C_PARTS;
constexpr int C_STAGE = 2 * C_IH * C_IW;         // float2 per stage (ref + sec)

// Kahan compensated summation (W. Kahan, "Further remarks on reducing
// truncation errors", CACM 1965).
struct Kahan {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ float value() const { return s; }
};

// Kahan summation of two independent sums at once (re and im of one complex
// sum) with paired FP32 operations; nc holds the negated compensation.  Each
// lane performs exactly the scalar Kahan steps.
struct Kahan2 {
  float2 s = make_float2(0.f, 0.f), nc = make_float2(0.f, 0.f);
  __device__ __forceinline__ void step(float2 y) {
    const float2 t = __fadd2_rn(s, y);
    nc = __fadd2_rn(__ffma2_rn(t, make_float2(-1.f, -1.f), s), y);  // (s - t) + y
    s = t;
  }
  __device__ __forceinline__ void add(float2 x) { step(__fadd2_rn(x, nc)); }
  __device__ __forceinline__ void sub(float2 x) { step(__ffma2_rn(x, make_float2(-1.f, -1.f), nc)); }
};

__device__ __forceinline__ void tma_tile(float2 *dst_r, float2 *dst_s, const CUtensorMap &tr, const CUtensorMap &ts,
                                         int x0, int y0, uint32_t bar) {
  const uint32_t bytes = (uint32_t)C_STAGE * sizeof(float2);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst_r)),
      "l"(reinterpret_cast<uint64_t>(&tr)), "r"(x0), "r"(y0), "r"(bar)
      : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst_s)),
      "l"(reinterpret_cast<uint64_t>(&ts)), "r"(x0), "r"(y0), "r"(bar)
      : "memory");
}

template <bool kTma, int HALF>
__global__ __launch_bounds__(C_THREADS, 1) void box_coherence_kernel(const __grid_constant__ CUtensorMap tref,
                                                                     const __grid_constant__ CUtensorMap tsec,
                                                                     const float2 *__restrict__ ref,
                                                                     const float2 *__restrict__ sec, int L, int S,
                                                                     int ntx, int ntiles, float *__restrict__ coh,
                                                                     int *__restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float2 *stage0 = reinterpret_cast<float2 *>(smem_raw);
  __shared__ __align__(8) uint64_t bars[2];
  constexpr int WIN = 2 * HALF + 1;
  const int tp = threadIdx.x % C_PAIRS, part = threadIdx.x / C_PAIRS;
  if (kTma) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[0])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[1])) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && blockIdx.x < ntiles) {
      const int t = blockIdx.x;
      tma_tile(stage0, stage0 + C_IH * C_IW, tref, tsec, (t % ntx) * C_TW - C_HX, (t / ntx) * C_TH - C_MAXH,
               smem_addr(&bars[0]));
    }
  }
  for (int k = 0;; ++k) {
    const int t = blockIdx.x + k * gridDim.x;
    if (t >= ntiles) break;
    bool ok = true;  // this thread saw the tile's staging complete
    float2 *sr = stage0 + (k & 1) * C_STAGE;
    float2 *ss = sr + C_IH * C_IW;
    const int col0 = (t % ntx) * C_TW, row0 = (t / ntx) * C_TH;
    const int x0 = col0 - C_HX, y0 = row0 - C_MAXH;  // x0 even: TMA needs 16-byte column starts
    if (kTma) {
      const int tn = t + gridDim.x;
      if (threadIdx.x == 0 && tn < ntiles) {
        float2 *nr = stage0 + ((k + 1) & 1) * C_STAGE;
        tma_tile(nr, nr + C_IH * C_IW, tref, tsec, (tn % ntx) * C_TW - C_HX, (tn / ntx) * C_TH - C_MAXH,
                 smem_addr(&bars[(k + 1) & 1]));
      }
      ok = mbar_wait(smem_addr(&bars[k & 1]), (k >> 1) & 1);
    } else {
      for (int idx = threadIdx.x; idx < C_IH * C_IW; idx += C_THREADS) {
        const int r = idx / C_IW, c = idx - r * C_IW;
        const int gr = y0 + r, gc = x0 + c;
        const bool inside = gr >= 0 && gr < L && gc >= 0 && gc < S;
        sr[idx] = inside ? __ldg(ref + (size_t)gr * S + gc) : make_float2(0.f, 0.f);
        ss[idx] = inside ? __ldg(sec + (size_t)gr * S + gc) : make_float2(0.f, 0.f);
      }
      __syncthreads();
    }
    // products once per staged pixel, in place: sr <- conj(r) s, ss <- (|r|^2, |s|^2);
    // two pixels per 16-byte access (rows are 16-byte aligned).  A thread
    // whose staging wait gave up works on whatever the stage holds: the
    // barrier below then ends the whole block before any result is stored.
    {
      float4 *sr4 = reinterpret_cast<float4 *>(sr);
      float4 *ss4 = reinterpret_cast<float4 *>(ss);
      for (int idx = threadIdx.x; idx < C_IH * C_IW / 2; idx += C_THREADS) {
        const float4 a4 = sr4[idx], b4 = ss4[idx];
        float2 cp[2], pw[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float2 a = h ? make_float2(a4.z, a4.w) : make_float2(a4.x, a4.y);
          const float2 b = h ? make_float2(b4.z, b4.w) : make_float2(b4.x, b4.y);
          cp[h] = __ffma2_rn(make_float2(a.y, -a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
          const float2 xx = make_float2(a.x, b.x), yy = make_float2(a.y, b.y);
          pw[h] = __ffma2_rn(yy, yy, __fmul2_rn(xx, xx));
        }
        sr4[idx] = make_float4(cp[0].x, cp[0].y, cp[1].x, cp[1].y);
        ss4[idx] = make_float4(pw[0].x, pw[0].y, pw[1].x, pw[1].y);
      }
    }
    if (__syncthreads_or(!ok)) {
      // never expected: record it, give this tile's and the next tile's copies
      // a second bounded wait so none lands after the block exits, and stop
      // (decided for the whole block)
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        mbar_wait(smem_addr(&bars[k & 1]), (k >> 1) & 1);
        if (t + gridDim.x < ntiles) mbar_wait(smem_addr(&bars[(k + 1) & 1]), ((k + 1) >> 1) & 1);
      }
      return;
    }
    // Two output columns per thread, c and c + 1 of the tile: their windows
    // cover staged columns s0 .. s0 + WIN, read as 16-byte pairs from the
    // even column below s0; the WIN - 1 taps they share are summed once.
    constexpr int O = HALF & 1;                   // s0 is odd exactly when HALF is
    constexpr int NPX = (WIN + 1 + O + 1) & ~1;   // staged pixels read per row
    const int c = 2 * tp;
    const int orow0 = part * C_ROWS;
    const int first = orow0 + C_MAXH - HALF;  // staged row of the first window row
    const int cs = c + C_HX - HALF - O;       // even staged column of the first pixel read
    float2 rc[2][WIN], rp[2][WIN];            // rings of horizontal sums per column
    Kahan2 vs[2];                             // sliding, compensated sums of the complex channel
#pragma unroll
    for (int j = 0; j < C_ROWS + WIN - 1; ++j) {
      const float4 *pr = reinterpret_cast<const float4 *>(sr + (first + j) * C_IW + cs);
      const float4 *pp = reinterpret_cast<const float4 *>(ss + (first + j) * C_IW + cs);
      float2 vr[NPX], vp[NPX];
#pragma unroll
      for (int k = 0; k < NPX / 2; ++k) {
        const float4 a = pr[k], b = pp[k];
        vr[2 * k] = make_float2(a.x, a.y);
        vr[2 * k + 1] = make_float2(a.z, a.w);
        vp[2 * k] = make_float2(b.x, b.y);
        vp[2 * k + 1] = make_float2(b.z, b.w);
      }
      float2 ir = make_float2(0.f, 0.f), ip = ir;  // taps shared by both windows
#pragma unroll
      for (int k = 1; k < WIN; ++k) {
        ir = k == 1 ? vr[O + 1] : __fadd2_rn(ir, vr[O + k]);
        ip = k == 1 ? vp[O + 1] : __fadd2_rn(ip, vp[O + k]);
      }
      float2 hc[2], hp[2];
      if (WIN == 1) {
        hc[0] = vr[O];
        hc[1] = vr[O + 1];
        hp[0] = vp[O];
        hp[1] = vp[O + 1];
      } else {
        hc[0] = __fadd2_rn(vr[O], ir);
        hc[1] = __fadd2_rn(ir, vr[O + WIN]);
        hp[0] = __fadd2_rn(vp[O], ip);
        hp[1] = __fadd2_rn(ip, vp[O + WIN]);
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (j >= WIN) vs[q].sub(rc[q][j % WIN]);  // the row leaving the window
        rc[q][j % WIN] = hc[q];
        rp[q][j % WIN] = hp[q];
        vs[q].add(hc[q]);
      }
      if (j >= WIN - 1) {
        const int orow = row0 + orow0 + (j - (WIN - 1));
        float out[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          // powers: direct sums of non-negative terms (exact zeros stay zero)
          float2 pw = rp[q][0];
#pragma unroll
          for (int m = 1; m < WIN; ++m) pw = __fadd2_rn(pw, rp[q][m]);
          // |I| / sqrt(P1 P2) = sqrt(|I|^2) * rsqrt(P1 P2); 0 where a power is 0
          const float den2 = pw.x * pw.y;
          const float2 v = vs[q].s;
          const float num2 = fmaf(v.x, v.x, v.y * v.y);
          out[q] = den2 > 0.f ? sqrtf(num2) * rsqrtf(den2) : 0.f;
        }
        const int col = col0 + c;
        if (orow < L) {
          float *dst = coh + (size_t)orow * S + col;
          if (kTma && col + 1 < S) {  // a tensor map implies an even width: 8-byte aligned pair
            __stcs(reinterpret_cast<float2 *>(dst), make_float2(out[0], out[1]));
          } else {
            if (col < S) __stcs(dst, out[0]);
            if (col + 1 < S) __stcs(dst + 1, out[1]);
          }
        }
      }
    }
    // order this stage's generic-proxy stores before the TMA that refills it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
  }
}

template <int HALF>
int launch_box(bool tma, const CUtensorMap &mr, const CUtensorMap &ms, const void *ref, const void *sec, int lines,
               int samples, float *coh, int *status, cudaStream_t st) {
  const int ntx = (samples + C_TW - 1) / C_TW, nty = (lines + C_TH - 1) / C_TH;
  const int ntiles = ntx * nty;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = ntiles < sms ? ntiles : sms;
  const size_t smem = 2 * (size_t)C_STAGE * sizeof(float2);
  cudaError_t e;
  if (tma) {
    e = cudaFuncSetAttribute(box_coherence_kernel<true, HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
    box_coherence_kernel<true, HALF><<<grid, C_THREADS, smem, st>>>(mr, ms, nullptr, nullptr, lines, samples, ntx,
                                                                     ntiles, coh, status);
  } else {
    e = cudaFuncSetAttribute(box_coherence_kernel<false, HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
    box_coherence_kernel<false, HALF><<<grid, C_THREADS, smem, st>>>(mr, ms, (const float2 *)ref,
                                                                      (const float2 *)sec, lines, samples, ntx,
                                                                      ntiles, coh, status);
  }
  return s1b_launch_status();
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D tensor map over a row-major raster of `width` x `height` elements of
// `esize` bytes (FLOAT32 or FLOAT64 elements; complex64 travels as one
// 8-byte element), box bw x bh, zero fill outside.  False when the raster
// cannot be described (row pitch not a multiple of 16 bytes, base not
// 16-byte aligned) or the driver lacks the entry point.
bool make_map_2d(CUtensorMap *m, const void *base, CUtensorMapDataType dtype, int esize, int width, int height,
                 int bw, int bh) {
  if (((size_t)width * esize) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) % 16) != 0) return false;
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)height};
  cuuint64_t strides[1] = {(cuuint64_t)width * esize};
  cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, dtype, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool make_tile_map(CUtensorMap *m, const void *base, int L, int S) {
  return make_map_2d(m, base, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, S, L, C_IW, C_IH);
}

// Resident CTAs of the persistent resampler per device (0: not usable).
int resample_tma_slots() {
  static std::mutex mu;
  static int slots[64] = {};
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  std::lock_guard<std::mutex> lock(mu);
  if (!done[dev]) {
    done[dev] = true;
    int sms = 0, per_sm = 0;
    if (cudaFuncSetAttribute(resample_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(RtSmem)) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, resample_tma_kernel, RT_THREADS, sizeof(RtSmem)) ==
            cudaSuccess)
      slots[dev] = sms * per_sm;
    cudaGetLastError();
  }
  return slots[dev];
}

// ------------------------------------------------- box coherence, row walk
// Windows up to 5 x 5 (the coherence window of the chain).  One warp per
// strip of 64 columns x W_ROWS output rows; each lane owns two adjacent
// columns and walks down the strip.  Strips overlap by 4 columns: lanes 0
// and 31 only supply their columns to their neighbours, lanes 1..30 produce
// the strip's 60 output columns.  Rows are brought into a per-warp ring of
// W_PD shared-memory slots by cp.async (16 bytes per lane and array, zero
// fill outside the raster), W_PD - 1 rows ahead of the one being reduced, so
// the copies in flight hold no registers; a lane reads back only what it
// copied itself, so no barrier is needed.  Per row: the conj product and both
// powers of the lane's two columns, the neighbours' by lane shuffles,
// horizontal sums, then a ring of the last WIN rows' horizontal sums in
// registers: the complex channel slides with Kahan compensation, the powers
// are summed directly over the ring (exact zeros stay zero).  Between the HBM
// reads and the coherence store everything stays in registers: 16 B read and
// 4 B written per pixel.
constexpr int W_ROWS = 64;  // output rows per strip
constexpr int W_PD = 4;     // shared-memory row slots per warp (rows W_PD - 1 ahead)
constexpr int W_WARPS = 4;  // strips per CTA, side by side
constexpr int W_OUT = 60;   // output columns per strip

struct WalkSlot {  // one staged row of a warp's strip: the lanes' column pairs of ref and sec
  float4 r[32], s[32];
};

template <bool kVec16>
__device__ __forceinline__ void walk_copy_pair(float4 *dst, const float2 *src, const float2 *base, bool in0,
                                               bool in1) {
  if (kVec16) {  // S even, 16-byte rows: a pair is inside or outside as a whole
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(in0 ? src : base),
                 "r"(in0 ? 16 : 0)
                 : "memory");
  } else {
    const uint32_t d = smem_addr(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(in0 ? src : base), "r"(in0 ? 8 : 0)
                 : "memory");
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d + 8), "l"(in1 ? src + 1 : base),
                 "r"(in1 ? 8 : 0)
                 : "memory");
  }
}

// conj(a) b and (|a|^2, |b|^2) of one pixel as (re, im, |a|^2, |b|^2)
__device__ __forceinline__ float4 walk_products(float ax, float ay, float bx, float by) {
  return make_float4(fmaf(ax, bx, ay * by), fmaf(ax, by, -(ay * bx)), fmaf(ax, ax, ay * ay), fmaf(bx, bx, by * by));
}
__device__ __forceinline__ float4 walk_add(float4 a, float4 b) {
  const float2 c = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  const float2 p = __fadd2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w));
  return make_float4(c.x, c.y, p.x, p.y);
}
__device__ __forceinline__ float4 walk_shfl(float4 v, int src) {
  return make_float4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                     __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

template <int HALF, bool kVec16>
__global__ __launch_bounds__(32 * W_WARPS) void box_walk_kernel(const float2 *__restrict__ ref,
                                                                const float2 *__restrict__ sec, int L, int S,
                                                                float *__restrict__ coh) {
  static_assert(HALF >= 0 && HALF <= 2, "the row walk serves windows up to 5 x 5");
  constexpr int WIN = 2 * HALF + 1;
  __shared__ WalkSlot slots[W_WARPS][W_PD];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int W0 = (blockIdx.x * W_WARPS + warp) * W_OUT;  // first output column of the strip
  if (W0 >= S) return;                                    // warp-uniform; no block barrier below
  const int y0 = blockIdx.y * W_ROWS;
  const int nout = min(W_ROWS, L - y0);
  const int NR = nout + 2 * HALF;    // rows staged: y0 - HALF .. y0 + nout - 1 + HALF
  const int c0 = W0 - 2 + 2 * lane;  // the lane's first column
  const bool in0 = c0 >= 0 && c0 < S, in1 = c0 + 1 >= 0 && c0 + 1 < S;
  const bool out_lane = lane >= 1 && lane <= 30;
  WalkSlot *ring = slots[warp];
  // the lane's pair of the next row to stage, and that row
  int ys = y0 - HALF;
  const float2 *pr = ref + (ptrdiff_t)ys * S + c0, *ps = sec + (ptrdiff_t)ys * S + c0;
  auto stage = [&](int slot) {
    const bool rin = (unsigned)ys < (unsigned)L;
    WalkSlot &sl = ring[slot];
    walk_copy_pair<kVec16>(&sl.r[lane], pr, ref, rin && in0, rin && in1);
    walk_copy_pair<kVec16>(&sl.s[lane], ps, sec, rin && in0, rin && in1);
    ++ys;
    pr += S;
    ps += S;
  };
#pragma unroll
  for (int j = 0; j < W_PD - 1; ++j) {
    if (j < NR) stage(j);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  // rings of the last WIN rows' horizontal sums, complex (rc) and powers (rp),
  // of the lane's columns c0 (index 0) and c0 + 1 (index 1)
  float2 rc[WIN][2], rp[WIN][2];
#pragma unroll
  for (int u = 0; u < WIN; ++u)
#pragma unroll
    for (int q = 0; q < 2; ++q) rc[u][q] = rp[u][q] = make_float2(0.f, 0.f);
  Kahan2 vs[2];
  float *dst = coh + (ptrdiff_t)y0 * S + c0;  // output row y0 - 2 HALF + j at step j >= 2 HALF
  dst -= (ptrdiff_t)2 * HALF * S;
  static_assert((W_PD & (W_PD - 1)) == 0, "ring slots are taken modulo a power of two");
  for (int jb = 0; jb < NR; jb += WIN) {
#pragma unroll
    for (int u = 0; u < WIN; ++u) {
      const int j = jb + u;
      if (j >= NR) break;  // warp-uniform
      // this lane's copies of row j have landed (rows j + 1 .. j + W_PD - 2 may still fly)
      asm volatile("cp.async.wait_group %0;" ::"n"(W_PD - 2) : "memory");
      const WalkSlot &sl = ring[j & (W_PD - 1)];
      const float4 ra = sl.r[lane], sa = sl.s[lane];
      const float4 Pa = walk_products(ra.x, ra.y, sa.x, sa.y), Pb = walk_products(ra.z, ra.w, sa.z, sa.w);
      // the slot of row j - 1 is free (its values were consumed a step ago): stage row j + W_PD - 1
      if (j + W_PD - 1 < NR) stage((j + W_PD - 1) & (W_PD - 1));
      asm volatile("cp.async.commit_group;" ::: "memory");
      float4 Ha = Pa, Hb = Pb;  // horizontal sums of the lane's two columns
      if (HALF > 0) {
        const float4 A = walk_add(Pa, Pb);
        const float4 Lb = walk_shfl(Pb, lane - 1);  // lane 0 gets its own: not an output lane
        const float4 Ra = walk_shfl(Pa, lane + 1);  // lane 31 likewise
        if (HALF == 1) {
          Ha = walk_add(Lb, A);
          Hb = walk_add(A, Ra);
        } else {
          const float4 LA = walk_shfl(A, lane - 1), RA = walk_shfl(A, lane + 1);
          Ha = walk_add(walk_add(LA, A), Ra);
          Hb = walk_add(walk_add(Lb, A), RA);
        }
      }
      const float2 hc[2] = {make_float2(Ha.x, Ha.y), make_float2(Hb.x, Hb.y)};
      const float2 hp[2] = {make_float2(Ha.z, Ha.w), make_float2(Hb.z, Hb.w)};
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (j >= WIN) vs[q].sub(rc[u][q]);  // the row leaving the window
        rc[u][q] = hc[q];
        rp[u][q] = hp[q];
        vs[q].add(hc[q]);
      }
      if (j >= 2 * HALF && out_lane) {
        float out[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          float2 pw = rp[0][q];
#pragma unroll
          for (int m = 1; m < WIN; ++m) pw = __fadd2_rn(pw, rp[m][q]);
          const float den2 = pw.x * pw.y;
          const float2 v = vs[q].s;
          const float num2 = fmaf(v.x, v.x, v.y * v.y);
          out[q] = den2 > 0.f ? sqrtf(num2) * rsqrtf(den2) : 0.f;
        }
        if (kVec16) {
          if (in0) __stcs(reinterpret_cast<float2 *>(dst), make_float2(out[0], out[1]));
        } else {
          if (in0) __stcs(dst, out[0]);
          if (in1) __stcs(dst + 1, out[1]);
        }
      }
      dst += S;
    }
  }
}

template <int HALF>
int launch_walk(const void *ref, const void *sec, int lines, int samples, float *coh, cudaStream_t st) {
  const bool vec16 = samples % 2 == 0 && reinterpret_cast<uintptr_t>(ref) % 16 == 0 &&
                     reinterpret_cast<uintptr_t>(sec) % 16 == 0 && reinterpret_cast<uintptr_t>(coh) % 8 == 0;
  const dim3 grid((samples + W_OUT * W_WARPS - 1) / (W_OUT * W_WARPS), (lines + W_ROWS - 1) / W_ROWS);
  if (vec16)
    box_walk_kernel<HALF, true><<<grid, 32 * W_WARPS, 0, st>>>((const float2 *)ref, (const float2 *)sec, lines,
                                                                samples, coh);
  else
    box_walk_kernel<HALF, false><<<grid, 32 * W_WARPS, 0, st>>>((const float2 *)ref, (const float2 *)sec, lines,
                                                                 samples, coh);
  return s1b_launch_status();
}

}  // namespace

extern "C" int s1b_geo2rdr_offsets(const s1b_burst_plan_t *plan, const double *lat, const double *lon,
                                   const double *hgt, int32_t lines, int32_t samples, float *az_off,
                                   float *rg_off, void *stream) {
  if (!plan || !lat || !lon || !hgt || !az_off || !rg_off)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr_offsets: null argument");
  if (lines < 1 || samples < 1) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr_offsets: empty grid");
  dim3 grid((samples + O_TX - 1) / O_TX, (lines + O_RY - 1) / O_RY);
  if (grid.y > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_geo2rdr_offsets: grid too tall");
  offsets_kernel<false><<<grid, O_TX, 0, (cudaStream_t)stream>>>(*plan, RefOrbit{}, lat, lon, hgt, lines, samples,
                                                                 az_off, rg_off, nullptr, nullptr);
  return s1b_launch_status();
}

extern "C" int s1b_geo2rdr_offsets_dh(const s1b_burst_plan_t *plan, const s1b_burst_plan_t *ref_plan,
                                      const double *lat, const double *lon, const double *hgt, int32_t lines,
                                      int32_t samples, float *az_off, float *rg_off, float *daz_dh, float *drg_dh,
                                      void *stream) {
  if (!plan || !ref_plan || !lat || !lon || !hgt || !az_off || !rg_off || !daz_dh || !drg_dh)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr_offsets_dh: null argument");
  if (lines < 1 || samples < 1) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr_offsets_dh: empty grid");
  dim3 grid((samples + O_TX - 1) / O_TX, (lines + O_RY - 1) / O_RY);
  if (grid.y > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_geo2rdr_offsets_dh: grid too tall");
  RefOrbit ro;
  ro.orbit = ref_plan->orbit;
  ro.tstart = ref_plan->tstart;
  ro.dtaz = ref_plan->dtaz;
  offsets_kernel<true><<<grid, O_TX, 0, (cudaStream_t)stream>>>(*plan, ro, lat, lon, hgt, lines, samples, az_off,
                                                                rg_off, daz_dh, drg_dh);
  return s1b_launch_status();
}

// Polls of each staging wait of the TMA resampler before it gives up
// (s1b_set_staging_poll_limit; the drain after a failed wait always uses
// kSpinLimit, so every copy in flight lands before the block exits).
static uint32_t g_stage_poll_limit = kSpinLimit;

extern "C" uint32_t s1b_set_staging_poll_limit(uint32_t polls) {
  const uint32_t prev = g_stage_poll_limit;
  g_stage_poll_limit = polls;
  return prev;
}

extern "C" int s1b_resample(const s1b_burst_plan_t *plan, const void *sec, const float *az_off,
                            const float *rg_off, int32_t lines, int32_t samples, int32_t interp, void *out,
                            int32_t *status, void *stream) {
  if (!plan || !sec || !az_off || !rg_off || !out || !status)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_resample: null argument");
  if (interp != S1B_INTERP_BILINEAR && interp != S1B_INTERP_SINC8)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_resample: interp must be S1B_INTERP_BILINEAR or S1B_INTERP_SINC8");
  if (lines < 1 || samples < 1 || plan->lines < 2 || plan->samples < 2)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_resample: empty grid");
  int s = ensure_sinc_table();
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int32_t), st);
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  const int ntx = (samples + R_TX - 1) / R_TX, nty = (lines + R_TH - 1) / R_TH;
  const long long ntiles = (long long)ntx * nty;
  const int sinc = interp == S1B_INTERP_SINC8 ? 1 : 0;
  CUtensorMap msec, maz, mrg;
  const int slots = resample_tma_slots();
  if (slots > 0 && ntiles <= INT_MAX &&
      make_map_2d(&msec, sec, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, plan->samples, plan->lines, RT_WC, RT_WR) &&
      make_map_2d(&maz, az_off, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, samples, lines, R_TX, R_TH) &&
      make_map_2d(&mrg, rg_off, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, samples, lines, R_TX, R_TH)) {
    const int grid = (int)std::min<long long>(ntiles, slots);
    resample_tma_kernel<<<grid, RT_THREADS, sizeof(RtSmem), st>>>(*plan, msec, maz, mrg, (const float2 *)sec, lines,
                                                                  samples, sinc, ntx, (int)ntiles, (float2 *)out,
                                                                  status, g_stage_poll_limit);
    return s1b_launch_status();
  }
  dim3 block(R_TX, R_TY);
  dim3 grid(ntx, nty);
  if (grid.y > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_resample: grid too tall");
  resample_kernel<<<grid, block, 0, st>>>(*plan, (const float2 *)sec, az_off, rg_off, lines, samples, sinc,
                                          (float2 *)out);
  return s1b_launch_status();
}

extern "C" int s1b_box_coherence(const void *ref, const void *sec, int32_t lines, int32_t samples, int32_t win,
                                 float *coh, int32_t *status, void *stream) {
  if (!ref || !sec || !coh || !status)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_box_coherence: null argument");
  if (win < 1 || win % 2 == 0 || win > 2 * C_MAXH + 1)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_box_coherence: window must be odd and <= 9");
  if (lines < 1 || samples < 1) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_box_coherence: empty raster");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int32_t), st);
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  // windows up to 5 x 5: the register row walk; 7 x 7 and 9 x 9: TMA halo tiles
  switch (win / 2) {
    case 0: return launch_walk<0>(ref, sec, lines, samples, coh, st);
    case 1: return launch_walk<1>(ref, sec, lines, samples, coh, st);
    case 2: return launch_walk<2>(ref, sec, lines, samples, coh, st);
    default: break;
  }
  CUtensorMap mr, ms;
  const bool tma = make_tile_map(&mr, ref, lines, samples) && make_tile_map(&ms, sec, lines, samples);
  return win / 2 == 3 ? launch_box<3>(tma, mr, ms, ref, sec, lines, samples, coh, status, st)
                      : launch_box<4>(tma, mr, ms, ref, sec, lines, samples, coh, status, st);
}

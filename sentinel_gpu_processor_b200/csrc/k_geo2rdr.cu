// geo2rdr on sm_100a: TOPS deramp, and per-DEM-pixel FP64 zero-Doppler
// geocoding with bilinear resampling, reramp and range phase.
//
// Replaces csrc/src/geo2rdr.cu:86-248 (deramp_burst, reproject,
// find_first_last_nonzero_rows_kernel) of the reference.  Differences in
// method (same results within FP64 rounding):
//   * the orbit is a per-window degree-7 polynomial evaluated by Horner
//     (s1b_orbit_poly_t) instead of the Lagrange-form Hermite with ~60
//     divisions per call;
//   * the zero-Doppler Newton uses the exact derivative (3 steps instead of
//     7-11);
//   * llh->ECEF trigonometry is computed once per DEM row / column per warp;
//   * FP64 phases are reduced mod 2 pi in FP64, then rotated in FP32;
//   * the non-zero-row search is folded into the geocoding epilogue.
#include <climits>
#include <cstddef>
#include <type_traits>
#include <cuda_runtime.h>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_frame.h"
#include "s1b_internal.h"

namespace {

constexpr double kRaD = 6378137.0;
constexpr double kRe2D = 0.00669437999015;

// ------------------------------------------------------------------ deramp
// Tile: 256 threads x 2 columns = 512 columns, ROWS rows.  Per-column TOPS
// coefficients are formed once per thread and reused down the rows.  Input
// samples are complex64 (float2) or the measurement TIFF's complex int16
// (short2: re, im), widened exactly to float in registers.
constexpr int DERAMP_ROWS = 16;

// int16 -> float without the conversion unit: 1.5 * 2^23 has a unit ulp, so
// adding a small integer to its bit pattern adds it to the value (exact for
// |x| < 2^22) and subtracting 1.5 * 2^23 leaves x exactly.  The same value as
// (float)x, from an integer add and an FP32 add.
__device__ __forceinline__ float i16_to_f32(int x) { return __int_as_float(0x4B400000 + x) - 12582912.0f; }
// int -> double: i32_to_f64 in s1b_device.cuh.

// Two adjacent samples from an address aligned to their size (16 bytes for
// complex64, 8 for complex int16), streamed.
__device__ __forceinline__ void load_pair(const float2 *p, float2 &a0, float2 &a1) {
  const float4 v = __ldcs(reinterpret_cast<const float4 *>(p));
  a0 = make_float2(v.x, v.y);
  a1 = make_float2(v.z, v.w);
}
__device__ __forceinline__ void load_pair(const short2 *p, float2 &a0, float2 &a1) {
  const short4 v = __ldcs(reinterpret_cast<const short4 *>(p));
  a0 = make_float2(i16_to_f32(v.x), i16_to_f32(v.y));
  a1 = make_float2(i16_to_f32(v.z), i16_to_f32(v.w));
}
__device__ __forceinline__ float2 load_one(const float2 *p) { return __ldcs(p); }
__device__ __forceinline__ float2 load_one(const short2 *p) {
  const short2 v = __ldcs(p);
  return make_float2(i16_to_f32(v.x), i16_to_f32(v.y));
}

// TOPS deramp coefficients of burst column c (geo2rdr.cu:533-541): -pi kt
// and etaref.  One function for the deramp kernels and the frame's column
// table, so the fused geocoding forms exactly the deramp kernel's phases.
__device__ __forceinline__ void tops_kt(const s1b_burst_plan_t &P, int c, double &kt, double &etaref) {
  const double tr = P.slant_range_time + c / P.range_sampling_rate;
  double dt = tr - P.fm[0];
  const double ka = P.fm[1] + dt * (P.fm[2] + P.fm[3] * dt);
  dt = tr - P.dc[0];
  const double fnc = P.dc[1] + dt * (P.dc[2] + P.dc[3] * dt);
  kt = ka * P.ks / (ka - P.ks);
  etaref = -fnc / ka - P.etac0;
}

__device__ __forceinline__ void tops_column(const s1b_burst_plan_t &P, int c, double &mkt, double &etaref) {
  double kt;
  tops_kt(P, c, kt, etaref);
  mkt = -kPiD * kt;
}

// Azimuth time of line r relative to the burst centre: eta_r = -L ati / 2 +
// r ati (geo2rdr.cu:530-531).
template <typename PL>
__device__ __forceinline__ double deramp_eta(const PL &P, int r) {
  return -P.lines * P.ati / 2. + i32_to_f64(r) * P.ati;
}

// Deramped sample: a * exp(i mkt (eta - etaref)^2) (geo2rdr.cu:151-152).
__device__ __forceinline__ float2 deramp_at(float2 a, double eta, double mkt, double etaref) {
  const double d = eta - etaref;
  return cmul(a, phasor(mkt * d * d));
}

__device__ __forceinline__ float2 deramp_sample(const s1b_burst_plan_t &P, float2 a, int r, double mkt,
                                                double etaref) {
  return deramp_at(a, deramp_eta(P, r), mkt, etaref);
}

template <bool kVec, int ROWS, typename TIn>
__device__ __forceinline__ void deramp_tile(const s1b_burst_plan_t &P, const TIn *__restrict__ in,
                                            float2 *__restrict__ out, int tile_x, int tile_y) {
  const int S = P.samples, L = P.lines;
  const int c0 = (tile_x * 256 + threadIdx.x) * 2;
  if (c0 >= S) return;
  const int r0 = tile_y * ROWS;
  // geo2rdr.cu:533-541 for the thread's two columns: -pi*kt and etaref
  double mkt[2], etaref[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) tops_column(P, c0 + j < S ? c0 + j : c0, mkt[j], etaref[j]);
  const bool two = (c0 + 1) < S;
  if constexpr (std::is_same<TIn, float2>::value) {
    // complex64: rows in batches of 8 whose loads are all issued before any
    // of their arithmetic (predicated, no early exit between them).  Measured
    // 0.088 ms against 0.095 ms per 1500 x 21000 burst; the complex int16
    // path, with half the bytes per load, measured slower this way (the
    // batch halves the resident CTAs) and keeps the row loop below.
    constexpr int B = 8;
    static_assert(ROWS % B == 0, "deramp rows per tile");
#pragma unroll 1
    for (int rb = 0; rb < ROWS; rb += B) {
      float2 a[B][2];
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int r = r0 + rb + k;
        const size_t base = (size_t)r * S + c0;
        a[k][0] = a[k][1] = make_float2(0.f, 0.f);
        if (r < L) {
          if (kVec) {
            load_pair(in + base, a[k][0], a[k][1]);
          } else {
            a[k][0] = load_one(in + base);
            if (two) a[k][1] = load_one(in + base + 1);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < B; ++k) {
        const int r = r0 + rb + k;
        if (r < L) {
          const size_t base = (size_t)r * S + c0;
          const float2 b0 = deramp_sample(P, a[k][0], r, mkt[0], etaref[0]);
          const float2 b1 = deramp_sample(P, a[k][1], r, mkt[1], etaref[1]);
          if (kVec) {
            __stcs(reinterpret_cast<float4 *>(out + base), make_float4(b0.x, b0.y, b1.x, b1.y));
          } else {
            __stcs(out + base, b0);
            if (two) __stcs(out + base + 1, b1);
          }
        }
      }
    }
    return;
  }
#pragma unroll 4
  for (int rr = 0; rr < ROWS; ++rr) {
    const int r = r0 + rr;
    if (r >= L) break;
    const size_t base = (size_t)r * S + c0;
    float2 a0, a1;
    if (kVec) {
      load_pair(in + base, a0, a1);
    } else {
      a0 = load_one(in + base);
      a1 = two ? load_one(in + base + 1) : make_float2(0.f, 0.f);
    }
    const float2 b0 = deramp_sample(P, a0, r, mkt[0], etaref[0]);
    const float2 b1 = deramp_sample(P, a1, r, mkt[1], etaref[1]);
    if (kVec) {
      __stcs(reinterpret_cast<float4 *>(out + base), make_float4(b0.x, b0.y, b1.x, b1.y));
    } else {
      __stcs(out + base, b0);
      if (two) __stcs(out + base + 1, b1);
    }
  }
}

template <bool kVec, typename TIn>
__global__ __launch_bounds__(256) void deramp_kernel(const __grid_constant__ s1b_burst_plan_t P,
                                                     const TIn *__restrict__ in,
                                                     float2 *__restrict__ out) {
  deramp_tile<kVec, DERAMP_ROWS>(P, in, out, blockIdx.x, blockIdx.y);
}

// ----------------------------------------------------------------- geo2rdr
// Tile: G_TX columns x G_RY rows of the DEM window, one thread per column
// walking down the rows.  Every pixel solves its zero-Doppler equation on the
// warp's patch model (a quintic-truncated-to-cubic Doppler polynomial from
// the cubic orbit expansion at the warp centre's zero-Doppler time): four dot
// products per pixel, three FMA per chord-Newton step, and the range from the
// same coefficients.  The first pixel of a column starts from the warp's
// centre time, the others from the linear extrapolation of the two pixels
// above.
// Latitude terms depend only on the row: lanes 0..G_RY-1 of every warp form
// them once and the warp shares them by shuffles (no block barrier);
// longitude terms depend only on the column and stay in registers.  Warps
// cover 32 consecutive columns of a row, so DEM reads and output writes
// coalesce; the next row's DEM sample is loaded one row ahead.
// Rows per tile (a multiple of 32): the per-warp set-up (the centre pixel's
// exact Newton on the orbit polynomial, FP64 row trigonometry) is amortised
// over the tile's rows.  Measured per 27-pair frame: 16 rows 11.15 ms, 32
// rows 9.88 ms, 64 rows 9.41 ms (unfused), and for the fused frame kernel 64
// rows 13.30 ms, 128 rows 13.08 ms (kFrameGeoRows); a single burst's grid is
// too small for 64-row tiles (0.195 ms at 32 rows, 0.221 ms at 64).
constexpr int G_TX = 128, G_RY = 32;  // single-burst launch; the frame launch tunes the width

__global__ void rows_init_kernel(int32_t *rows, int nrow) {
  rows[0] = nrow;
  rows[1] = -1;
}

// Culling of the geocoding blocks outside the burst's valid lines (on by
// default; off only to compare the two, which give identical products).
static int g_cull_geo = 1;

// exp(i pi q) for the small phase differences between neighbouring burst
// columns (|pi q| <= 0.1 rad): Taylor series of cos and sin to the fourth
// and fifth order (truncation error < 1e-7); larger angles through phasor_pi.
__device__ __forceinline__ float2 rotation_pi(double q) {
  const float x = (float)q * 3.14159265f;
  if (fabsf(x) > 0.1f) return phasor_pi(q);
  const float x2 = x * x;
  return make_float2(fmaf(x2, fmaf(x2, 1.f / 24.f, -0.5f), 1.f), x * fmaf(x2, -1.f / 6.f, 1.f));
}

__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float f) {
  return make_float2(fmaf(f, b.x - a.x, a.x), fmaf(f, b.y - a.y, a.y));
}

// Read-only (L1-cached) sample loads for the bilinear gathers.
__device__ __forceinline__ float2 load_ro(const float2 *p) { return __ldg(p); }
__device__ __forceinline__ float2 load_ro(const short2 *p) {
  const short2 v = __ldg(p);
  return make_float2(i16_to_f32(v.x), i16_to_f32(v.y));
}

// Geocoding of one tile.  Unfused (kFused false): `burst` is the deramped
// burst (complex64).  Fused: `burst` holds the raw samples (complex64 or
// complex int16) and `tops` the burst's per-column TOPS coefficients
// (-kt, etaref); the four bilinear samples are deramped where they are
// gathered and the deramped copy of the burst is never written.  Bilinear
// interpolation is linear, so each gathered line's deramp phasor (at its
// first column) merges with the pixel's reramp into one phasor, and the
// second column's sample turns by the small difference of the two columns'
// deramp phases; the pixel's kt and etaref come from the two table entries
// interpolated at its range.  The products differ from the unfused path's by
// float rounding.
//
// Culling (cull true): a DEM window is the bounding box of a burst footprint
// turned by the orbit heading, and about 40% of an IW burst's window lies
// before its first valid line or after its last.  Each warp fits a
// zero-height line model, affine in (row, column), to its corner solutions,
// with the line shift per metre of height; a block of 32 rows whose lines
// stay outside [first_valid_line + 5, last_valid_line - 5) at every int16
// height is written as zeros without solving its pixels.  Every pixel seeds
// its Newton iteration from the line model, so its result does not depend on
// whether the blocks before it were culled.
// Per-burst constants of the pixel loop.  The validity bounds and the
// line-0 times are kept as doubles here, formed by the same operations as
// the per-pixel expressions they replace: converting the plan's integers per
// pixel cost the pair kernel 6 % of its time.
struct GeoConsts {
  double inv_dmrg, prf, two_over_c, k4_wvl;  // k4_wvl: two-way range phase, half-cycles per metre
  double rg_lo, rg_hi, az_lo, az_hi;         // validity window fvs < rg < lvs - 1, fvl + 5 <= az < lvl - 5
  double eta0, ea0;                          // -lines dtaz / 2, -lines ati / 2: line 0 from the burst centre
  float ati_f;                               // ati in FP32
};

template <typename PL>
__device__ __forceinline__ GeoConsts geo_consts(const PL &P) {
  return GeoConsts{1.0 / P.dmrg, 1.0 / P.dtaz, 2.0 / kSolD, 4.0 / P.wvl,
                   (double)P.first_valid_sample, (double)(P.last_valid_sample - 1),
                   (double)(P.first_valid_line + 5), (double)(P.last_valid_line - 5),
                   -P.lines * P.dtaz / 2., -P.lines * P.ati / 2., (float)P.ati};
}

// Per-warp setup of one burst's geocoding.  The warp's pixels lie in window
// rows rT .. rB and columns cL .. cR (inside the window); tile row r is
// window row row0 + r.  One cubic orbit expansion per warp, at the
// zero-Doppler time of the warp's centre pixel, solved on the window
// polynomial from the burst centre (geo2rdr.cu:588-600).  The warp's 32 x RY
// pixels lie within ~0.2 s of it, where the dropped fourth-order term is
// < 1e-9 m.  Lanes 1 to 3 solve three corners at the same time; the four
// solutions bound the warp's footprint in the burst, whose lines are
// prefetched into L2 before the per-pixel solves, so the bilinear gathers
// hit L2, and give the line model that seeds and culls the pixel solves.
// Lane 0 writes the patch to zd and the seed model to seed; the result has
// bit j set when block j of 32 tile rows is culled.
// kPrefetch: prefetch the burst lines of the tile's footprint into L2.
template <int RY, typename TSrc, typename PL, bool kPrefetch = true>
__device__ __forceinline__ unsigned geo_warp_setup(const PL &P, const s1b_orbit_poly_t &orbit,
                                                   const int16_t *__restrict__ dem, int64_t pitch,
                                                   const TSrc *__restrict__ burst, int row0, int rT,
                                                   int rB, int cL, int cR, bool cull, ZeroDopplerPatch &zd,
                                                   double4 &seed) {
  const int lane = threadIdx.x & 31;
  const double inv_dmrg = 1.0 / P.dmrg, prf = 1.0 / P.dtaz;
  const int rC = min(rT + RY / 2, rB), cC = min(cL + 16, cR);
  double faz = 0.0, frg = 0.0, zl = 0.0, kl = 0.0;
  bool conv = true;
  if (lane < 4) {
    // lane 0: centre; 1: top left; 2: bottom right; 3: top right
    const int cr = lane == 0 ? rC : (lane == 2 ? rB : rT);
    const int cc = lane == 0 ? cC : (lane == 1 ? cL : cR);
    double sla, cla, slo, clo;
    sincos((P.lat0 + cr * P.dlat) * kPiD / 180, &sla, &cla);
    sincos((P.lon0 + cc * P.dlon) * kPiD / 180, &slo, &clo);
    const double hc = (double)__ldg(dem + (int64_t)cr * pitch + cc);
    const double rc = kRaD / sqrt(1. - kRe2D * sla * sla);
    const double pc[3] = {(rc + hc) * cla * clo, (rc + hc) * cla * slo, (rc * (1 - kRe2D) + hc) * sla};
    OrbitState st;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      st.x[i] = P.xmid[i];
      st.v[i] = P.vmid[i];
      st.a[i] = P.amid[i];
    }
    double tc = P.tmid, drc[3];
    conv = zero_doppler(orbit, pc, tc, st, drc) < 51;
    faz = (tc - P.tstart) * prf;
    frg = (sqrt(drc[0] * drc[0] + drc[1] * drc[1] + drc[2] * drc[2]) - P.rngstart) * inv_dmrg;
    // lines per metre of height: the zero-Doppler condition (p - X).V = 0
    // moved along the ellipsoid normal n = dp/dh gives
    // dt/dh = -(V.n) / ((p - X).A - V.V)
    const double nrm[3] = {cla * clo, cla * slo, sla};
    double vn = 0.0, fp = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      vn = fma(st.v[i], nrm[i], vn);
      fp = fma(drc[i], st.a[i], fp);
      fp = fma(-st.v[i], st.v[i], fp);
    }
    kl = -vn * rcp_newton(fp) * prf;
    zl = faz - kl * hc;  // the point's line at zero height
    if (lane == 0) {
      OrbitCubic oc;
      orbit_cubic(orbit, tc, oc);
      zero_doppler_patch(oc, zd);
      zd.inv_c1 = rcp_newton(fp);  // f' at the centre point: the chord slope of the warp's pixels
    }
  }
  {
    double a0 = faz, a1 = faz, g0 = frg, g1 = frg;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
      const double a = __shfl_sync(0xffffffffu, faz, k), g = __shfl_sync(0xffffffffu, frg, k);
      a0 = fmin(a0, a);
      a1 = fmax(a1, a);
      g0 = fmin(g0, g);
      g1 = fmax(g1, g);
    }
    a0 = __shfl_sync(0xffffffffu, a0, 0);
    a1 = __shfl_sync(0xffffffffu, a1, 0);
    g0 = __shfl_sync(0xffffffffu, g0, 0);
    g1 = __shfl_sync(0xffffffffu, g1, 0);
    // footprint with a margin of 2 samples, clamped to the burst; skipped when
    // it is not a small patch (e.g. a warp far outside the burst)
    const int l0 = max(0, (int)fmax(a0 - 2.0, -1.0)), l1 = min(P.lines - 1, (int)fmin(a1 + 3.0, 1e9));
    const int s0 = max(0, (int)fmax(g0 - 2.0, -1.0)), s1 = min(P.samples - 1, (int)fmin(g1 + 3.0, 1e9));
    const int nl = l1 - l0 + 1;
    if (kPrefetch && nl > 0 && nl <= 3 * RY && s1 >= s0 && s1 - s0 < 256) {
      const int nch = (((s1 - s0 + 1) * (int)sizeof(TSrc)) + 127) / 128 + 1;  // 128-byte lines per line segment
      for (int k = lane; k < nl * nch; k += 32) {
        const int li = k / nch, ch = k - li * nch;
        const TSrc *ptr = burst + (size_t)(l0 + li) * P.samples + s0;
        const char *line = reinterpret_cast<const char *>(ptr) + ch * 128;
        if (line <= reinterpret_cast<const char *>(burst + (size_t)(l0 + li) * P.samples + s1))
          asm volatile("prefetch.global.L2 [%0];" ::"l"(line));
      }
    }
  }
  // Line model of the warp (identical in every lane): zero-height line
  // zTL + zr (row - rT) + zc (col - cL) from the top corners and the bottom
  // right one, plus kC lines per metre of height.  The centre's distance
  // from the model measures its curvature; the cull margin covers four times
  // that, the heights (-32768 .. 32767 m, the slope with a quarter to spare
  // for its change over the warp and with height) and 2 lines.
  // The seed model, as times from the centre's, in tile rows:
  // h = s.x + s.y col + s.z r + s.w hgt.
  unsigned cullmask = 0;
  const double zTL = __shfl_sync(0xffffffffu, zl, 1), zBR = __shfl_sync(0xffffffffu, zl, 2);
  const double zTR = __shfl_sync(0xffffffffu, zl, 3), zC = __shfl_sync(0xffffffffu, zl, 0);
  const double kC = __shfl_sync(0xffffffffu, kl, 0), fazC = __shfl_sync(0xffffffffu, faz, 0);
  const double zr = rB > rT ? (zBR - zTR) * rcp_newton(rB - rT) : 0.0;
  const double zc = cR > cL ? (zTR - zTL) * rcp_newton(cR - cL) : 0.0;
  const double kmax = fmax(fmax(fabs(kC), fabs(__shfl_sync(0xffffffffu, kl, 1))),
                           fmax(fabs(__shfl_sync(0xffffffffu, kl, 2)), fabs(__shfl_sync(0xffffffffu, kl, 3))));
  const double resid = fabs(zC - (zTL + zr * (rC - rT) + zc * (cC - cL)));
  const double slack = 2.0 + 4.0 * resid + 1.25 * 32768.0 * kmax;
  const int rTr = rT - row0, rBr = rB - row0;  // tile rows of the warp's first and last rows
  // every corner converged and the model is sound (NaN fails each test)
  if (__all_sync(0xffffffffu, conv) && cull && resid < 1.0 && slack < 1.0e4) {
    const double zcs = zc * (cR - cL);  // the model's change across the warp's columns
#pragma unroll
    for (int j = 0; j < RY / 32; ++j) {
      const int ra = max(32 * j, rTr), re = min(32 * j + 32, rBr + 1);
      const double za = zTL + zr * (ra - rTr), zb = zTL + zr * (re - 1 - rTr);
      const double lo = fmin(za, zb) + fmin(zcs, 0.0) - slack, hi = fmax(za, zb) + fmax(zcs, 0.0) + slack;
      if (ra < re && (hi < P.first_valid_line + 5 || lo >= P.last_valid_line - 5)) cullmask |= 1u << j;
    }
  }
  if (lane == 0)
    seed = make_double4((zTL - zr * rTr - zc * cL - fazC) * P.dtaz, zc * P.dtaz, zr * P.dtaz, kC * P.dtaz);
  return cullmask;
}

// One pixel of a burst's geocoding: ECEF point p of height hgt, tile row r,
// window column col.  `first` takes the chord slope of this point for the
// block (f' changes by < 1e-3 over 32 rows); every point starts from the
// warp's line model m, within ~1e-6 s of its root.  Returns the geocoded
// sample, 0 outside the validity window.
template <typename TSrc, bool kFused, typename PL>
__device__ __forceinline__ float2 geo_pixel(const PL &P, const GeoConsts &gc,
                                            const ZeroDopplerPatch &zd, const double4 &m, const double p[3],
                                            double hgt, int r, int col, bool first, double &inv_c1,
                                            const TSrc *__restrict__ burst, const double2 *__restrict__ tops) {
  float2 res = make_float2(0.f, 0.f);
  const ZeroDopplerPoint q = zero_doppler_point(zd, p);
  if (first) inv_c1 = rcp_newton(q.c1);
  double h = fma(m.w, hgt, fma(m.z, i32_to_f64(r), fma(m.y, i32_to_f64(col), m.x)));
  const double rng = sqrt_heron(zero_doppler_solve(q, zd.c3, inv_c1, h));
  const double t = zd.t0 + h;
  const double rgoff = (rng - P.rngstart) * gc.inv_dmrg;
  const double azoff = (t - P.tstart) * gc.prf;
  // validity window, geo2rdr.cu:208-209
  bool valid = rgoff > P.first_valid_sample && rgoff < P.last_valid_sample - 1 &&
               azoff >= P.first_valid_line + 5 && azoff < P.last_valid_line - 5;
  const int intr = (int)rgoff, inta = (int)azoff;
  // the 2x2 neighbourhood must lie inside the burst even if the validity
  // limits passed in exceed the raster
  valid = valid && intr >= 0 && intr + 1 < P.samples && inta >= 0 && inta + 1 < P.lines;
  if (valid) {
    const double eta = -P.lines * P.dtaz / 2. + t - P.tstart;
    const double frd = rgoff - i32_to_f64(intr);
    // bilinear interpolation of the deramped burst (geo2rdr.cu:220-237)
    const float fr = (float)frd, fa = (float)(azoff - i32_to_f64(inta));
    const size_t i1 = (size_t)inta * P.samples + intr;
    if constexpr (kFused) {
      // the samples' deramp phases -kt (eta_line - etaref)^2 and the
      // reramp + range phase (geo2rdr.cu:210-219, 238-243) in half-cycles
      const double2 t0 = __ldg(tops + intr), t1 = __ldg(tops + intr + 1);
      const double ed = eta - fma(frd, t1.y - t0.y, t0.y);
      const double hr = fma(-fma(frd, t1.x - t0.x, t0.x), ed * ed, gc.k4_wvl * rng);
      const double ea = deramp_eta(P, inta), eb = deramp_eta(P, inta + 1);
      double d0 = ea - t0.y, d1 = ea - t1.y;
      const double qa0 = t0.x * d0 * d0, qa1 = t1.x * d1 * d1;
      d0 = eb - t0.y;
      d1 = eb - t1.y;
      const double qb0 = t0.x * d0 * d0, qb1 = t1.x * d1 * d1;
      const float2 s2 = cmul(load_ro(burst + i1 + 1), rotation_pi(qa1 - qa0));
      const float2 s4 = cmul(load_ro(burst + i1 + P.samples + 1), rotation_pi(qb1 - qb0));
      const float2 ca = cmul(lerp2(load_ro(burst + i1), s2, fr), phasor_pi(hr + qa0));
      const float2 cb = cmul(lerp2(load_ro(burst + i1 + P.samples), s4, fr), phasor_pi(hr + qb0));
      res = lerp2(ca, cb, fa);
    } else {
      // per-pixel TOPS reramp (geo2rdr.cu:210-219); kt = ka ks / (ka - ks)
      // and etac = -fnc / ka share one reciprocal of ka (ka - ks)
      const double tr = rng * gc.two_over_c;
      double dt = tr - P.fm[0];
      const double ka = P.fm[1] + dt * (P.fm[2] + P.fm[3] * dt);
      dt = tr - P.dc[0];
      const double fnc = P.dc[1] + dt * (P.dc[2] + P.dc[3] * dt);
      const double kmk = ka - P.ks;
      const double inv = rcp_newton(ka * kmk);
      const double kt = ka * P.ks * (ka * inv);
      const double ed = eta - (-fnc * (kmk * inv) - P.etac0);
      const float2 c1 = lerp2(__ldg(burst + i1), __ldg(burst + i1 + 1), fr);
      const float2 c2 = lerp2(__ldg(burst + i1 + P.samples), __ldg(burst + i1 + P.samples + 1), fr);
      // range phase and reramp (geo2rdr.cu:238-243): 4 pi rng / wvl + pi kt ed^2
      // rad, formed in half-cycles
      res = cmul(lerp2(c1, c2, fa), phasor_pi(fma(kt, ed * ed, gc.k4_wvl * rng)));
    }
  }
  return res;
}

// ECEF point of a DEM pixel from its row terms (sin lat, cos lat, prime
// vertical radius), column terms and height (orbit.cu:20-27).
__device__ __forceinline__ void llh_point(double sinlat, double coslat, double re, double sinlon, double coslon,
                                          double hgt, double p[3]) {
  p[0] = (re + hgt) * coslat * coslon;
  p[1] = (re + hgt) * coslat * sinlon;
  p[2] = (re * (1 - kRe2D) + hgt) * sinlat;
}

template <int TX, int RY, typename TSrc = float2, bool kFused = false, typename PL = s1b_burst_plan_t>
__device__ __forceinline__ void geo2rdr_tile(const PL &P, const s1b_orbit_poly_t &orbit,
                                             const int16_t *__restrict__ dem, int64_t pitch,
                                             const TSrc *__restrict__ burst,
                                             float2 *__restrict__ out, int32_t *__restrict__ rows, int nrow,
                                             int ncol, int tile_x, int tile_y, bool cull,
                                             const double2 *__restrict__ tops = nullptr) {
  const int tx = threadIdx.x, lane = tx & 31;
  const int col = tile_x * TX + tx;
  static_assert(RY % 32 == 0, "tile rows");
  const int row0 = tile_y * RY;
  // llh->ECEF trigonometry (orbit.cu:20-27): lane l holds the row terms of
  // row r + l for the current 32 rows r .. r + 31 of the tile
  double r_sin = 0.0, r_cos = 0.0, r_re = 0.0;
  auto row_terms = [&](int r) {
    const double lat = (P.lat0 + (row0 + r + lane) * P.dlat) * kPiD / 180;
    sincos(lat, &r_sin, &r_cos);
    r_re = kRaD / sqrt(1. - kRe2D * r_sin * r_sin);
  };
  row_terms(0);
  double sinlon, coslon;
  sincos((P.lon0 + col * P.dlon) * kPiD / 180, &sinlon, &coslon);
  const bool colok = col < ncol;
  const GeoConsts gc = geo_consts(P);
  __shared__ ZeroDopplerPatch s_zd[TX / 32];
  __shared__ double4 s_seed[TX / 32];
  const int wid = tx >> 5;
  // the warp's pixels span rows row0 .. rB and columns cL .. cR of the window
  const int c0 = tile_x * TX + wid * 32;
  const int rmax = min(RY, nrow - row0);
  const unsigned cullmask = geo_warp_setup<RY>(P, orbit, dem, pitch, burst, row0, row0, row0 + rmax - 1,
                                               min(c0, ncol - 1), min(c0 + 31, ncol - 1), cull, s_zd[wid],
                                               s_seed[wid]);
  __syncwarp();  // lane 0's patch and seed models are visible to the warp
  const ZeroDopplerPatch &zd = s_zd[wid];
  double inv_c1 = 0.0;
  int16_t hn = colok && rmax > 0 && !(cullmask & 1u) ? __ldg(dem + (int64_t)row0 * pitch + col) : 0;
  int rlo = INT_MAX, rhi = -1;
  for (int r = 0; r < rmax; ++r) {
    if ((r & 31) == 0) {  // a new block of 32 rows (warp-uniform)
      if ((cullmask >> (r >> 5)) & 1u) {
        const int rend = min(r + 32, rmax);
        if (colok)
          for (; r < rend; ++r) __stcs(out + (size_t)(row0 + r) * ncol + col, make_float2(0.f, 0.f));
        // the next block's first height (none was loaded ahead)
        if (colok && r < rmax) hn = __ldg(dem + (int64_t)(row0 + r) * pitch + col);
        r = rend - 1;
        continue;
      }
      if (r > 0) row_terms(r);
    }
    const int row = row0 + r;
    const double sinlat = __shfl_sync(0xffffffffu, r_sin, r & 31);
    const double coslat = __shfl_sync(0xffffffffu, r_cos, r & 31);
    const double re = __shfl_sync(0xffffffffu, r_re, r & 31);
    const double hgt = i32_to_f64(hn);
    if (colok && r + 1 < rmax) hn = __ldg(dem + (int64_t)(row + 1) * pitch + col);
    float2 res = make_float2(0.f, 0.f);
    if (colok) {
      double p[3];
      llh_point(sinlat, coslat, re, sinlon, coslon, hgt, p);
      res = geo_pixel<TSrc, kFused>(P, gc, zd, s_seed[wid], p, hgt, r, col, (r & 31) == 0, inv_c1, burst, tops);
      __stcs(out + (size_t)row * ncol + col, res);
    }
    if (res.x != 0.f || res.y != 0.f) {
      rlo = min(rlo, row);
      rhi = row + 1;
    }
  }
  // first / last non-zero output row (geo2rdr.cu:86-128): the warp's extent
  // over its rows, one reduction pair per warp and tile (per-row
  // reductions on one address serialise in its L2 slice)
  rlo = __reduce_min_sync(0xffffffffu, rlo);
  rhi = __reduce_max_sync(0xffffffffu, rhi);
  if (lane == 0 && rows && rhi >= 0) {
    atomicMin(rows, rlo);
    atomicMax(rows + 1, rhi);
  }
}

// No register cap: on the 1500 x 21000 burst 32-row tiles at the compiler's
// 96 registers beat 72 registers and 64- or 128-row tiles (0.219 against
// 0.226-0.260 ms).
__global__ __launch_bounds__(G_TX) void geo2rdr_kernel(
    const __grid_constant__ s1b_burst_plan_t P, const int16_t *__restrict__ dem, int64_t pitch,
    const float2 *__restrict__ burst, float2 *__restrict__ out, int32_t *__restrict__ rows,
    int nrow, int ncol, bool cull) {
  geo2rdr_tile<G_TX, G_RY>(P, P.orbit, dem, pitch, burst, out, rows, nrow, ncol, blockIdx.x, blockIdx.y, cull);
}

// Zero-Doppler sample coordinates of every DEM pixel of a burst's window, as
// the geocoding solves them: the same per-warp orbit patch, line-model seeds
// and chord Newton (geo_warp_setup, zero_doppler_point, zero_doppler_solve)
// in tiles of kFrameGeoRows rows, as the frame's geocoding, with no culling
// and no gathers.  az = line (geo2rdr.cu:205-207 azoff), rg = sample (rgoff),
// float64 [nrow * ncol].
template <int TX, int RY>
__global__ __launch_bounds__(TX) void geo2rdr_grid_offsets_kernel(const __grid_constant__ s1b_burst_plan_t P,
                                                                  const int16_t *__restrict__ dem, int64_t pitch,
                                                                  double *__restrict__ az, double *__restrict__ rg,
                                                                  int nrow, int ncol) {
  const int tx = threadIdx.x, lane = tx & 31, wid = tx >> 5;
  const int col = blockIdx.x * TX + tx, row0 = blockIdx.y * RY;
  double r_sin = 0.0, r_cos = 0.0, r_re = 0.0;
  auto row_terms = [&](int r) {
    const double lat = (P.lat0 + (row0 + r + lane) * P.dlat) * kPiD / 180;
    sincos(lat, &r_sin, &r_cos);
    r_re = kRaD / sqrt(1. - kRe2D * r_sin * r_sin);
  };
  row_terms(0);
  double sinlon, coslon;
  sincos((P.lon0 + col * P.dlon) * kPiD / 180, &sinlon, &coslon);
  const bool colok = col < ncol;
  const GeoConsts gc = geo_consts(P);
  __shared__ ZeroDopplerPatch s_zd[TX / 32];
  __shared__ double4 s_seed[TX / 32];
  const int c0 = blockIdx.x * TX + wid * 32;
  const int rmax = min(RY, nrow - row0);
  geo_warp_setup<RY, float2, s1b_burst_plan_t, false>(P, P.orbit, dem, pitch, nullptr, row0, row0, row0 + rmax - 1,
                                                      min(c0, ncol - 1), min(c0 + 31, ncol - 1), false, s_zd[wid],
                                                      s_seed[wid]);
  __syncwarp();
  const ZeroDopplerPatch &zd = s_zd[wid];
  const double4 m = s_seed[wid];
  double inv_c1 = 0.0;
  for (int r = 0; r < rmax; ++r) {
    if ((r & 31) == 0 && r > 0) row_terms(r);
    const double sinlat = __shfl_sync(0xffffffffu, r_sin, r & 31);
    const double coslat = __shfl_sync(0xffffffffu, r_cos, r & 31);
    const double re = __shfl_sync(0xffffffffu, r_re, r & 31);
    if (!colok) continue;
    const double hgt = i32_to_f64(__ldg(dem + (int64_t)(row0 + r) * pitch + col));
    double p[3];
    llh_point(sinlat, coslat, re, sinlon, coslon, hgt, p);
    const ZeroDopplerPoint q = zero_doppler_point(zd, p);
    if ((r & 31) == 0) inv_c1 = rcp_newton(q.c1);
    double h = fma(m.w, hgt, fma(m.z, i32_to_f64(r), fma(m.y, i32_to_f64(col), m.x)));
    const double rng = sqrt_heron(zero_doppler_solve(q, zd.c3, inv_c1, h));
    const size_t o = (size_t)(row0 + r) * ncol + col;
    az[o] = (zd.t0 + h - P.tstart) * gc.prf;
    rg[o] = (rng - P.rngstart) * gc.inv_dmrg;
  }
}

// ------------------------------------------------------------ frame stages
// Persistent kernels over the flat tile space of every burst of a frame.
// Tiles are taken round-robin; the geocoding CTA copies the plan of the burst
// it works on (orbit polynomials included) into shared memory when the burst
// changes (consecutive tiles of a CTA usually stay in one burst).

__global__ void frame_init_kernel(const FrameDev d, s1b_frame_pair_t *pout) {
  for (int b = threadIdx.x; b < d.n_bursts; b += blockDim.x) {
    d.rows[2 * b] = d.bursts[b].nrow;
    d.rows[2 * b + 1] = -1;
  }
  for (int k = threadIdx.x; k < d.n_pairs; k += blockDim.x) pout[k].ok = 0;
}

// Burst owning flat tile `idx` (tile0 ascending); uniform over the CTA.
template <bool kGeo>
__device__ __forceinline__ int frame_burst_of(const FrameDev &d, int64_t idx) {
  int lo = 0, hi = d.n_bursts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int64_t s = kGeo ? d.bursts[mid].geo_tile0 : d.bursts[mid].deramp_tile0;
    if (s <= idx) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The scalar part of a burst plan, everything after its orbit polynomials,
// laid out as in s1b_burst_plan_t.  The frame's geocoding CTAs copy only
// this part to shared memory (0.34 KB instead of 12.5 KB), which leaves the
// SM's L1 to the bilinear gathers; the orbit polynomials, read only by the
// per-warp setup, stay in global memory.
struct PlanTail {
  int32_t lines, samples;
  int32_t first_valid_line, last_valid_line, first_valid_sample, last_valid_sample;
  int32_t win_left, win_top, win_right, win_bottom;
  int32_t rsc_nlat, rsc_nlon;
  double tstart, dtaz, ati;
  double rngstart, dmrg;
  double slant_range_time, range_sampling_rate;
  double wvl, k4pi_wvl;
  double tmid, xmid[3], vmid[3], amid[3];
  double ks, etac0;
  double fm[4];
  double dc[4];
  double lat0, lon0, dlat, dlon;
  double latlon_box[4];
};
#define S1B_TAIL_AT(f) (offsetof(s1b_burst_plan_t, f) - offsetof(s1b_burst_plan_t, lines) == offsetof(PlanTail, f))
static_assert(offsetof(s1b_burst_plan_t, lines) == sizeof(s1b_orbit_poly_t) &&
                  sizeof(s1b_burst_plan_t) - sizeof(s1b_orbit_poly_t) == sizeof(PlanTail) && S1B_TAIL_AT(tstart) &&
                  S1B_TAIL_AT(tmid) && S1B_TAIL_AT(fm) && S1B_TAIL_AT(lat0) && S1B_TAIL_AT(latlon_box),
              "plan tail layout");
#undef S1B_TAIL_AT
// The plan table is an array of 8-byte-aligned structs: copy in 8-byte words.
static_assert(sizeof(s1b_burst_plan_t) % 8 == 0 && alignof(s1b_burst_plan_t) == 8 &&
                  sizeof(s1b_orbit_poly_t) % 8 == 0, "plan layout");

__device__ __forceinline__ void frame_load_plan(PlanTail &sp, const s1b_burst_plan_t *src) {
  __syncthreads();  // every thread is done with the previous burst's plan
  const long long *s = reinterpret_cast<const long long *>(reinterpret_cast<const char *>(src) +
                                                           sizeof(s1b_orbit_poly_t));
  long long *d = reinterpret_cast<long long *>(&sp);
  for (int i = threadIdx.x; i < (int)(sizeof(PlanTail) / 8); i += blockDim.x) d[i] = s[i];
  __syncthreads();
}

// Deramp reads a dozen plan fields once per tile (uniform loads), so it
// takes the plan from the table directly.
template <int ROWS, typename TIn>
__global__ __launch_bounds__(256, 4) void frame_deramp_kernel(const FrameDev d, const FrameIO io) {
  for (int64_t idx = blockIdx.x; idx < d.n_deramp_tiles; idx += gridDim.x) {
    const int b = frame_burst_of<false>(d, idx);
    const s1b_burst_plan_t &sp = d.plans[b];
    const FrameBurst &fb = d.bursts[b];
    const int tiles_x = (sp.samples + kFrameDerampCols - 1) / kFrameDerampCols;
    const int64_t local = idx - fb.deramp_tile0;
    const int ty = (int)(local / tiles_x), tx = (int)(local - (int64_t)ty * tiles_x);
    const TIn *in = static_cast<const TIn *>(io.slc) + fb.slc_off;
    float2 *out = io.work + fb.der_off;
    const bool vec = sp.samples % 2 == 0 && (reinterpret_cast<uintptr_t>(in) % (2 * sizeof(TIn))) == 0 &&
                     (reinterpret_cast<uintptr_t>(out) % 16) == 0;
    if (vec)
      deramp_tile<true, ROWS>(sp, in, out, tx, ty);
    else
      deramp_tile<false, ROWS>(sp, in, out, tx, ty);
  }
}

// One CTA per tile: blockIdx.z indexes a list of bursts that share a load
// width, (x, y) is the tile inside the burst.  The grid spans the largest
// burst; CTAs past a smaller one return at once.  No tile search and no
// persistent loop, so each instantiation keeps the single-burst register
// budget and the hardware keeps every SM full of streaming CTAs.
template <bool kVec, int ROWS, typename TIn>
__global__ __launch_bounds__(256) void frame_deramp_grid_kernel(const FrameDev d, const FrameIO io,
                                                                const __grid_constant__ FrameBurstList list) {
  const int b = list.idx[blockIdx.z];
  const s1b_burst_plan_t &sp = d.plans[b];
  if ((int)blockIdx.x * kFrameDerampCols >= sp.samples || (int)blockIdx.y * ROWS >= sp.lines) return;
  const FrameBurst &fb = d.bursts[b];
  deramp_tile<kVec, ROWS>(sp, static_cast<const TIn *>(io.slc) + fb.slc_off, io.work + fb.der_off, blockIdx.x,
                          blockIdx.y);
}

template <bool kVec, typename TIn>
void launch_deramp_grid(const FrameDev &d, const FrameIO &io, int rows, const int32_t *bursts, int n,
                        cudaStream_t st) {
  for (int k0 = 0; k0 < n; k0 += kFrameListMax) {
    FrameBurstList list;
    list.n = n - k0 < kFrameListMax ? n - k0 : kFrameListMax;
    for (int k = 0; k < list.n; ++k) list.idx[k] = bursts[k0 + k];
    const dim3 grid((unsigned)d.deramp_tiles_x, (unsigned)d.deramp_tiles_y, (unsigned)list.n);
    switch (rows) {
      case 8: frame_deramp_grid_kernel<kVec, 8, TIn><<<grid, 256, 0, st>>>(d, io, list); break;
      case 16: frame_deramp_grid_kernel<kVec, 16, TIn><<<grid, 256, 0, st>>>(d, io, list); break;
      default: frame_deramp_grid_kernel<kVec, 32, TIn><<<grid, 256, 0, st>>>(d, io, list); break;
    }
  }
}

// One tile of the frame's geocoding: unfused from the burst's deramped copy,
// fused from its raw samples and its column table (both at der_off).
template <int TX, typename TSrc, bool kFused>
__device__ __forceinline__ void frame_geo_tile(const PlanTail &sp, const s1b_orbit_poly_t &orbit,
                                               const FrameBurst &fb, const FrameIO &io, int32_t *rows, int tx, int ty,
                                               bool cull) {
  const int16_t *dem = io.dem + (int64_t)sp.win_top * io.dem_pitch + sp.win_left;
  if constexpr (kFused)
    geo2rdr_tile<TX, kFrameGeoRows, TSrc, true>(sp, orbit, dem, io.dem_pitch,
                                                static_cast<const TSrc *>(io.slc) + fb.slc_off, io.work + fb.geo_off,
                                                rows, fb.nrow, fb.ncol, tx, ty, cull,
                                                reinterpret_cast<const double2 *>(io.work + fb.der_off));
  else
    geo2rdr_tile<TX, kFrameGeoRows>(sp, orbit, dem, io.dem_pitch, io.work + fb.der_off, io.work + fb.geo_off, rows,
                                    fb.nrow, fb.ncol, tx, ty, cull);
}

// Per-column TOPS coefficients of every burst for the fused geocoding:
// blockIdx.y = burst, a thread per column, written into the burst's
// deramped-copy slot of the workspace (unused when fused): S double2
// (-kt, etaref) for the per-burst gathers, then S float4 (kt, kt' - kt,
// etaref' - etaref, etaref) with ' the next column, the differences formed in
// FP64, for the pair kernel's FP32 phase differences.
__global__ void frame_tops_table_kernel(const FrameDev d, const FrameIO io) {
  const int b = blockIdx.y;
  const s1b_burst_plan_t &sp = d.plans[b];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= sp.samples) return;
  double kt, eref, kt1 = 0.0, eref1 = 0.0;
  tops_kt(sp, c, kt, eref);
  if (c + 1 < sp.samples) tops_kt(sp, c + 1, kt1, eref1);
  double2 *slot = reinterpret_cast<double2 *>(io.work + d.bursts[b].der_off);
  slot[c] = make_double2(-kt, eref);
  reinterpret_cast<float4 *>(slot + sp.samples)[c] =
      c + 1 < sp.samples ? make_float4((float)kt, (float)(kt1 - kt), (float)(eref1 - eref), (float)eref)
                         : make_float4((float)kt, 0.f, 0.f, (float)eref);
}

// Minimum resident CTAs the frame's geocoding kernels are compiled for: 72
// registers at TX 64 and 128, 64 at TX 256.
template <int TX>
constexpr int kGeoGridMinBlocks = TX == 256 ? 4 : 896 / TX;

template <int TX, typename TSrc, bool kFused>
__global__ __launch_bounds__(TX, kGeoGridMinBlocks<TX>) void frame_geo2rdr_kernel(const FrameDev d, const FrameIO io) {
  __shared__ __align__(16) PlanTail sp;
  int cur = -1;
  for (int64_t idx = blockIdx.x; idx < d.n_geo_tiles; idx += gridDim.x) {
    const int b = frame_burst_of<true>(d, idx);
    if (b != cur) {
      frame_load_plan(sp, d.plans + b);
      cur = b;
    }
    const FrameBurst &fb = d.bursts[b];
    const int tiles_x = (fb.ncol + TX - 1) / TX;
    const int64_t local = idx - fb.geo_tile0;
    const int ty = (int)(local / tiles_x), tx = (int)(local - (int64_t)ty * tiles_x);
    frame_geo_tile<TX, TSrc, kFused>(sp, d.plans[b].orbit, fb, io, d.rows + 2 * b, tx, ty, d.cull_geo != 0);
  }
}

// One CTA per tile: blockIdx.z is the burst, (x, y) the tile in its DEM
// window.  The CTA copies its burst's plan scalars to shared memory first:
// the pixel loop's plan scalars then come from shared memory rather than
// uniform global loads (measured 13.67 -> 13.28 ms per 27-pair frame).  The
// grid spans the largest window; CTAs past a smaller one return before the
// copy's barriers (a uniform test of the block index).  Registers are held
// to 72 (896 threads per SM) at TX 64 and 128 and to 64 at TX 256, with a
// few spills: geocoding of the 27-pair frame 9.16 -> 8.78 ms at TX 128 and
// 9.32 -> 8.91 ms at TX 256 against 80 registers.
template <int TX, typename TSrc, bool kFused>
__global__ __launch_bounds__(TX, kGeoGridMinBlocks<TX>) void frame_geo2rdr_grid_kernel(const FrameDev d, const FrameIO io) {
  __shared__ __align__(16) PlanTail sp;
  const int b = blockIdx.z;
  const FrameBurst &fb = d.bursts[b];
  if ((int)blockIdx.x * TX >= fb.ncol || (int)blockIdx.y * kFrameGeoRows >= fb.nrow) return;
  frame_load_plan(sp, d.plans + b);
  frame_geo_tile<TX, TSrc, kFused>(sp, d.plans[b].orbit, fb, io, d.rows + 2 * b, blockIdx.x, blockIdx.y,
                                   d.cull_geo != 0);
}

// Crossmul fused into the geocoding.  One CTA per tile of a pair's grid of
// look rows (blockIdx.z = pair) geocodes both bursts of the pair at every
// DEM pixel of the union of their windows -- the DEM height, the ECEF point
// and the row and column terms serve both -- and sums conj(ref) sec and the
// two powers down each column over `rowlook` rows (xm_accumulate, in the
// order crossmul_rows_tile sums them): one float4 per column and look row.
// The geocoded windows are never written; the crop rows are voted as the
// geocoding does.  A burst is zero outside its window, as the reference's
// crossmul reads a .gslc (zero-filled around its crop).  Tiles hold whole
// look rows, so no look row spans two CTAs and the sums need no atomics.
// Compiled for 5 CTAs per SM (96 registers): with two bursts' state per warp,
// 72 or 80 registers spill and measured slower (9.74, 9.81 against 9.60 ms
// per 27-pair frame).
constexpr int kXmTX = kFrameXmCols;  // columns per tile

// Both bursts of a pair at one DEM pixel (bit q of MASK: burst q is solved
// in this block; act[q]: the pixel lies in burst q's window).  The solves
// are straight-line (zero_doppler_solve2 with the warp patch's chord slope),
// so the two bursts' instruction streams interleave; gathers are predicated
// on the validity window.  Fused (raw samples + column table): the TOPS
// phases of the two gathered lines relative to the pixel's reramp are formed
// in FP32 from differences that are small by construction: with
// K = kt, u = eta_line - etaref_c0 and the pixel's eta - etaref = u + w,
//   kt_p (u + w)^2 - K0 u^2 = K0 w (2u + w) + frd (K1 - K0) (u + w)^2,
// a few half-cycles, so FP32 keeps them to ~1e-6 half-cycles; only the
// two-way range phase 4 R / wvl (~6e7 half-cycles) is reduced in FP64.  The
// phasors use the hardware sine and cosine (~4e-7 rad).  The column rotation
// of the second sample of a line is likewise
//   -K1 (u - de)^2 + K0 u^2 = K0 de (2u - de) - (K1 - K0) (u - de)^2.
template <typename TSrc, bool kFused, int MASK>
__device__ __forceinline__ void geo_pair_pixel(const PlanTail *sp, const GeoConsts *gc, const ZeroDopplerPatch *zd0,
                                               const ZeroDopplerPatch *zd1, const double4 *m0, const double4 *m1,
                                               const double p[3], double hgt, double rd, const double *hb,
                                               const bool *act, const TSrc *__restrict__ src0,
                                               const TSrc *__restrict__ src1, const float4 *__restrict__ tops0,
                                               const float4 *__restrict__ tops1, float2 *v) {
  double h[2], r2[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (!((MASK >> q) & 1)) continue;
    const ZeroDopplerPatch &z = q ? *zd1 : *zd0;
    const double4 &m = q ? *m1 : *m0;
    const ZeroDopplerPoint pt = zero_doppler_point(z, p);
    h[q] = fma(m.w, hgt, fma(m.z, rd, hb[q]));
    r2[q] = zero_doppler_solve2(pt, z.c3, z.inv_c1, h[q], act[q]);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    v[q] = make_float2(0.f, 0.f);
    if (!((MASK >> q) & 1)) continue;
    const PlanTail &P = sp[q];
    const ZeroDopplerPatch &z = q ? *zd1 : *zd0;
    const TSrc *burst = q ? src1 : src0;
    const double rng = sqrt_heron(r2[q]);
    const double t = z.t0 + h[q];
    const double rgoff = (rng - P.rngstart) * gc[q].inv_dmrg;
    const double azoff = (t - P.tstart) * gc[q].prf;
    // validity window, geo2rdr.cu:208-209, and the 2 x 2 neighbourhood inside the burst
    bool valid = act[q] && rgoff > gc[q].rg_lo && rgoff < gc[q].rg_hi && azoff >= gc[q].az_lo && azoff < gc[q].az_hi;
    const int intr = valid ? (int)rgoff : 0, inta = valid ? (int)azoff : 0;
    valid = valid && intr >= 0 && intr + 1 < P.samples && inta >= 0 && inta + 1 < P.lines;
    if (!valid) continue;
    const double frd = rgoff - i32_to_f64(intr);
    const float fr = (float)frd, fa = (float)(azoff - i32_to_f64(inta));
    const size_t i1 = (size_t)inta * P.samples + intr;
    const double eta = gc[q].eta0 + t - P.tstart;
    if constexpr (kFused) {
      const float4 tc = __ldg((q ? tops1 : tops0) + intr);  // (kt, kt' - kt, etaref' - etaref, etaref)
      const double ea = gc[q].ea0 + i32_to_f64(inta) * P.ati;  // deramp_eta(P, inta)
      const float k0 = tc.x, dk = tc.y, de = tc.z;
      const float u = (float)ea - tc.w, ati = gc[q].ati_f;
      const float w = fmaf(-fr, de, (float)(eta - ea));
      const float ub = u + ati, wb = w - ati, e = u + w;
      const float kfe = fr * dk * e * e;
      const float ta = fmaf(k0 * w, 2.f * u + w, kfe), tb = fmaf(k0 * wb, 2.f * ub + wb, kfe);
      const float ua = u - de, uc = ub - de;
      const float ra = fmaf(k0 * de, 2.f * u - de, -dk * ua * ua);
      const float rb = fmaf(k0 * de, 2.f * ub - de, -dk * uc * uc);
      const double hr = gc[q].k4_wvl * rng;  // two-way range phase, half-cycles
      const float rr = (float)fma(-2.0, rint(0.5 * hr), hr);
      const float2 s2 = cmul(load_ro(burst + i1 + 1), rotation_pi_f(ra));
      const float2 s4 = cmul(load_ro(burst + i1 + P.samples + 1), rotation_pi_f(rb));
      const float2 ca = cmul(lerp2(load_ro(burst + i1), s2, fr), phasor_pi_f(rr + ta));
      const float2 cb = cmul(lerp2(load_ro(burst + i1 + P.samples), s4, fr), phasor_pi_f(rr + tb));
      v[q] = lerp2(ca, cb, fa);
    } else {
      // per-pixel TOPS reramp of the deramped burst (geo2rdr.cu:210-219, 238-243)
      const double tr = rng * gc[q].two_over_c;
      double dt = tr - P.fm[0];
      const double ka = P.fm[1] + dt * (P.fm[2] + P.fm[3] * dt);
      dt = tr - P.dc[0];
      const double fnc = P.dc[1] + dt * (P.dc[2] + P.dc[3] * dt);
      const double kmk = ka - P.ks;
      const double inv = rcp_newton(ka * kmk);
      const double kt = ka * P.ks * (ka * inv);
      const double ed = eta - (-fnc * (kmk * inv) - P.etac0);
      const float2 a1 = lerp2(__ldg(burst + i1), __ldg(burst + i1 + 1), fr);
      const float2 a2 = lerp2(__ldg(burst + i1 + P.samples), __ldg(burst + i1 + P.samples + 1), fr);
      v[q] = cmul(lerp2(a1, a2, fa), phasor_pi(fma(kt, ed * ed, gc[q].k4_wvl * rng)));
    }
  }
}

template <typename TSrc, bool kFused>
__global__ __launch_bounds__(kXmTX, 5) void frame_geo_xmul_kernel(const FrameDev d, const FrameIO io) {
  constexpr int RY = kFrameGeoRows;
  __shared__ __align__(16) PlanTail sp[2];
  __shared__ ZeroDopplerPatch s_zd[2][kXmTX / 32];
  __shared__ double4 s_seed[2][kXmTX / 32];
  __shared__ GeoConsts s_gc[2];

  const FramePair pr = d.pairs[blockIdx.z];
  const int lrows = RY / d.rowlook;  // look rows per tile
  if ((int)blockIdx.x * kXmTX >= pr.part_cols || (int)blockIdx.y * lrows >= pr.part_rows) return;  // uniform
  {
    const long long *a = reinterpret_cast<const long long *>(&d.plans[pr.ref].lines);
    const long long *b = reinterpret_cast<const long long *>(&d.plans[pr.sec].lines);
    long long *ta = reinterpret_cast<long long *>(&sp[0]), *tb = reinterpret_cast<long long *>(&sp[1]);
    for (int i = threadIdx.x; i < (int)(sizeof(PlanTail) / 8); i += blockDim.x) {
      ta[i] = a[i];
      tb[i] = b[i];
    }
    __syncthreads();
    if (threadIdx.x < 2) s_gc[threadIdx.x] = geo_consts(sp[threadIdx.x]);
    __syncthreads();
  }
  const int tx = threadIdx.x, lane = tx & 31, wid = tx >> 5;
  const int R0 = pr.part_top + (int)blockIdx.y * lrows * d.rowlook;  // RSC row of tile row 0
  const int nr = min(lrows, pr.part_rows - (int)blockIdx.y * lrows) * d.rowlook;
  const int Cw = pr.part_left + (int)blockIdx.x * kXmTX + wid * 32;  // RSC column of the warp's lane 0
  const int C = Cw + lane;
  const bool colin = C < pr.part_left + pr.part_cols;
  // row and column terms on the RSC grid (the reference burst's plan)
  const PlanTail &P0 = sp[0];
  double r_sin = 0.0, r_cos = 0.0, r_re = 0.0;
  auto row_terms = [&](int r) {
    const double lat = (P0.lat0 + (R0 - P0.win_top + r + lane) * P0.dlat) * kPiD / 180;
    sincos(lat, &r_sin, &r_cos);
    r_re = kRaD / sqrt(1. - kRe2D * r_sin * r_sin);
  };
  double sinlon, coslon;
  sincos((P0.lon0 + (C - P0.win_left) * P0.dlon) * kPiD / 180, &sinlon, &coslon);
  // per burst: window row of tile row 0, window column of the thread, block masks
  int row0w[2], colw[2], nrw[2];
  unsigned off[2];  // bit j: block j of 32 rows culled or outside the window
  int rlim = 0;     // tile rows below rlim lie inside the hull of the two windows
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const PlanTail &P = sp[q];
    const FrameBurst &fb = d.bursts[q ? pr.sec : pr.ref];
    row0w[q] = R0 - P.win_top;
    colw[q] = C - P.win_left;
    nrw[q] = fb.nrow;
    rlim = max(rlim, min(nr, fb.nrow - row0w[q]));
    const int c0 = Cw - P.win_left;
    const int rT = max(row0w[q], 0), rB = min(row0w[q] + nr - 1, fb.nrow - 1);
    const int cL = max(c0, 0), cR = min(c0 + 31, fb.ncol - 1);
    off[q] = ~0u;
    if (rT <= rB && cL <= cR) {  // warp-uniform
      const int16_t *dem = io.dem + (int64_t)P.win_top * io.dem_pitch + P.win_left;
      const TSrc *src = kFused ? static_cast<const TSrc *>(io.slc) + fb.slc_off
                               : reinterpret_cast<const TSrc *>(io.work + fb.der_off);
      // no prefetch of the footprint: the pair's gathers are served better by
      // L2 without it (8.46 against 8.95 ms per frame with the tile's lines
      // prefetched, 9.1 ms with lines prefetched 4 or 8 rows ahead)
      off[q] = geo_warp_setup<RY, TSrc, PlanTail, false>(P, d.plans[q ? pr.sec : pr.ref].orbit, dem, io.dem_pitch,
                                                         src, row0w[q], rT, rB, cL, cR, d.cull_geo != 0,
                                                         s_zd[q][wid], s_seed[q][wid]);
#pragma unroll
      for (int j = 0; j < RY / 32; ++j)
        if (32 * j + 31 < rT - row0w[q] || 32 * j > rB - row0w[q]) off[q] |= 1u << j;
    }
    if (colw[q] < 0 || colw[q] >= fb.ncol) colw[q] = -1;  // the thread's column is outside this window
  }
  __syncwarp();  // lane 0's patch and seed models are visible to the warp
  // the seed model's column term of the thread's column, per burst
  const double hb[2] = {fma(s_seed[0][wid].y, i32_to_f64(colw[0]), s_seed[0][wid].x),
                        fma(s_seed[1][wid].y, i32_to_f64(colw[1]), s_seed[1][wid].x)};
  const TSrc *src0, *src1;
  // tile rows [alo, ahi) of each burst's window at the thread's column
  int alo[2], ahi[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    alo[q] = max(0, -row0w[q]);
    ahi[q] = colw[q] >= 0 ? max(alo[q], nrw[q] - row0w[q]) : alo[q];
  }
  const float4 *tops0 = nullptr, *tops1 = nullptr;
  {
    const FrameBurst &f0 = d.bursts[pr.ref], &f1 = d.bursts[pr.sec];
    if constexpr (kFused) {
      src0 = static_cast<const TSrc *>(io.slc) + f0.slc_off;
      src1 = static_cast<const TSrc *>(io.slc) + f1.slc_off;
      tops0 = reinterpret_cast<const float4 *>(io.work + f0.der_off) + sp[0].samples;
      tops1 = reinterpret_cast<const float4 *>(io.work + f1.der_off) + sp[1].samples;
    } else {
      src0 = reinterpret_cast<const TSrc *>(io.work + f0.der_off);
      src1 = reinterpret_cast<const TSrc *>(io.work + f1.der_off);
    }
  }
  const int16_t *demc = io.dem + (int64_t)R0 * io.dem_pitch + C;  // the thread's column at tile row 0
  float4 *part = reinterpret_cast<float4 *>(io.work + pr.part_off) +
                 (int64_t)blockIdx.y * lrows * pr.part_cols + (C - pr.part_left);
  float ir = 0.f, ii = 0.f, p1 = 0.f, p2 = 0.f;
  int lr = 0;  // rows summed into the current look row
  int rlo0 = INT_MAX, rhi0 = -1, rlo1 = INT_MAX, rhi1 = -1;
  // the rows rb .. rend - 1 of one block of 32, with the bursts of MASK solved
  auto block_rows = [&](auto mask_tag, int rb, int rend) {
    constexpr int MASK = decltype(mask_tag)::value;
    row_terms(rb);
    int16_t hn = colin && rb < rlim ? __ldg(demc + (int64_t)rb * io.dem_pitch) : 0;
    // two rows per trip: the second row's solve overlaps the first row's
    // gathers (8.32 against 8.48 ms per frame, although it spills 36 bytes)
#pragma unroll 2
    for (int r = rb; r < rend; ++r) {
      const double sinlat = __shfl_sync(0xffffffffu, r_sin, r & 31);
      const double coslat = __shfl_sync(0xffffffffu, r_cos, r & 31);
      const double re = __shfl_sync(0xffffffffu, r_re, r & 31);
      const double hgt = i32_to_f64(hn);
      if (colin && r + 1 < rend && r + 1 < rlim) hn = __ldg(demc + (int64_t)(r + 1) * io.dem_pitch);
      double p[3];
      llh_point(sinlat, coslat, re, sinlon, coslon, hgt, p);
      const bool act[2] = {r >= alo[0] && r < ahi[0], r >= alo[1] && r < ahi[1]};
      float2 v[2];
      geo_pair_pixel<TSrc, kFused, MASK>(sp, s_gc, &s_zd[0][wid], &s_zd[1][wid], &s_seed[0][wid], &s_seed[1][wid], p,
                                         hgt, i32_to_f64(r), hb, act,
                                         src0, src1, tops0, tops1, v);
      if ((MASK & 1) && (v[0].x != 0.f || v[0].y != 0.f)) {
        rlo0 = min(rlo0, r);
        rhi0 = r + 1;
      }
      if ((MASK & 2) && (v[1].x != 0.f || v[1].y != 0.f)) {
        rlo1 = min(rlo1, r);
        rhi1 = r + 1;
      }
      xm_accumulate(v[0], v[1], ir, ii, p1, p2);
      if (++lr == d.rowlook) {
        if (colin) __stcs(part, make_float4(ir, ii, p1, p2));
        part += pr.part_cols;
        ir = ii = p1 = p2 = 0.f;
        lr = 0;
      }
    }
  };
  for (int rb = 0; rb < nr; rb += 32) {
    const int rend = min(rb + 32, nr), j = rb >> 5;
    const bool on0 = !((off[0] >> j) & 1u), on1 = !((off[1] >> j) & 1u);  // warp-uniform
    if (on0 && on1) {
      block_rows(std::integral_constant<int, 3>{}, rb, rend);
    } else if (on0) {
      block_rows(std::integral_constant<int, 1>{}, rb, rend);
    } else if (on1) {
      block_rows(std::integral_constant<int, 2>{}, rb, rend);
    } else {
      // neither burst has a pixel to solve here: their samples are zero
      for (int r = rb; r < rend; ++r) {
        if (++lr == d.rowlook) {
          if (colin) __stcs(part, make_float4(ir, ii, p1, p2));
          part += pr.part_cols;
          ir = ii = p1 = p2 = 0.f;
          lr = 0;
        }
      }
    }
  }
  // crop rows of both windows (geo2rdr.cu:86-128), one reduction pair per warp
  rlo0 = __reduce_min_sync(0xffffffffu, rlo0);
  rhi0 = __reduce_max_sync(0xffffffffu, rhi0);
  rlo1 = __reduce_min_sync(0xffffffffu, rlo1);
  rhi1 = __reduce_max_sync(0xffffffffu, rhi1);
  if (lane == 0) {
    if (rhi0 >= 0) {
      atomicMin(d.rows + 2 * pr.ref, rlo0 + R0 - sp[0].win_top);
      atomicMax(d.rows + 2 * pr.ref + 1, rhi0 + R0 - sp[0].win_top);
    }
    if (rhi1 >= 0) {
      atomicMin(d.rows + 2 * pr.sec, rlo1 + R0 - sp[1].win_top);
      atomicMax(d.rows + 2 * pr.sec + 1, rhi1 + R0 - sp[1].win_top);
    }
  }
}

template <typename K>
int resident_ctas(K kernel, int threads) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return sms * per_sm;
}

// ------------------------------------------------- generic geometry kernels
__global__ void zero_doppler_kernel(const __grid_constant__ s1b_orbit_poly_t P, const double *xyz,
                                    int64_t n, double t0, double *tline, double *drout) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double p[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
  double t = t0;
  OrbitState st;
  orbit_eval(P, t, st);
  double dr[3];
  zero_doppler(P, p, t, st, dr);
  tline[i] = t;
  if (drout) {
    drout[3 * i] = dr[0];
    drout[3 * i + 1] = dr[1];
    drout[3 * i + 2] = dr[2];
  }
}

__global__ void llh2xyz_kernel(const double *llh, double *xyz, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double lat = llh[3 * i] * kPiD / 180, lon = llh[3 * i + 1] * kPiD / 180, h = llh[3 * i + 2];
  double sl, cl, so, co;
  sincos(lat, &sl, &cl);
  sincos(lon, &so, &co);
  const double re = kRaD / sqrt(1. - kRe2D * sl * sl);
  xyz[3 * i] = (re + h) * cl * co;
  xyz[3 * i + 1] = (re + h) * cl * so;
  xyz[3 * i + 2] = (re * (1 - kRe2D) + h) * sl;
}

// Line of sight and look angle of every pixel of an RSC grid
// (s1proc/utils.py:240-292, _los): the pixel's geodetic point (row lat, column
// lon, DEM height) to ECEF, its zero-Doppler time by Newton from t0 (the
// middle state vector's time, s1proc/orbit.py:168-188), the unit vector
// satellite -> point, stored as float32, and the look angle
// acos(clip(los32 . n, -1, 1)) in degrees with n = -(cos lat cos lon,
// cos lat sin lon, sin lat) formed from the float32 vector, as the reference
// casts before its dot product.  Grid coordinates are start + index * step
// with a separate multiply and add, as numpy.mgrid forms them.
__global__ void los_grid_kernel(const __grid_constant__ s1b_orbit_poly_t P, double t0, double lat0, double lat_step,
                                double lon0, double lon_step, const int16_t *__restrict__ dem, int64_t pitch,
                                int nrow, int ncol, float *__restrict__ los, float *__restrict__ theta) {
  const int col = blockIdx.y * blockDim.x + threadIdx.x, row = blockIdx.x;
  if (col >= ncol || row >= nrow) return;
  const double latd = __dadd_rn(__dmul_rn((double)row, lat_step), lat0);
  const double lond = __dadd_rn(__dmul_rn((double)col, lon_step), lon0);
  const double lat = latd * kPiD / 180, lon = lond * kPiD / 180, h = (double)__ldg(dem + (int64_t)row * pitch + col);
  double sl, cl, so, co;
  sincos(lat, &sl, &cl);
  sincos(lon, &so, &co);
  const double re = kRaD / sqrt(1. - kRe2D * sl * sl);
  const double p[3] = {(re + h) * cl * co, (re + h) * cl * so, (re * (1 - kRe2D) + h) * sl};
  OrbitState st;
  orbit_eval(P, t0, st);
  double t = t0, dr[3];
  zero_doppler(P, p, t, st, dr);
  const double inv = 1.0 / sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
  const float l0 = (float)(dr[0] * inv), l1 = (float)(dr[1] * inv), l2 = (float)(dr[2] * inv);
  const int64_t o = (int64_t)row * ncol + col;
  los[3 * o] = l0;
  los[3 * o + 1] = l1;
  los[3 * o + 2] = l2;
  const double n0 = -(cl * co), n1 = -(cl * so), n2 = -sl;
  double c = __dadd_rn(__dadd_rn(__dmul_rn((double)l0, n0), __dmul_rn((double)l1, n1)), __dmul_rn((double)l2, n2));
  c = fmin(fmax(c, -1.0), 1.0);
  theta[o] = (float)(acos(c) * (180.0 / kPiD));
}

// ECEF -> geodetic with the one-step Bowring formula of s1proc/geometry.py:166-193
// (the form bounds.cu uses), degrees and metres.
__global__ void xyz2llh_kernel(const double *xyz, double *llh, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
  const double q2 = 1.0 / (1.0 - kRe2D), q = sqrt(q2), q3 = q2 - 1.0, b = kRaD * sqrt(1 - kRe2D);
  double lon = atan2(y, x);
  if (y < 0 && lon > 0) lon -= kPiD;
  if (y > 0 && lon < 0) lon += kPiD;
  const double rp = sqrt(x * x + y * y);
  const double th = atan((z / rp) * q);
  const double st = sin(th), ct = cos(th);
  const double lat = atan((z + q3 * b * st * st * st) / (rp - kRe2D * kRaD * ct * ct * ct));
  const double sl = sin(lat);
  const double re = kRaD / sqrt(1.0 - kRe2D * sl * sl);
  llh[3 * i] = lat * (180.0 / kPiD);
  llh[3 * i + 1] = lon * (180.0 / kPiD);
  llh[3 * i + 2] = rp / cos(lat) - re;
}

template <typename TIn>
int launch_deramp(const char *name, const s1b_burst_plan_t *plan, const void *in, void *out, void *stream) {
  if (!plan || !in || !out) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, name);
  const int S = plan->samples, L = plan->lines;
  if (S < 1 || L < 1) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "deramp: empty burst");
  cudaStream_t st = (cudaStream_t)stream;
  dim3 grid((S + 511) / 512, (L + DERAMP_ROWS - 1) / DERAMP_ROWS);
  const bool vec = (S % 2 == 0) && ((uintptr_t)in % (2 * sizeof(TIn)) == 0) && ((uintptr_t)out % 16 == 0);
  if (vec)
    deramp_kernel<true, TIn><<<grid, 256, 0, st>>>(*plan, (const TIn *)in, (float2 *)out);
  else
    deramp_kernel<false, TIn><<<grid, 256, 0, st>>>(*plan, (const TIn *)in, (float2 *)out);
  return s1b_launch_status();
}

}  // namespace

extern "C" int s1b_deramp(const s1b_burst_plan_t *plan, const void *in, void *out, void *stream) {
  return launch_deramp<float2>("s1b_deramp: null argument", plan, in, out, stream);
}

extern "C" int s1b_deramp_ci16(const s1b_burst_plan_t *plan, const void *in, void *out, void *stream) {
  return launch_deramp<short2>("s1b_deramp_ci16: null argument", plan, in, out, stream);
}

extern "C" int s1b_geo2rdr(const s1b_burst_plan_t *plan, const int16_t *dem, int64_t dem_pitch,
                           const void *deramped, void *out, int32_t *rows, void *stream) {
  if (!plan || !dem || !deramped || !out)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr: null argument");
  const int nrow = plan->win_bottom - plan->win_top;
  const int ncol = plan->win_right - plan->win_left;
  if (nrow <= 0 || ncol <= 0) return s1b_fail(S1B_ERR_EMPTY, "s1b_geo2rdr: empty DEM window");
  if (dem_pitch < ncol) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr: dem_pitch < window width");
  cudaStream_t st = (cudaStream_t)stream;
  if (rows) {
    rows_init_kernel<<<1, 1, 0, st>>>(rows, nrow);
    int s = s1b_launch_status();
    if (s) return s;
  }
  dim3 grid((ncol + G_TX - 1) / G_TX, (nrow + G_RY - 1) / G_RY);
  if (grid.y > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_geo2rdr: DEM window too tall");
  geo2rdr_kernel<<<grid, G_TX, 0, st>>>(*plan, dem, dem_pitch, (const float2 *)deramped,
                                         (float2 *)out, rows, nrow, ncol, g_cull_geo != 0);
  return s1b_launch_status();
}

extern "C" int s1b_geo2rdr_grid_offsets(const s1b_burst_plan_t *plan, const int16_t *dem, int64_t dem_pitch,
                                        double *az, double *rg, void *stream) {
  if (!plan || !dem || !az || !rg) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr_grid_offsets: null argument");
  const int nrow = plan->win_bottom - plan->win_top;
  const int ncol = plan->win_right - plan->win_left;
  if (nrow <= 0 || ncol <= 0) return s1b_fail(S1B_ERR_EMPTY, "s1b_geo2rdr_grid_offsets: empty DEM window");
  if (dem_pitch < ncol)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_geo2rdr_grid_offsets: dem_pitch < window width");
  dim3 grid((ncol + G_TX - 1) / G_TX, (nrow + kFrameGeoRows - 1) / kFrameGeoRows);
  if (grid.y > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_geo2rdr_grid_offsets: DEM window too tall");
  geo2rdr_grid_offsets_kernel<G_TX, kFrameGeoRows><<<grid, G_TX, 0, (cudaStream_t)stream>>>(*plan, dem, dem_pitch,
                                                                                             az, rg, nrow, ncol);
  return s1b_launch_status();
}

extern "C" int s1b_set_geocode_culling(int32_t on) {
  const int prev = g_cull_geo;
  g_cull_geo = on ? 1 : 0;
  return prev;
}

extern "C" int s1b_zero_doppler(const s1b_orbit_poly_t *orbit, const double *xyz, int64_t n,
                                double tline0, double *tline, double *dr, void *stream) {
  if (!orbit || (n > 0 && (!xyz || !tline))) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_zero_doppler: null argument");
  if (n <= 0) return S1B_OK;
  zero_doppler_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*orbit, xyz, n, tline0, tline, dr);
  return s1b_launch_status();
}

extern "C" int s1b_llh2xyz(const double *llh, double *xyz, int64_t n, void *stream) {
  if (n > 0 && (!llh || !xyz)) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_llh2xyz: null argument");
  if (n <= 0) return S1B_OK;
  llh2xyz_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(llh, xyz, n);
  return s1b_launch_status();
}

extern "C" int s1b_los_grid(const s1b_orbit_poly_t *orbit, double t0, double lat0, double lat_step, double lon0,
                            double lon_step, const int16_t *dem, int64_t dem_pitch, int32_t nrow, int32_t ncol,
                            float *los, float *theta, void *stream) {
  if (!orbit || !dem || !los || !theta) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_los_grid: null argument");
  if (nrow < 0 || ncol < 0 || (ncol > 0 && dem_pitch < ncol))
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_los_grid: bad grid size or pitch");
  if (nrow == 0 || ncol == 0) return S1B_OK;
  if ((ncol + 127) / 128 > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_los_grid: grid too wide");
  const dim3 grid((unsigned)nrow, (unsigned)((ncol + 127) / 128));
  los_grid_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(*orbit, t0, lat0, lat_step, lon0, lon_step, dem, dem_pitch,
                                                          nrow, ncol, los, theta);
  return s1b_launch_status();
}

extern "C" int s1b_xyz2llh(const double *xyz, double *llh, int64_t n, void *stream) {
  if (n > 0 && (!xyz || !llh)) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_xyz2llh: null argument");
  if (n <= 0) return S1B_OK;
  xyz2llh_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(xyz, llh, n);
  return s1b_launch_status();
}

// ------------------------------------------------------------ frame launchers
int frame_launch_init(const FrameDev &d, const FrameIO &io, cudaStream_t st) {
  frame_init_kernel<<<1, 256, 0, st>>>(d, io.pout);
  return s1b_launch_status();
}

int frame_max_ctas_deramp(int rows) {
  switch (rows) {
    case 8: return resident_ctas(frame_deramp_kernel<8, float2>, 256);
    case 16: return resident_ctas(frame_deramp_kernel<16, float2>, 256);
    case 32: return resident_ctas(frame_deramp_kernel<32, float2>, 256);
    default: return 0;
  }
}

template <typename TSrc, bool kFused>
int max_ctas_geo(int cols) {
  switch (cols) {
    case 64: return resident_ctas(frame_geo2rdr_kernel<64, TSrc, kFused>, 64);
    case 128: return resident_ctas(frame_geo2rdr_kernel<128, TSrc, kFused>, 128);
    case 256: return resident_ctas(frame_geo2rdr_kernel<256, TSrc, kFused>, 256);
    default: return 0;
  }
}

int frame_max_ctas_geo2rdr(const FrameDev &d, int cols) {
  if (!d.fused_deramp) return max_ctas_geo<float2, false>(cols);
  return d.sample_format == S1B_SAMPLES_CI16 ? max_ctas_geo<short2, true>(cols) : max_ctas_geo<float2, true>(cols);
}

int frame_launch_deramp(const FrameDev &d, const FrameIO &io, int rows, int ctas, const FrameDerampSplit &split,
                        cudaStream_t st) {
  const int full = frame_max_ctas_deramp(rows);
  if (full <= 0) return s1b_fail(S1B_ERR_UNSUPPORTED, "frame deramp: tile rows must be 8, 16 or 32");
  if (d.n_deramp_tiles == 0) return S1B_OK;
  if (d.fused_deramp) {  // the geocoding deramps its gathers: only the column tables
    const int ncols = d.deramp_tiles_x * kFrameDerampCols;
    frame_tops_table_kernel<<<dim3((unsigned)((ncols + 255) / 256), (unsigned)d.n_bursts), 256, 0, st>>>(d, io);
    return s1b_launch_status();
  }
  const bool ci16 = d.sample_format == S1B_SAMPLES_CI16;
  if (ctas == 0) {  // one CTA per tile, one launch per load width
    if (ci16) {
      launch_deramp_grid<true, short2>(d, io, rows, split.vec.data(), (int)split.vec.size(), st);
      launch_deramp_grid<false, short2>(d, io, rows, split.scalar.data(), (int)split.scalar.size(), st);
    } else {
      launch_deramp_grid<true, float2>(d, io, rows, split.vec.data(), (int)split.vec.size(), st);
      launch_deramp_grid<false, float2>(d, io, rows, split.scalar.data(), (int)split.scalar.size(), st);
    }
    return s1b_launch_status();
  }
  long long g = ctas < full ? ctas : full;
  if (g > d.n_deramp_tiles) g = d.n_deramp_tiles;
  if (ci16) {
    switch (rows) {
      case 8: frame_deramp_kernel<8, short2><<<(unsigned)g, 256, 0, st>>>(d, io); break;
      case 16: frame_deramp_kernel<16, short2><<<(unsigned)g, 256, 0, st>>>(d, io); break;
      default: frame_deramp_kernel<32, short2><<<(unsigned)g, 256, 0, st>>>(d, io); break;
    }
  } else {
    switch (rows) {
      case 8: frame_deramp_kernel<8, float2><<<(unsigned)g, 256, 0, st>>>(d, io); break;
      case 16: frame_deramp_kernel<16, float2><<<(unsigned)g, 256, 0, st>>>(d, io); break;
      default: frame_deramp_kernel<32, float2><<<(unsigned)g, 256, 0, st>>>(d, io); break;
    }
  }
  return s1b_launch_status();
}

template <typename TSrc, bool kFused>
int launch_geo(const FrameDev &d, const FrameIO &io, int cols, int ctas, cudaStream_t st) {
  const int full = max_ctas_geo<TSrc, kFused>(cols);
  if (full <= 0) return s1b_fail(S1B_ERR_UNSUPPORTED, "frame geo2rdr: tile columns must be 64, 128 or 256");
  if (d.n_geo_tiles == 0) return S1B_OK;
  if (ctas == 0) {  // one CTA per tile
    const dim3 grid((unsigned)d.geo_tiles_x, (unsigned)d.geo_tiles_y, (unsigned)d.n_bursts);
    switch (cols) {
      case 64: frame_geo2rdr_grid_kernel<64, TSrc, kFused><<<grid, 64, 0, st>>>(d, io); break;
      case 128: frame_geo2rdr_grid_kernel<128, TSrc, kFused><<<grid, 128, 0, st>>>(d, io); break;
      default: frame_geo2rdr_grid_kernel<256, TSrc, kFused><<<grid, 256, 0, st>>>(d, io); break;
    }
    return s1b_launch_status();
  }
  long long g = ctas < full ? ctas : full;
  if (g > d.n_geo_tiles) g = d.n_geo_tiles;
  switch (cols) {
    case 64: frame_geo2rdr_kernel<64, TSrc, kFused><<<(unsigned)g, 64, 0, st>>>(d, io); break;
    case 128: frame_geo2rdr_kernel<128, TSrc, kFused><<<(unsigned)g, 128, 0, st>>>(d, io); break;
    default: frame_geo2rdr_kernel<256, TSrc, kFused><<<(unsigned)g, 256, 0, st>>>(d, io); break;
  }
  return s1b_launch_status();
}

template <typename TSrc, bool kFused>
int launch_geo_xmul(const FrameDev &d, const FrameIO &io, cudaStream_t st) {
  if (d.xm_tiles_x <= 0 || d.xm_tiles_y <= 0) return S1B_OK;
  if (d.xm_tiles_y > 65535 || d.n_pairs > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "frame geo2rdr: grid too large");
  frame_geo_xmul_kernel<TSrc, kFused>
      <<<dim3((unsigned)d.xm_tiles_x, (unsigned)d.xm_tiles_y, (unsigned)d.n_pairs), kXmTX, 0, st>>>(d, io);
  return s1b_launch_status();
}

int frame_launch_geo2rdr(const FrameDev &dev, const FrameIO &io, int cols, int ctas, cudaStream_t st) {
  FrameDev d = dev;
  d.cull_geo = g_cull_geo;
  if (d.fused_xmul) {  // crossmul look-row sums instead of geocoded windows (tile shape fixed)
    if (!d.fused_deramp) return launch_geo_xmul<float2, false>(d, io, st);
    return d.sample_format == S1B_SAMPLES_CI16 ? launch_geo_xmul<short2, true>(d, io, st)
                                               : launch_geo_xmul<float2, true>(d, io, st);
  }
  if (!d.fused_deramp) return launch_geo<float2, false>(d, io, cols, ctas, st);
  return d.sample_format == S1B_SAMPLES_CI16 ? launch_geo<short2, true>(d, io, cols, ctas, st)
                                             : launch_geo<float2, true>(d, io, cols, ctas, st);
}

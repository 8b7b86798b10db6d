// Radar-grid coregistration on sm_100a: secondary sample offsets from
// float64 lat/lon/height rasters of the reference grid, TOPS-aware resampling
// of the secondary onto the reference grid (8-tap windowed sinc or
// bilinear), and boxcar coherence at full resolution.
//
// The reference geocodes every SLC onto a lat/lon grid instead
// (csrc/src/geo2rdr.cu:170-248); this mode has no reference counterpart.  It
// reuses the reference's geometry (orbit interpolant, zero-Doppler
// condition, range/azimuth sample formulas geo2rdr.cu:205-207) and its TOPS
// phase (geo2rdr.cu:151-152, 210-219).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <climits>
#include <mutex>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_internal.h"

namespace {

constexpr double kRaD = 6378137.0;
constexpr double kRe2D = 0.00669437999015;

// -------------------------------------------------------------- offsets
// Same column walk as the geocoding kernel: thread = reference column, the
// pixel above seeds the zero-Doppler Newton.
constexpr int O_TX = 128, O_RY = 16;

__global__ __launch_bounds__(O_TX) void offsets_kernel(const __grid_constant__ s1b_burst_plan_t P,
                                                       const double *__restrict__ lat,
                                                       const double *__restrict__ lon,
                                                       const double *__restrict__ hgt, int L, int S,
                                                       float *__restrict__ az_off,
                                                       float *__restrict__ rg_off) {
  const int col = blockIdx.x * O_TX + threadIdx.x;
  const int row0 = blockIdx.y * O_RY;
  if (col >= S) return;
  const double inv_dmrg = 1.0 / P.dmrg, prf = 1.0 / P.dtaz;
  double t = P.tmid;
  OrbitState st;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    st.x[i] = P.xmid[i];
    st.v[i] = P.vmid[i];
    st.a[i] = P.amid[i];
  }
  const int rmax = min(O_RY, L - row0);
  for (int r = 0; r < rmax; ++r) {
    const int row = row0 + r;
    const size_t i = (size_t)row * S + col;
    double sl, cl, so, co;
    sincospi(__ldcs(lat + i) * (1.0 / 180.0), &sl, &cl);
    sincospi(__ldcs(lon + i) * (1.0 / 180.0), &so, &co);
    const double h = __ldcs(hgt + i);
    const double re = kRaD / sqrt(1. - kRe2D * sl * sl);  // orbit.cu:27-30
    double p[3] = {(re + h) * cl * co, (re + h) * cl * so, (re * (1 - kRe2D) + h) * sl};
    double dr[3];
    zero_doppler(P.orbit, p, t, st, dr);
    const double rng = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    // residuals relative to the pixel index keep float32 at ~1e-5 px
    __stcs(az_off + i, (float)((t - P.tstart) * prf - row));
    __stcs(rg_off + i, (float)((rng - P.rngstart) * inv_dmrg - col));
  }
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

// TOPS coefficients at a continuous range sample: -pi kt and etaref
// (geo2rdr.cu:533-541 with i the fractional sample).
__device__ __forceinline__ void tops_range(const s1b_burst_plan_t &P, double rs, double &mkt, double &etaref) {
  const double tr = P.slant_range_time + rs / P.range_sampling_rate;
  double dt = tr - P.fm[0];
  const double ka = P.fm[1] + dt * (P.fm[2] + P.fm[3] * dt);
  dt = tr - P.dc[0];
  const double fnc = P.dc[1] + dt * (P.dc[2] + P.dc[3] * dt);
  const double kmk = ka - P.ks;
  const double inv = 1.0 / (ka * kmk);
  mkt = -kPiD * (ka * P.ks * (ka * inv));
  etaref = -fnc * (kmk * inv) - P.etac0;
}

__device__ __forceinline__ float2 deramped_tap(const s1b_burst_plan_t &P, const float2 *sec, int r, int c) {
  const float2 v = __ldg(sec + (size_t)r * P.samples + c);
  double mkt, etaref;
  tops_range(P, (double)c, mkt, etaref);
  const double d = (-P.lines * P.ati / 2. + r * P.ati) - etaref;
  return cmul(v, phasor(mkt * d * d));
}

__device__ __forceinline__ float2 fma2(float w, float2 v, float2 acc) {
  return __ffma2_rn(make_float2(w, w), v, acc);
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
  if (tid == 0) {
    s_red[0] = INT_MAX;
    s_red[1] = INT_MIN;
    s_red[2] = INT_MAX;
    s_red[3] = INT_MIN;
  }
  double az[R_RPT], rg[R_RPT];
  int na[R_RPT], nr[R_RPT];
  bool in[R_RPT], ok[R_RPT];
  int mna = INT_MAX, xna = INT_MIN, mnr = INT_MAX, xnr = INT_MIN;
#pragma unroll
  for (int q = 0; q < R_RPT; ++q) {
    const int row = rowb + q;
    in[q] = row < L && col < S;
    ok[q] = false;
    na[q] = 0;
    nr[q] = 0;
    if (in[q]) {
      const size_t i = (size_t)row * S + col;
      az[q] = row + (double)__ldg(az_off + i);
      rg[q] = col + (double)__ldg(rg_off + i);
      // the kernel support must lie inside the secondary burst
      const double fa = floor(az[q]), fr = floor(rg[q]);
      ok[q] = fa - lo >= 0.0 && fa + hi < (double)P.lines && fr - lo >= 0.0 && fr + hi < (double)P.samples;
      if (ok[q]) {
        na[q] = (int)fa;
        nr[q] = (int)fr;
        mna = min(mna, na[q]);
        xna = max(xna, na[q]);
        mnr = min(mnr, nr[q]);
        xnr = max(xnr, nr[q]);
      }
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
  const double eta0 = -P.lines * P.ati / 2.;
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
        const double u = (eta0 + (wa0 + r0) * P.ati) - eref;
        float2 ph = phasor(mkt * u * u);
        float2 step = phasor(mkt * P.ati * (2.0 * u + P.ati));
        const float2 dstep = phasor(2.0 * mkt * P.ati * P.ati);
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
  // fractions in [0, 1): a double fraction just below 1 can round to 1.0f,
  // which would put a sinc tap at distance 0 from the wrong sample
  float fa[R_RPT], fr[R_RPT];
#pragma unroll
  for (int q = 0; q < R_RPT; ++q) {
    fa[q] = fminf((float)(az[q] - na[q]), 0x1.fffffep-1f);
    fr[q] = fminf((float)(rg[q] - nr[q]), 0x1.fffffep-1f);
  }
  float2 acc[R_RPT];
#pragma unroll
  for (int q = 0; q < R_RPT; ++q) acc[q] = make_float2(0.f, 0.f);
  const bool block4 = staged && sinc && ok[0] && ok[1] && ok[2] && ok[3] && na[1] == na[0] + 1 &&
                      na[2] == na[0] + 2 && na[3] == na[0] + 3 && nr[1] == nr[0] && nr[2] == nr[0] &&
                      nr[3] == nr[0];
  if (block4) {
    // four outputs on consecutive lines: 11 tap rows shared by all four
    float wr[R_RPT][8], wa[R_RPT][8];
#pragma unroll
    for (int q = 0; q < R_RPT; ++q) {
      sinc8_weights(fr[q], wr[q]);
      sinc8_weights(fa[q], wa[q]);
    }
    const float2 *base = &win[na[0] - 3 - wa0][nr[0] - 3 - wr0];
#pragma unroll
    for (int rr = 0; rr < 8 + R_RPT - 1; ++rr) {
      float2 tap[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) tap[k] = base[rr * R_WCOLS + k];
#pragma unroll
      for (int q = 0; q < R_RPT; ++q) {
        const int ka = rr - q;  // tap row of output q
        if (ka < 0 || ka > 7) continue;
        float2 rs = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 8; ++k) rs = fma2(wr[q][k], tap[k], rs);
        acc[q] = fma2(wa[q][ka], rs, acc[q]);
      }
    }
  } else {
#pragma unroll 1
    for (int q = 0; q < R_RPT; ++q) {
      if (!ok[q]) continue;
      if (sinc) {
        float wr[8], wa[8];
        sinc8_weights(fr[q], wr);
        sinc8_weights(fa[q], wa);
        if (staged) {
          const float2 *base = &win[na[q] - 3 - wa0][nr[q] - 3 - wr0];
#pragma unroll
          for (int ka = 0; ka < 8; ++ka) {
            float2 rs = make_float2(0.f, 0.f);
#pragma unroll
            for (int kr = 0; kr < 8; ++kr) rs = fma2(wr[kr], base[ka * R_WCOLS + kr], rs);
            acc[q] = fma2(wa[ka], rs, acc[q]);
          }
        } else {
          for (int ka = 0; ka < 8; ++ka) {
            float2 rs = make_float2(0.f, 0.f);
            for (int kr = 0; kr < 8; ++kr) rs = fma2(wr[kr], deramped_tap(P, sec, na[q] + ka - 3, nr[q] + kr - 3), rs);
            acc[q] = fma2(wa[ka], rs, acc[q]);
          }
        }
      } else {
        float2 b[4];
        if (staged) {
#pragma unroll
          for (int k = 0; k < 4; ++k) b[k] = win[na[q] + (k >> 1) - wa0][nr[q] + (k & 1) - wr0];
        } else {
          for (int k = 0; k < 4; ++k) b[k] = deramped_tap(P, sec, na[q] + (k >> 1), nr[q] + (k & 1));
        }
        const float2 c1 = make_float2(fmaf(fr[q], b[1].x - b[0].x, b[0].x), fmaf(fr[q], b[1].y - b[0].y, b[0].y));
        const float2 c2 = make_float2(fmaf(fr[q], b[3].x - b[2].x, b[2].x), fmaf(fr[q], b[3].y - b[2].y, b[2].y));
        acc[q] = make_float2(fmaf(fa[q], c2.x - c1.x, c1.x), fmaf(fa[q], c2.y - c1.y, c1.y));
      }
    }
  }
  // reramp: restore the secondary's TOPS phase at the fractional position;
  // -pi kt and etaref at the fractional sample from the staged per-column
  // values (smooth in range: linear interpolation is exact to ~1e-7 rad)
#pragma unroll
  for (int q = 0; q < R_RPT; ++q) {
    if (!in[q]) continue;
    float2 v = make_float2(0.f, 0.f);
    if (ok[q]) {
      double mkt, eref;
      if (staged) {
        const int c = nr[q] - wr0;
        const double t = rg[q] - nr[q];
        mkt = s_mkt[c] + t * (s_mkt[c + 1] - s_mkt[c]);
        eref = s_eref[c] + t * (s_eref[c + 1] - s_eref[c]);
      } else {
        tops_range(P, rg[q], mkt, eref);
      }
      const double d = (eta0 + az[q] * P.ati) - eref;
      v = cmul(acc[q], phasor(-(mkt * d * d)));
    }
    __stcs(out + (size_t)(rowb + q) * S + col, v);
  }
}

// ------------------------------------------------------- box coherence
// Persistent kernel, one CTA of 512 threads per SM, output tiles of 128
// columns x 32 rows taken round-robin.  Both SLC tiles plus a halo are
// brought into shared memory by TMA (cp.async.bulk.tensor, zero fill
// outside the raster) through a two-stage pipeline: the next tile streams in
// while the current one is reduced.  The conj product and both powers are
// formed once per staged pixel in place; each thread then slides a window
// down one column (8 output rows): horizontal sums per row, a ring of the last
// `win` of them, and the vertical sum.  The vertical sum of the complex
// channel slides (add the entering row, subtract the leaving one) with Kahan
// compensation; the power sums, of non-negative terms, are summed directly.  Without a tensor map (odd width, unaligned base) tiles are staged
// by plain loads.
constexpr int C_TW = 128, C_TH = 32, C_HX = 4;  // halo columns (even, >= half window)
constexpr int C_IW = C_TW + 2 * C_HX;            // 136 staged columns
constexpr int C_MAXH = 4;                        // half window <= 4 (win <= 9)
constexpr int C_IH = C_TH + 2 * C_MAXH;          // 40 staged rows
constexpr int C_THREADS = 512, C_PARTS = C_THREADS / C_TW, C_ROWS = C_TH / C_PARTS;  // 4 parts x 8 rows
constexpr int C_STAGE = 2 * C_IH * C_IW;         // float2 per stage (ref + sec)
constexpr uint32_t kSpinLimit = 1u << 22;

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

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
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
  const int tx = threadIdx.x % C_TW, part = threadIdx.x / C_TW;
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
      const uint32_t b = smem_addr(&bars[k & 1]);
      if (!mbar_wait(b, (k >> 1) & 1)) {
        // never expected: record it, give the copies a second bounded wait so
        // none lands after the block exits, and stop
        if (threadIdx.x == 0) atomicExch(err, 1);
        mbar_wait(b, (k >> 1) & 1);
        return;
      }
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
    // products once per staged pixel, in place: sr <- conj(r) s, ss <- (|r|^2, |s|^2)
    for (int idx = threadIdx.x; idx < C_IH * C_IW; idx += C_THREADS) {
      const float2 a = sr[idx], b = ss[idx];
      float2 cp = __fmul2_rn(make_float2(a.x, a.x), b);
      cp = __ffma2_rn(make_float2(a.y, -a.y), make_float2(b.y, b.x), cp);
      const float2 xx = make_float2(a.x, b.x), yy = make_float2(a.y, b.y);
      sr[idx] = cp;
      ss[idx] = __ffma2_rn(yy, yy, __fmul2_rn(xx, xx));
    }
    __syncthreads();
    const int col = col0 + tx;
    const int orow0 = part * C_ROWS;
    const int first = orow0 + C_MAXH - HALF;  // staged row of the first window row
    // ring of the last WIN horizontal sums: (re, im) of conj(r)s and (|r|^2, |s|^2)
    float2 rc[WIN], rp[WIN];
    Kahan vre, vim;  // sliding, compensated sum of the complex channel
#pragma unroll
    for (int j = 0; j < C_ROWS + WIN - 1; ++j) {
      const float2 *pr = sr + (first + j) * C_IW + tx + C_HX - HALF;
      const float2 *pp = ss + (first + j) * C_IW + tx + C_HX - HALF;
      float2 hc = pr[0], hp = pp[0];
#pragma unroll
      for (int dx = 1; dx < WIN; ++dx) {
        hc = __fadd2_rn(hc, pr[dx]);
        hp = __fadd2_rn(hp, pp[dx]);
      }
      if (j >= WIN) {  // the row leaving the window
        vre.add(-rc[j % WIN].x);
        vim.add(-rc[j % WIN].y);
      }
      rc[j % WIN] = hc;
      rp[j % WIN] = hp;
      vre.add(hc.x);
      vim.add(hc.y);
      if (j >= WIN - 1) {
        // powers: direct sums of non-negative terms (exact zeros stay zero)
        float2 pw = rp[0];
#pragma unroll
        for (int q = 1; q < WIN; ++q) pw = __fadd2_rn(pw, rp[q]);
        const int orow = row0 + orow0 + (j - (WIN - 1));
        if (col < S && orow < L) {
          // |I| / sqrt(P1 P2) = sqrt(|I|^2) * rsqrt(P1 P2); 0 where a power is 0
          const float den2 = pw.x * pw.y;
          const float re = vre.value(), im = vim.value();
          const float num2 = fmaf(re, re, im * im);
          __stcs(coh + (size_t)orow * S + col, den2 > 0.f ? sqrtf(num2) * rsqrtf(den2) : 0.f);
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

// 2-D tensor map over a complex64 raster (8-byte elements), box C_IW x C_IH,
// zero fill outside.  False when the raster cannot be described (odd width,
// unaligned base) or the driver lacks the entry point.
bool make_tile_map(CUtensorMap *m, const void *base, int L, int S) {
  if (S % 2 != 0 || (reinterpret_cast<uintptr_t>(base) % 16) != 0) return false;
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)S, (cuuint64_t)L};
  cuuint64_t strides[1] = {(cuuint64_t)S * sizeof(float2)};
  cuuint32_t box[2] = {(cuuint32_t)C_IW, (cuuint32_t)C_IH};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
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
  offsets_kernel<<<grid, O_TX, 0, (cudaStream_t)stream>>>(*plan, lat, lon, hgt, lines, samples, az_off, rg_off);
  return s1b_launch_status();
}

extern "C" int s1b_resample(const s1b_burst_plan_t *plan, const void *sec, const float *az_off,
                            const float *rg_off, int32_t lines, int32_t samples, int32_t interp, void *out,
                            void *stream) {
  if (!plan || !sec || !az_off || !rg_off || !out)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_resample: null argument");
  if (interp != S1B_INTERP_BILINEAR && interp != S1B_INTERP_SINC8)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_resample: interp must be S1B_INTERP_BILINEAR or S1B_INTERP_SINC8");
  if (lines < 1 || samples < 1 || plan->lines < 2 || plan->samples < 2)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_resample: empty grid");
  int s = ensure_sinc_table();
  if (s) return s;
  dim3 block(R_TX, R_TY);
  dim3 grid((samples + R_TX - 1) / R_TX, (lines + R_TH - 1) / R_TH);
  if (grid.y > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_resample: grid too tall");
  resample_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(*plan, (const float2 *)sec, az_off, rg_off, lines,
                                                            samples, interp == S1B_INTERP_SINC8 ? 1 : 0,
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
  CUtensorMap mr, ms;
  const bool tma = make_tile_map(&mr, ref, lines, samples) && make_tile_map(&ms, sec, lines, samples);
  switch (win / 2) {
    case 0: return launch_box<0>(tma, mr, ms, ref, sec, lines, samples, coh, status, st);
    case 1: return launch_box<1>(tma, mr, ms, ref, sec, lines, samples, coh, status, st);
    case 2: return launch_box<2>(tma, mr, ms, ref, sec, lines, samples, coh, status, st);
    case 3: return launch_box<3>(tma, mr, ms, ref, sec, lines, samples, coh, status, st);
    default: return launch_box<4>(tma, mr, ms, ref, sec, lines, samples, coh, status, st);
  }
}

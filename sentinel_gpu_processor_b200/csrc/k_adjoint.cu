// Coherence objective of radar-grid coregistration and its hand-written
// adjoint, fused: resample -> crossmul -> multilook windows -> coherence
// (-> gradient), for a stack of bursts of one size.  No reference
// counterpart (the reference has no differentiable path); the geometry and
// TOPS phase are the reference's (csrc/src/geo2rdr.cu:151-152, 210-219).
//
// Model, per burst b and pixel (row, col) of the reference grid:
//   az = row + az0 + p0 + p1 xa + p2 xr + daz_dh dh
//   rg = col + rg0 + p3 + p4 xa + p5 xr + drg_dh dh,
//   xa = (row - L/2) / L, xr = (col - S/2) / S,
//   s  = reramp(az, rg) * sum_ka sum_kr wa(fa)[ka] wr(fr)[kr] deramp(sec)[na + ka - 3, nr + kr - 3]
// (8-tap windowed sinc, zero where the support leaves the burst); over the
// rl x cl windows of the multilook grid I = sum conj(r) s, P1 = sum |r|^2,
// P2 = sum |s|^2, gamma = |I| / sqrt(P1 P2); J = -sum gamma / (windows).
// Gradient of gamma w.r.t. s (real/imaginary parts as one complex number):
//   g = gamma (I r / |I|^2 - s / P2),  d gamma / d theta = Re(conj(g) ds/dtheta),
//   ds/daz = rot (acc_a + i dPhi/daz acc),  ds/drg = rot (acc_r + i dPhi/drg acc),
// with acc_a, acc_r the interpolations with the weight derivatives dw/df.
// The backward recomputes the window sums instead of storing them.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <mutex>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_internal.h"

struct s1b_adjoint {
  int device = 0;
  int n_bursts = 0, lines = 0, samples = 0, rowlook = 1, collook = 1;
  int tile_cols = 0, tiles_x = 0, tiles_y = 0;
  long long windows = 0;  // multilook windows over all bursts
  s1b_burst_plan_t *d_plans = nullptr;
};

namespace {

constexpr int A_TX = 64, A_TY = 4, A_RPT = 4, A_TH = A_TY * A_RPT;  // 16 rows x <= 64 columns
constexpr int A_WROWS = 32, A_WCOLS = 96;
// rows per deramp segment: at least two column groups share the window
// (A_TX * A_TY / A_WCOLS >= 2), so a segment has at most A_WROWS / 2 rows
constexpr int A_SEG = A_WROWS / 2;
static_assert(A_TX * A_TY / A_WCOLS >= 2, "deramp segments hold at most A_SEG rows");
constexpr int A_BINS = 1024;
constexpr int A_PARTS = 8;  // per-tile partials: 6 parameter sums, sum of gamma, windows

// Normalised 8-tap windowed-sinc weights and their derivatives d/df at
// A_BINS + 1 fractions (taps k = -3..4 at x = k - f: u = sinc(x) (0.5 + 0.5
// cos(pi x / 4)), w = u / sum u), from the host in double precision.
__device__ __align__(16) float g_w[(A_BINS + 1) * 8];
__device__ __align__(16) float g_dw[(A_BINS + 1) * 8];
std::mutex g_tab_mu;
bool g_tab_ready[64] = {};

cudaError_t set_smem_attributes();  // after the kernels (dynamic shared memory of the current device)

int ensure_tables() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return s1b_fail(S1B_ERR_UNSUPPORTED, "adjoint: device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_tab_mu);
  if (g_tab_ready[dev]) return S1B_OK;
  static float w[(A_BINS + 1) * 8], dw[(A_BINS + 1) * 8];
  for (int b = 0; b <= A_BINS; ++b) {
    const double f = (double)b / A_BINS;
    double u[8], du[8], su = 0.0, sdu = 0.0;
    for (int k = 0; k < 8; ++k) {
      const double x = (k - 3) - f;
      const double px = kPiD * x;
      const double sc = x == 0.0 ? 1.0 : std::sin(px) / px;
      const double dsc = x == 0.0 ? 0.0 : (std::cos(px) - sc) / x;  // d sinc / dx
      const double win = 0.5 + 0.5 * std::cos(px / 4.0);
      const double dwin = -0.125 * kPiD * std::sin(px / 4.0);
      u[k] = sc * win;
      du[k] = -(dsc * win + sc * dwin);  // d/df = -d/dx
      su += u[k];
      sdu += du[k];
    }
    for (int k = 0; k < 8; ++k) {
      w[b * 8 + k] = (float)(u[k] / su);
      dw[b * 8 + k] = (float)((du[k] * su - u[k] * sdu) / (su * su));
    }
  }
  e = cudaMemcpyToSymbol(g_w, w, sizeof(w));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_dw, dw, sizeof(dw));
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  e = set_smem_attributes();
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  g_tab_ready[dev] = true;
  return S1B_OK;
}

// Weights (or derivatives) at fraction f by linear interpolation of a table.
__device__ __forceinline__ void lut8(const float *tab, float f, float w[8]) {
  const float pos = f * A_BINS;
  const int b = min((int)pos, A_BINS - 1);
  const float t = pos - (float)b;
  const float4 *T = reinterpret_cast<const float4 *>(tab) + 2 * b;
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

__device__ __forceinline__ float2 fma2(float w, float2 v, float2 acc) {
  return __ffma2_rn(make_float2(w, w), v, acc);
}

// TOPS terms at a continuous range sample, phase in half-cycles: -kt and
// etaref (geo2rdr.cu:533-541 with the sample index fractional).
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

struct AdjArgs {
  const s1b_burst_plan_t *plans;
  const float2 *ref, *sec;
  const float *az0, *rg0, *daz_dh, *drg_dh, *params, *dh;
  float *grad_dh;
  double *partials;  // [n_bursts * tiles][A_PARTS]
  int L, S, rl, cl, tile_cols, tiles_x, tiles_per_burst;
  float inv_windows;  // 1 / (windows over all bursts)
};

struct AdjSmem {
  float2 win[A_WROWS][A_WCOLS];  // deramped secondary window
  double mkt[A_WCOLS], eref[A_WCOLS];
  float2 r[A_TH][A_TX], s[A_TH][A_TX], da[A_TH][A_TX], dr[A_TH][A_TX];
  float4 pix[A_TH][A_TX];  // per pixel: Re I, Im I, P1, P2; then per window at its first pixel: A I, B, gamma
  double part[A_TX * A_TY / 32][A_PARTS];
  int red[4];
};

// 8 x 8 taps of one pixel: value and, with kGrad, the range / azimuth
// derivative interpolations.  tap(ka, kr) returns the deramped sample.
template <bool kGrad, typename Tap>
__device__ __forceinline__ void interp_taps(const float wr[8], const float wa[8], const float dwr[8],
                                            const float dwa[8], Tap tap, float2 &acc, float2 &acc_a,
                                            float2 &acc_r) {
#pragma unroll
  for (int ka = 0; ka < 8; ++ka) {
    float2 rs = make_float2(0.f, 0.f), rsd = rs;
#pragma unroll
    for (int kr = 0; kr < 8; ++kr) {
      const float2 v = tap(ka, kr);
      rs = fma2(wr[kr], v, rs);
      if (kGrad) rsd = fma2(dwr[kr], v, rsd);
    }
    acc = fma2(wa[ka], rs, acc);
    if (kGrad) {
      acc_a = fma2(dwa[ka], rs, acc_a);
      acc_r = fma2(wa[ka], rsd, acc_r);
    }
  }
}

template <bool kGrad>
__global__ __launch_bounds__(A_TX *A_TY, 2) void adjoint_kernel(const AdjArgs a) {
  extern __shared__ __align__(16) unsigned char adj_raw[];
  AdjSmem &sm = *reinterpret_cast<AdjSmem *>(adj_raw);
  const int b = blockIdx.y;
  const s1b_burst_plan_t &P = a.plans[b];
  const int tile = blockIdx.x;
  const int tile_y = tile / a.tiles_x, tile_x = tile - tile_y * a.tiles_x;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * A_TX + tx;
  const int L = a.L, S = a.S;
  const int col = tile_x * a.tile_cols + tx;
  const int row0 = tile_y * A_TH;
  const int nwr = L / a.rl, nwc = S / a.cl;  // multilook grid
  const bool colin = tx < a.tile_cols && col < nwc * a.cl;
  const size_t boff = (size_t)b * L * S;
  const float *pr = a.params + 6 * b;
  const float p0 = pr[0], p1 = pr[1], p2 = pr[2], p3 = pr[3], p4 = pr[4], p5 = pr[5];
  if (tid == 0) {
    sm.red[0] = INT_MAX;
    sm.red[1] = INT_MIN;
    sm.red[2] = INT_MAX;
    sm.red[3] = INT_MIN;
  }
  // coordinates of the thread's 4 pixels
  int na[A_RPT], nr[A_RPT];
  float fa[A_RPT], fr[A_RPT];
  bool ok[A_RPT], in[A_RPT];
  double azd[A_RPT], rgd[A_RPT];
  int mna = INT_MAX, xna = INT_MIN, mnr = INT_MAX, xnr = INT_MIN;
  const float xr = ((float)col - 0.5f * S) / S;
#pragma unroll
  for (int q = 0; q < A_RPT; ++q) {
    const int row = row0 + ty * A_RPT + q;
    in[q] = colin && row < nwr * a.rl;
    ok[q] = false;
    na[q] = nr[q] = 0;
    fa[q] = fr[q] = 0.f;
    azd[q] = rgd[q] = 0.0;
    if (in[q]) {
      const size_t i = boff + (size_t)row * S + col;
      const float xa = ((float)row - 0.5f * L) / L;
      const float h = __ldg(a.dh + i);
      const float oa = __ldg(a.az0 + i) + fmaf(p2, xr, fmaf(p1, xa, p0)) + __ldg(a.daz_dh + i) * h;
      const float orr = __ldg(a.rg0 + i) + fmaf(p5, xr, fmaf(p4, xa, p3)) + __ldg(a.drg_dh + i) * h;
      if (fabsf(oa) < 0x1p20f && fabsf(orr) < 0x1p20f) {
        const float fla = floorf(oa), flr = floorf(orr);
        na[q] = row + (int)fla;
        nr[q] = col + (int)flr;
        fa[q] = fminf(oa - fla, 0x1.fffffep-1f);
        fr[q] = fminf(orr - flr, 0x1.fffffep-1f);
        azd[q] = (double)na[q] + (double)fa[q];
        rgd[q] = (double)nr[q] + (double)fr[q];
        ok[q] = na[q] - 3 >= 0 && na[q] + 4 < P.lines && nr[q] - 3 >= 0 && nr[q] + 4 < P.samples;
      }
      if (ok[q]) {
        mna = min(mna, na[q]);
        xna = max(xna, na[q]);
        mnr = min(mnr, nr[q]);
        xnr = max(xnr, nr[q]);
      }
    }
  }
  __syncthreads();
  if (mna <= xna) {
    atomicMin(&sm.red[0], mna);
    atomicMax(&sm.red[1], xna);
    atomicMin(&sm.red[2], mnr);
    atomicMax(&sm.red[3], xnr);
  }
  __syncthreads();
  const int wa0 = sm.red[0] - 3, wr0 = sm.red[2] - 3;
  const int wrows = sm.red[1] + 4 - wa0 + 1, wcols = sm.red[3] + 4 - wr0 + 1;
  const bool staged = sm.red[0] <= sm.red[1] && wrows <= A_WROWS && wcols <= A_WCOLS;
  const float2 *sec = a.sec + (size_t)b * P.lines * P.samples;
  if (staged) {
    // deramped window: column walks with the phasor recurrence (drift ~1e-6 rad)
    for (int c = tid; c < wcols; c += A_TX * A_TY) tops_range(P, (double)(wr0 + c), sm.mkt[c], sm.eref[c]);
    __syncthreads();
    const int groups = max(1, (A_TX * A_TY) / wcols);
    const int seg = (wrows + groups - 1) / groups;
    const int g = tid / wcols, c = tid - g * wcols;
    if (g < groups) {
      const int r0 = g * seg, r1 = min(wrows, r0 + seg);
      if (r0 < r1) {
        const double mkt = sm.mkt[c], eref = sm.eref[c];
        const double u = fma((double)(wa0 + r0), P.ati, -P.lines * P.ati / 2.) - eref;
        float2 ph = phasor_pi(mkt * u * u);
        float2 step = phasor_pi(mkt * P.ati * (2.0 * u + P.ati));
        const float2 dstep = phasor_pi(2.0 * mkt * P.ati * P.ati);
        // the segment's samples are loaded first (at most A_SEG rows: wrows <=
        // A_WROWS and at least two groups), so their reads overlap
        const float2 *src = sec + (size_t)(wa0 + r0) * P.samples + (wr0 + c);
        float2 v[A_SEG];
#pragma unroll
        for (int k = 0; k < A_SEG; ++k)
          if (r0 + k < r1) v[k] = __ldg(src + (size_t)k * P.samples);
#pragma unroll
        for (int k = 0; k < A_SEG; ++k) {
          if (r0 + k < r1) {
            sm.win[r0 + k][c] = cmul(v[k], ph);
            ph = cmul(ph, step);
            step = cmul(step, dstep);
          }
        }
      }
    }
    __syncthreads();
  }
  // per pixel: resampled s, its derivatives, the products
#pragma unroll 1
  for (int q = 0; q < A_RPT; ++q) {
    const int lr = ty * A_RPT + q;
    const int row = row0 + lr;
    float2 s = make_float2(0.f, 0.f), sa = s, sr = s;
    float2 rv = make_float2(0.f, 0.f);
    if (in[q]) rv = __ldg(a.ref + boff + (size_t)row * S + col);
    if (ok[q]) {
      float wr[8], wa[8], dwr[8] = {}, dwa[8] = {};
      lut8(g_w, fr[q], wr);
      lut8(g_w, fa[q], wa);
      if (kGrad) {
        lut8(g_dw, fr[q], dwr);
        lut8(g_dw, fa[q], dwa);
      }
      float2 acc = make_float2(0.f, 0.f), acc_a = acc, acc_r = acc;
      const int n0 = na[q] - 3, m0 = nr[q] - 3;
      if (staged) {
        const float2 *base = &sm.win[n0 - wa0][m0 - wr0];
        interp_taps<kGrad>(wr, wa, dwr, dwa, [&](int ka, int kr) { return base[ka * A_WCOLS + kr]; }, acc, acc_a,
                           acc_r);
      } else {
        interp_taps<kGrad>(wr, wa, dwr, dwa, [&](int ka, int kr) { return deramped_tap(P, sec, n0 + ka, m0 + kr); },
                           acc, acc_a, acc_r);
      }
      // reramp with the secondary's TOPS phase at (az, rg): Phi = -pi mkt d^2
      double mkt, eref, dmkt = 0.0, deref = 0.0;
      if (staged) {
        const int c = nr[q] - wr0;
        const double t = fr[q];
        dmkt = sm.mkt[c + 1] - sm.mkt[c];
        deref = sm.eref[c + 1] - sm.eref[c];
        mkt = fma(t, dmkt, sm.mkt[c]);
        eref = fma(t, deref, sm.eref[c]);
      } else {
        double m1, e1;
        tops_range(P, (double)nr[q], mkt, eref);
        tops_range(P, (double)nr[q] + 1.0, m1, e1);
        dmkt = m1 - mkt;
        deref = e1 - eref;
        mkt = fma((double)fr[q], dmkt, mkt);
        eref = fma((double)fr[q], deref, eref);
      }
      const double d = fma(azd[q], P.ati, -P.lines * P.ati / 2.) - eref;
      const float2 rot = phasor_pi(-(mkt * d * d));
      s = cmul(acc, rot);
      if (kGrad) {
        // dPhi/daz = -2 pi mkt d ati; dPhi/drg = pi (2 mkt d deref - dmkt d^2)
        const float pa = (float)(-2.0 * kPiD * mkt * d * P.ati);
        const float pg = (float)(kPiD * (2.0 * mkt * d * deref - dmkt * d * d));
        sa = cmul(make_float2(acc_a.x - pa * acc.y, acc_a.y + pa * acc.x), rot);
        sr = cmul(make_float2(acc_r.x - pg * acc.y, acc_r.y + pg * acc.x), rot);
      }
    }
    sm.r[lr][tx] = rv;
    sm.s[lr][tx] = s;
    if (kGrad) {
      sm.da[lr][tx] = sa;
      sm.dr[lr][tx] = sr;
    }
    // conj(r) s, |r|^2, |s|^2
    sm.pix[lr][tx] = make_float4(rv.x * s.x + rv.y * s.y, rv.x * s.y - rv.y * s.x, rv.x * rv.x + rv.y * rv.y,
                                s.x * s.x + s.y * s.y);
  }
  __syncthreads();
  // window sums in a fixed order: one thread per window of the tile
  const int wpr = a.tile_cols / a.cl, wtile = (A_TH / a.rl) * wpr;
  float gsum = 0.f;
  for (int wi = tid; wi < wtile; wi += A_TX * A_TY) {
    const int wy = wi / wpr, wx = wi - wy * wpr;
    const int gr = tile_y * (A_TH / a.rl) + wy, gc = tile_x * wpr + wx;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gr < nwr && gc < nwc) {
      for (int r = 0; r < a.rl; ++r)
        for (int c = 0; c < a.cl; ++c) {
          const float4 v = sm.pix[wy * a.rl + r][wx * a.cl + c];
          acc.x += v.x;
          acc.y += v.y;
          acc.z += v.z;
          acc.w += v.w;
        }
    }
    const float den = acc.z * acc.w;
    const float i2 = acc.x * acc.x + acc.y * acc.y;
    float gam = 0.f, A = 0.f, B = 0.f;
    if (den > 0.f && i2 > 0.f) {
      gam = sqrtf(i2) * rsqrtf(den);
      A = gam / i2;  // g = (A I) r - B s
      B = gam / acc.w;
    }
    gsum += gam;
    // the window's own first pixel slot: no other window reads it
    sm.pix[wy * a.rl][wx * a.cl] = make_float4(A * acc.x, A * acc.y, B, gam);
  }
  double part[A_PARTS];
#pragma unroll
  for (int k = 0; k < A_PARTS; ++k) part[k] = 0.0;
  part[6] = gsum;
  if (kGrad) {
    __syncthreads();
    // per pixel: g = A r - B s, dJ/daz, dJ/drg, height gradient, parameter sums
    float ga0 = 0.f, ga1 = 0.f, ga2 = 0.f, gr0 = 0.f, gr1 = 0.f, gr2 = 0.f;
#pragma unroll 1
    for (int q = 0; q < A_RPT; ++q) {
      if (!in[q]) continue;
      const int lr = ty * A_RPT + q;
      const int row = row0 + lr;
      const float4 w = sm.pix[(lr / a.rl) * a.rl][(tx / a.cl) * a.cl];
      const float2 rv = sm.r[lr][tx], s = sm.s[lr][tx], sa = sm.da[lr][tx], sr = sm.dr[lr][tx];
      // g = (Ar + i Ai) r - B s
      const float gx = w.x * rv.x - w.y * rv.y - w.z * s.x;
      const float gy = w.x * rv.y + w.y * rv.x - w.z * s.y;
      const float dja = -a.inv_windows * (gx * sa.x + gy * sa.y);  // -Re(conj(g) ds/daz) / windows
      const float djr = -a.inv_windows * (gx * sr.x + gy * sr.y);
      const size_t i = boff + (size_t)row * S + col;
      a.grad_dh[i] = fmaf(dja, __ldg(a.daz_dh + i), djr * __ldg(a.drg_dh + i));
      const float xa = ((float)row - 0.5f * L) / L;
      ga0 += dja;
      ga1 += dja * xa;
      ga2 += dja * xr;
      gr0 += djr;
      gr1 += djr * xa;
      gr2 += djr * xr;
    }
    // pixels outside the multilook grid get a zero height gradient
#pragma unroll
    for (int q = 0; q < A_RPT; ++q) {
      const int row = row0 + ty * A_RPT + q;
      if (!in[q] && tx < a.tile_cols && col < S && row < L) a.grad_dh[boff + (size_t)row * S + col] = 0.f;
    }
    part[0] = ga0;
    part[1] = ga1;
    part[2] = ga2;
    part[3] = gr0;
    part[4] = gr1;
    part[5] = gr2;
  }
  // deterministic block reduction: warps by shuffles, then warp 0
#pragma unroll
  for (int k = 0; k < A_PARTS; ++k) {
    double v = part[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((tid & 31) == 0) sm.part[tid >> 5][k] = v;
  }
  __syncthreads();
  if (tid < A_PARTS) {
    double v = 0.0;
    for (int w = 0; w < A_TX * A_TY / 32; ++w) v += sm.part[w][tid];
    a.partials[((size_t)b * a.tiles_per_burst + tile) * A_PARTS + tid] = v;
  }
}

cudaError_t set_smem_attributes() {
  cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(AdjSmem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(adjoint_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(AdjSmem));
  return e;
}

// Per burst (one block), tiles summed in a fixed order: parameter gradients
// and the burst's sum of gamma (into gam[b]).
__global__ __launch_bounds__(256) void adjoint_reduce_kernel(const double *__restrict__ partials, int tiles,
                                                             double *__restrict__ gam,
                                                             float *__restrict__ grad_params) {
  __shared__ double s[7][256];
  const int b = blockIdx.x, t0 = threadIdx.x;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int t = t0; t < tiles; t += 256) {
    const double *p = partials + ((size_t)b * tiles + t) * A_PARTS;
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] += p[k];
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) s[k][t0] = v[k];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t0 < w)
#pragma unroll
      for (int k = 0; k < 7; ++k) s[k][t0] += s[k][t0 + w];
    __syncthreads();
  }
  if (t0 < 6 && grad_params) grad_params[6 * b + t0] = (float)s[t0][0];
  if (t0 == 6) gam[b] = s[6][0];
}

// Objective J = -(sum over bursts of gamma) / windows, bursts in order.
__global__ void adjoint_objective_kernel(const double *__restrict__ gam, int n_bursts, double inv_windows,
                                         double *__restrict__ objective) {
  double v = 0.0;
  for (int b = 0; b < n_bursts; ++b) v += gam[b];
  objective[0] = -v * inv_windows;
}

}  // namespace

extern "C" int s1b_adjoint_create(const s1b_burst_plan_t *sec_plans, int32_t n_bursts, int32_t lines,
                                  int32_t samples, int32_t rowlook, int32_t collook, s1b_adjoint_t **out) {
  if (!out) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_adjoint_create: null handle");
  *out = nullptr;
  if (!sec_plans || n_bursts < 1 || lines < 1 || samples < 1)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_adjoint_create: no bursts");
  if (rowlook < 1 || A_TH % rowlook != 0)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_adjoint_create: rowlook must divide 16");
  if (collook < 1 || collook > A_TX) return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_adjoint_create: collook above 64");
  if (lines / rowlook < 1 || samples / collook < 1)
    return s1b_fail(S1B_ERR_EMPTY, "s1b_adjoint_create: no multilook window");
  for (int b = 1; b < n_bursts; ++b)
    if (sec_plans[b].lines != sec_plans[0].lines || sec_plans[b].samples != sec_plans[0].samples)
      return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_adjoint_create: secondary bursts must have one size");
  int s = ensure_tables();
  if (s) return s;
  s1b_adjoint *h = new s1b_adjoint();
  cudaGetDevice(&h->device);
  h->n_bursts = n_bursts;
  h->lines = lines;
  h->samples = samples;
  h->rowlook = rowlook;
  h->collook = collook;
  h->tile_cols = (A_TX / collook) * collook;
  h->tiles_x = (samples + h->tile_cols - 1) / h->tile_cols;
  h->tiles_y = (lines + A_TH - 1) / A_TH;
  h->windows = (long long)n_bursts * (lines / rowlook) * (samples / collook);
  cudaError_t e = cudaMalloc(&h->d_plans, n_bursts * sizeof(s1b_burst_plan_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(h->d_plans, sec_plans, n_bursts * sizeof(s1b_burst_plan_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(h->d_plans);
    delete h;
    return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = h;
  return S1B_OK;
}

extern "C" void s1b_adjoint_destroy(s1b_adjoint_t *h) {
  if (!h) return;
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != h->device) cudaSetDevice(h->device);
  cudaFree(h->d_plans);
  if (prev >= 0 && prev != h->device) cudaSetDevice(prev);
  delete h;
}

extern "C" size_t s1b_adjoint_workspace_bytes(const s1b_adjoint_t *h) {
  if (!h) return 0;
  return ((size_t)h->n_bursts * h->tiles_x * h->tiles_y * A_PARTS + h->n_bursts) * sizeof(double);
}

extern "C" int s1b_adjoint_run(s1b_adjoint_t *h, const void *ref, const void *sec, const float *az0,
                               const float *rg0, const float *daz_dh, const float *drg_dh, const float *params,
                               const float *dh, double *objective, float *grad_params, float *grad_dh,
                               void *workspace, size_t workspace_bytes, void *stream) {
  if (!h || !ref || !sec || !az0 || !rg0 || !daz_dh || !drg_dh || !params || !dh || !objective || !workspace)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_adjoint_run: null argument");
  const bool grad = grad_params || grad_dh;
  if (grad && (!grad_params || !grad_dh))
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_adjoint_run: give both gradient outputs or neither");
  if (workspace_bytes < s1b_adjoint_workspace_bytes(h))
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_adjoint_run: workspace too small");
  const int tiles = h->tiles_x * h->tiles_y;
  if (h->n_bursts > 65535 || tiles < 1) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_adjoint_run: grid too large");
  cudaStream_t st = (cudaStream_t)stream;
  int s0 = ensure_tables();  // this device's tables and shared-memory limits
  if (s0) return s0;
  AdjArgs a;
  a.plans = h->d_plans;
  a.ref = (const float2 *)ref;
  a.sec = (const float2 *)sec;
  a.az0 = az0;
  a.rg0 = rg0;
  a.daz_dh = daz_dh;
  a.drg_dh = drg_dh;
  a.params = params;
  a.dh = dh;
  a.grad_dh = grad_dh;
  a.partials = (double *)workspace;
  a.L = h->lines;
  a.S = h->samples;
  a.rl = h->rowlook;
  a.cl = h->collook;
  a.tile_cols = h->tile_cols;
  a.tiles_x = h->tiles_x;
  a.tiles_per_burst = tiles;
  a.inv_windows = (float)(1.0 / (double)h->windows);
  dim3 grid(tiles, h->n_bursts);
  dim3 block(A_TX, A_TY);
  if (grad)
    adjoint_kernel<true><<<grid, block, sizeof(AdjSmem), st>>>(a);
  else
    adjoint_kernel<false><<<grid, block, sizeof(AdjSmem), st>>>(a);
  int s = s1b_launch_status();
  if (s) return s;
  double *gam = (double *)workspace + (size_t)h->n_bursts * tiles * A_PARTS;
  adjoint_reduce_kernel<<<h->n_bursts, 256, 0, st>>>((const double *)workspace, tiles, gam,
                                                     grad ? grad_params : nullptr);
  s = s1b_launch_status();
  if (s) return s;
  adjoint_objective_kernel<<<1, 1, 0, st>>>(gam, h->n_bursts, 1.0 / (double)h->windows, objective);
  return s1b_launch_status();
}

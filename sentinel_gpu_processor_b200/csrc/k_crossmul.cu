// Crossmul + multilook + power looks + coherence in one pass on sm_100a.
//
// Replaces, for one burst pair, the reference's three kernels conj_mul,
// cpx_col_look and cpx_row_look (csrc/src/sario.cu:199-286, launched at
// crossmul_daemon.cu:921-975), point_angle (sario.cu:231-239) and the NumPy
// amplitude multilook and coherence (s1proc/coherence.py:14-147,
// s1proc/sario.py:397-420).  Both SLCs are read once; nothing full-size is
// written.
//
// CTA = 256 threads = one multilooked row x M multilooked columns
// (M * collook <= 512 full-resolution columns, more for very wide looks).
// Threads read rows with coalesced 8-byte loads, sum the `rowlook` rows in
// registers, stage per-column sums in shared memory, and M threads finish
// the `collook` sums and the epilogue.
#include <cuda_runtime.h>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_frame.h"
#include "s1b_internal.h"

namespace {

constexpr int XM_THREADS = 256;
constexpr int XM_MAX_COLLOOK = 4096;

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  // SplitMix64 (Steele, Lea, Flood, OOPSLA 2014)
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform [0, 1) fill for coherence values > 1 (the reference draws these
// from an unseeded np.random.rand, s1proc/coherence.py:143-144).
__device__ __forceinline__ float fill_uniform(uint64_t seed, uint64_t index) {
  return (float)(splitmix64((seed << 32) + index) >> 40) * (1.0f / 16777216.0f);
}

struct XmArgs {
  const float2 *ref;
  const float2 *sec;
  int64_t ref_off;  // element offset of global pixel (top, left) in ref
  int64_t sec_off;
  int32_t ref_width, sec_width;
  int32_t nrow_ml, ncol_ml, rowlook, collook, m_per_cta;
  float2 *ifg;
  float *amp1, *amp2, *coh, *phase;
  uint64_t seed;
};

// Multilooked pixel o from its sums over the look window: mean over collook,
// then over rowlook, like cpx_col_look / cpx_row_look; amplitudes; coherence
// with the seeded fill; phase.
__device__ __forceinline__ void xm_finish(float ir, float ii, float p1, float p2, int rowlook, int collook, int64_t o,
                                          float2 *ifg, float *amp1, float *amp2, float *coh, float *phase,
                                          uint64_t seed) {
  const float fcl = (float)collook, frl = (float)rowlook;
  ir = ir / fcl / frl;
  ii = ii / fcl / frl;
  // s1proc's powlooks returns |s| rather than |s|^2 when both looks are 1
  // (s1proc/sario.py:416-418), so its amplitude is then sqrt(|s|); kept so
  // that .amp and coherence values match the reference's.
  const bool unit = (rowlook == 1 && collook == 1);
  const float am1 = unit ? sqrtf(sqrtf(p1)) : sqrtf(p1 / fcl / frl);
  const float am2 = unit ? sqrtf(sqrtf(p2)) : sqrtf(p2 / fcl / frl);
  if (ifg) ifg[o] = make_float2(ir, ii);
  if (amp1) amp1[o] = am1;
  if (amp2) amp2[o] = am2;
  if (coh) {
    // s1proc/coherence.py:142-144
    float c = hypotf(ir, ii) / (am1 + 1e-12f) / (am2 + 1e-12f);
    if (c > 1.f) c = fill_uniform(seed, (uint64_t)o);
    coh[o] = c;
  }
  if (phase) phase[o] = atan2f(ii, ir);
}

// One CTA: multilooked row i, columns [chunk * m_per_cta, ...).
__device__ __forceinline__ void crossmul_tile(const XmArgs &a, int i, int chunk, float4 *smem4) {
  const int W = a.m_per_cta * a.collook;  // full-res columns of this CTA
  float2 *sI = reinterpret_cast<float2 *>(smem4);
  float2 *sP = sI + W;  // (|ref|^2, |sec|^2) per column
  const int j0 = chunk * a.m_per_cta;
  const int mcta = min(a.m_per_cta, a.ncol_ml - j0);
  const int wcta = mcta * a.collook;
  const int64_t col0 = (int64_t)j0 * a.collook;
  const int64_t row0 = (int64_t)i * a.rowlook;
  // Each thread owns columns c and c + 256 of the chunk (when present) and
  // issues the loads of four rows of both SLCs for both columns before it
  // accumulates, so 16 independent 8-byte loads are in flight per thread.
  for (int c = threadIdx.x; c < wcta; c += 2 * XM_THREADS) {
    const bool two = c + XM_THREADS < wcta;
    const int cc = two ? c + XM_THREADS : c;
    float ir[2] = {0.f, 0.f}, ii[2] = {0.f, 0.f}, p1[2] = {0.f, 0.f}, p2[2] = {0.f, 0.f};
    const float2 *pr = a.ref + a.ref_off + row0 * a.ref_width + col0;
    const float2 *ps = a.sec + a.sec_off + row0 * a.sec_width + col0;
    int k = 0;
    for (; k + 4 <= a.rowlook; k += 4) {
      float2 r[4][2], s[4][2];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        r[u][0] = __ldg(pr + (int64_t)(k + u) * a.ref_width + c);
        r[u][1] = __ldg(pr + (int64_t)(k + u) * a.ref_width + cc);
        s[u][0] = __ldg(ps + (int64_t)(k + u) * a.sec_width + c);
        s[u][1] = __ldg(ps + (int64_t)(k + u) * a.sec_width + cc);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
#pragma unroll
        for (int q = 0; q < 2; ++q) xm_accumulate(r[u][q], s[u][q], ir[q], ii[q], p1[q], p2[q]);
      }
    }
    for (; k < a.rowlook; ++k) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int col = q ? cc : c;
        xm_accumulate(__ldg(pr + (int64_t)k * a.ref_width + col), __ldg(ps + (int64_t)k * a.sec_width + col), ir[q],
                      ii[q], p1[q], p2[q]);
      }
    }
    sI[c] = make_float2(ir[0], ii[0]);
    sP[c] = make_float2(p1[0], p2[0]);
    if (two) {
      sI[cc] = make_float2(ir[1], ii[1]);
      sP[cc] = make_float2(p1[1], p2[1]);
    }
  }
  __syncthreads();
  for (int m = threadIdx.x; m < mcta; m += XM_THREADS) {
    float ir = 0.f, ii = 0.f, p1 = 0.f, p2 = 0.f;
    const int base = m * a.collook;
    for (int u = 0; u < a.collook; ++u) {
      const float2 v = sI[base + u];
      const float2 p = sP[base + u];
      ir += v.x;
      ii += v.y;
      p1 += p.x;
      p2 += p.y;
    }
    xm_finish(ir, ii, p1, p2, a.rowlook, a.collook, (int64_t)i * a.ncol_ml + j0 + m, a.ifg, a.amp1, a.amp2, a.coh,
              a.phase, a.seed);
  }
}

// Frame form of crossmul_tile: one CTA walks XM_ROWS multilooked rows of a
// column chunk (frames give grids of hundreds of thousands of row chunks).
// Per row every thread sums the `rowlook` rows of its columns into a float4
// (conj product re, im, both powers) in one of two shared-memory buffers;
// after a barrier one warp (a different one each row, so the others go on
// loading the next row) or, for chunks of more than 32 outputs, the whole CTA
// forms the `collook` sums and the epilogue, with the same operations in the
// same order as crossmul_tile.  The buffer a row's epilogue reads is
// rewritten only after the next row's barrier, which that warp reaches once
// its epilogue is done.  (On single pairs, grids of a few thousand CTAs,
// this form measured slower than crossmul_tile, so they keep that one.)
constexpr int XM_ROWS = 4;

__device__ __forceinline__ void crossmul_rows_tile(const XmArgs &a, int i0, int chunk, float4 *smem4) {
  const int W = a.m_per_cta * a.collook;
  const int j0 = chunk * a.m_per_cta;
  const int mcta = min(a.m_per_cta, a.ncol_ml - j0);
  const int wcta = mcta * a.collook;
  const int64_t col0 = (int64_t)j0 * a.collook;
  const int i1 = min(i0 + XM_ROWS, a.nrow_ml);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = i0; i < i1; ++i) {
    float4 *buf = smem4 + ((i - i0) & 1) * W;
    const int64_t row0 = (int64_t)i * a.rowlook;
    for (int c = threadIdx.x; c < wcta; c += 2 * XM_THREADS) {
      const bool two = c + XM_THREADS < wcta;
      const int cc = two ? c + XM_THREADS : c;
      float ir[2] = {0.f, 0.f}, ii[2] = {0.f, 0.f}, p1[2] = {0.f, 0.f}, p2[2] = {0.f, 0.f};
      const float2 *pr = a.ref + a.ref_off + row0 * a.ref_width + col0;
      const float2 *ps = a.sec + a.sec_off + row0 * a.sec_width + col0;
      int k = 0;
      for (; k + 4 <= a.rowlook; k += 4) {
        float2 r[4][2], s[4][2];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          r[u][0] = __ldg(pr + (int64_t)(k + u) * a.ref_width + c);
          r[u][1] = __ldg(pr + (int64_t)(k + u) * a.ref_width + cc);
          s[u][0] = __ldg(ps + (int64_t)(k + u) * a.sec_width + c);
          s[u][1] = __ldg(ps + (int64_t)(k + u) * a.sec_width + cc);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
          for (int q = 0; q < 2; ++q) xm_accumulate(r[u][q], s[u][q], ir[q], ii[q], p1[q], p2[q]);
        }
      }
      for (; k < a.rowlook; ++k) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int col = q ? cc : c;
          xm_accumulate(__ldg(pr + (int64_t)k * a.ref_width + col), __ldg(ps + (int64_t)k * a.sec_width + col),
                        ir[q], ii[q], p1[q], p2[q]);
        }
      }
      buf[c] = make_float4(ir[0], ii[0], p1[0], p2[0]);
      if (two) buf[cc] = make_float4(ir[1], ii[1], p1[1], p2[1]);
    }
    __syncthreads();
    const bool one = mcta <= 32;
    if (one && warp != (i - i0) % (XM_THREADS / 32)) continue;
    for (int m = one ? lane : threadIdx.x; m < mcta; m += one ? 32 : XM_THREADS) {
      float ir = 0.f, ii = 0.f, p1 = 0.f, p2 = 0.f;
      const float4 *b = buf + m * a.collook;
#pragma unroll 4
      for (int u = 0; u < a.collook; ++u) {
        const float4 v = b[u];
        ir += v.x;
        ii += v.y;
        p1 += v.z;
        p2 += v.w;
      }
      xm_finish(ir, ii, p1, p2, a.rowlook, a.collook, (int64_t)i * a.ncol_ml + j0 + m, a.ifg, a.amp1, a.amp2,
                a.coh, a.phase, a.seed);
    }
  }
}

__global__ __launch_bounds__(XM_THREADS) void crossmul_looks_kernel(const XmArgs a) {
  extern __shared__ float4 smem4[];
  crossmul_tile(a, blockIdx.x, blockIdx.y, smem4);
}

// ----------------------------------------------- amplitude and coherence files
// Amplitude looks of one cropped SLC into a full-frame amplitude grid
// (s1proc/coherence.py:14-55): the crop's look-aligned part, sqrt of the
// mean power over rl x cl (|s| when both looks are 1, powlooks,
// s1proc/sario.py:416-420, so sqrt|s|), written where this is the first
// image of the date or the grid is still 0 and the new value is not.
__global__ void amp_looks_kernel(const float2 *__restrict__ slc, int width, int left, int top, int left_sm,
                                 int top_sm, int nrow_sm_crop, int ncol_sm_crop, int ncol0_sm, int rowlook,
                                 int collook, int first, float *__restrict__ amp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
  if (j >= ncol_sm_crop) return;
  const int r0 = (top_sm + i) * rowlook - top, c0 = (left_sm + j) * collook - left;
  float p = 0.f;
  for (int r = 0; r < rowlook; ++r)
    for (int c = 0; c < collook; ++c) {
      const float2 v = __ldg(slc + (int64_t)(r0 + r) * width + c0 + c);
      p += v.x * v.x + v.y * v.y;
    }
  const float a = (rowlook == 1 && collook == 1) ? sqrtf(sqrtf(p)) : sqrtf(p / (float)collook / (float)rowlook);
  float *dst = amp + (int64_t)(top_sm + i) * ncol0_sm + left_sm + j;
  if (first || (*dst == 0.f && a != 0.f)) *dst = a;
}

// .cc rows [amp1 amp2 | coherence] (s1proc/coherence.py:136-147, sario.py:387-394):
// coherence |ifg| / (amp1 + 1e-12) / (amp2 + 1e-12), values above 1 replaced
// by a uniform [0, 1) value of (seed, pixel index).
__global__ void coherence_cc_kernel(const float2 *__restrict__ ifg, const float *__restrict__ amp1,
                                    const float *__restrict__ amp2, int nrow, int ncol, uint64_t seed,
                                    float *__restrict__ cc) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
  if (j >= ncol) return;
  const int64_t o = (int64_t)i * ncol + j;
  const float2 v = ifg[o];
  const float a1 = amp1[o], a2 = amp2[o];
  float c = hypotf(v.x, v.y) / (a1 + 1e-12f) / (a2 + 1e-12f);
  if (c > 1.f) c = fill_uniform(seed, (uint64_t)o);
  cc[(int64_t)i * 2 * ncol + j] = a1 * a2;
  cc[(int64_t)i * 2 * ncol + ncol + j] = c;
}

// ------------------------------------------------------------ frame stages
// Per pair, from the crop rows the geocoding stage voted: the two .gslc
// headers (geo2rdr.cu:641-647), the overlap box aligned to the looks and the
// interferogram header (crossmul_daemon.cu:612-666), and the multilooked size.
__global__ void frame_box_kernel(const FrameDev d, s1b_frame_pair_t *pout) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.n_pairs) return;
  const FramePair pr = d.pairs[k];
  const s1b_burst_plan_t &p1 = d.plans[pr.ref], &p2 = d.plans[pr.sec];
  s1b_frame_pair_t r;
  r.ok = 0;
  r.nrow_ml = r.ncol_ml = r.filtered = 0;
  for (int q = 0; q < 6; ++q) r.header[q] = 0;
  for (int q = 0; q < 4; ++q) r.box[q] = 0;
  const int f1 = d.rows[2 * pr.ref], l1 = d.rows[2 * pr.ref + 1];
  const int f2 = d.rows[2 * pr.sec], l2 = d.rows[2 * pr.sec + 1];
  r.gslc_rows[0] = f1;
  r.gslc_rows[1] = l1;
  r.gslc_rows[2] = f2;
  r.gslc_rows[3] = l2;
  const bool rows_ok = f1 < d.bursts[pr.ref].nrow && l1 > f1 && f2 < d.bursts[pr.sec].nrow && l2 > f2;
  if (rows_ok) {
    // header words [nrow0, ncol0, left, top, right, bottom] of both .gslc
    const int top1 = p1.win_top + f1, bot1 = p1.win_top + l1;
    const int top2 = p2.win_top + f2, bot2 = p2.win_top + l2;
    int left = max(p1.win_left, p2.win_left), right = min(p1.win_right, p2.win_right);
    int top = max(top1, top2), bottom = min(bot1, bot2);
    left = (left + d.collook - 1) / d.collook * d.collook;
    right = right / d.collook * d.collook;
    top = (top + d.rowlook - 1) / d.rowlook * d.rowlook;
    bottom = bottom / d.rowlook * d.rowlook;
    if (bottom - top > 0 && right - left > 0) {
      r.ok = 1;
      r.box[0] = left;
      r.box[1] = top;
      r.box[2] = right;
      r.box[3] = bottom;
      r.header[0] = p1.rsc_nlat / d.rowlook;
      r.header[1] = p1.rsc_nlon / d.collook;
      r.header[2] = left / d.collook;
      r.header[3] = top / d.rowlook;
      r.header[4] = right / d.collook;
      r.header[5] = bottom / d.rowlook;
      r.nrow_ml = min((bottom - top) / d.rowlook, pr.max_nrow_ml);
      r.ncol_ml = min((right - left) / d.collook, pr.max_ncol_ml);
      r.filtered = r.nrow_ml >= d.n_win && r.ncol_ml >= d.n_win;
    }
  }
  pout[k] = r;
}

// Crossmul + looks of every pair: blockIdx.z = pair, x = group of XM_ROWS
// multilooked rows, y = column chunk; CTAs outside a pair's box return at once.
// Compiled for 4 CTAs per SM (64 registers): left to itself the compiler
// picks 48 registers and spills.
__global__ __launch_bounds__(XM_THREADS, 4) void frame_crossmul_kernel(const FrameDev d, const FrameIO io,
                                                                   int m_per_cta) {
  extern __shared__ float4 smem4[];
  const int k = blockIdx.z;
  const s1b_frame_pair_t &r = io.pout[k];
  if (!r.ok || (int)blockIdx.x * XM_ROWS >= r.nrow_ml || (int)blockIdx.y * m_per_cta >= r.ncol_ml) return;
  const FramePair pr = d.pairs[k];
  const s1b_burst_plan_t &p1 = d.plans[pr.ref], &p2 = d.plans[pr.sec];
  const FrameBurst &b1 = d.bursts[pr.ref], &b2 = d.bursts[pr.sec];
  XmArgs a;
  a.ref = io.work + b1.geo_off;
  a.sec = io.work + b2.geo_off;
  a.ref_off = (int64_t)(r.box[1] - p1.win_top) * b1.ncol + (r.box[0] - p1.win_left);
  a.sec_off = (int64_t)(r.box[1] - p2.win_top) * b2.ncol + (r.box[0] - p2.win_left);
  a.ref_width = b1.ncol;
  a.sec_width = b2.ncol;
  a.nrow_ml = r.nrow_ml;
  a.ncol_ml = r.ncol_ml;
  a.rowlook = d.rowlook;
  a.collook = d.collook;
  a.m_per_cta = m_per_cta;
  a.ifg = io.ifg + pr.ml_off;
  a.amp1 = io.amp1 ? io.amp1 + pr.ml_off : nullptr;
  a.amp2 = io.amp2 ? io.amp2 + pr.ml_off : nullptr;
  a.coh = io.coh ? io.coh + pr.ml_off : nullptr;
  a.phase = nullptr;
  a.seed = d.fill_seed;
  crossmul_rows_tile(a, blockIdx.x * XM_ROWS, blockIdx.y, smem4);
}

// Crossmul fused into the geocoding: the geocoding kernel left, per pair,
// the rowlook-row sums of every column of the pair's windows (one float4 per
// column and look row: conj product re, im, both powers, summed like
// crossmul_rows_tile sums them).  Each warp here takes 32 multilooked pixels
// of a row of the box: it stages their contiguous span of column sums in
// shared memory with coalesced loads, then each lane adds the collook
// columns of its pixel in order and forms the outputs.
// blockIdx.z = pair, y = multilooked row, x = groups of 128 multilooked columns.
constexpr int XC_SPAN = 704;  // float4 per warp buffer (11 KB)

__global__ __launch_bounds__(128) void frame_xm_cells_kernel(const FrameDev d, const FrameIO io) {
  __shared__ float4 buf[4][XC_SPAN];
  const int k = blockIdx.z, i = blockIdx.y, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const s1b_frame_pair_t &r = io.pout[k];
  const int jw = blockIdx.x * 128 + w * 32;  // the warp's first multilooked column
  if (!r.ok || i >= r.nrow_ml || jw >= r.ncol_ml) return;  // warp-uniform
  const FramePair pr = d.pairs[k];
  const int cl = d.collook;
  const float4 *row = reinterpret_cast<const float4 *>(io.work + pr.part_off) +
                      (int64_t)((r.box[1] - pr.part_top) / d.rowlook + i) * pr.part_cols + (r.box[0] - pr.part_left);
  float2 *ifg = io.ifg + pr.ml_off;
  float *amp1 = io.amp1 ? io.amp1 + pr.ml_off : nullptr, *amp2 = io.amp2 ? io.amp2 + pr.ml_off : nullptr;
  float *coh = io.coh ? io.coh + pr.ml_off : nullptr;
  if ((cl | 1) > XC_SPAN) {  // very wide looks: each lane reads its own columns
    const int j = jw + lane;
    if (j >= r.ncol_ml) return;
    float ir = 0.f, ii = 0.f, p1 = 0.f, p2 = 0.f;
    for (int u = 0; u < cl; ++u) {
      const float4 v = __ldcs(row + (int64_t)j * cl + u);
      ir += v.x;
      ii += v.y;
      p1 += v.z;
      p2 += v.w;
    }
    xm_finish(ir, ii, p1, p2, d.rowlook, cl, (int64_t)i * r.ncol_ml + j, ifg, amp1, amp2, coh, nullptr, d.fill_seed);
    return;
  }
  // each pixel's columns at an odd stride in float4 (cl | 1): the lanes'
  // 16-byte reads of column u then fall in distinct banks
  const int cs = cl | 1;
  const int per = min(32, XC_SPAN / cs);  // pixels per pass
  for (int m0 = 0; m0 < 32; m0 += per) {
    const int j0 = jw + m0, n = min(min(per, 32 - m0), r.ncol_ml - j0);
    if (n <= 0) break;
    const float4 *src = row + (int64_t)j0 * cl;
    __syncwarp();  // the previous pass is done with the buffer
    for (int e = lane; e < n * cl; e += 32) {
      const int m = e / cl;
      buf[w][e + m * (cs - cl)] = __ldcs(src + e);
    }
    __syncwarp();
    if (lane < n) {
      float ir = 0.f, ii = 0.f, p1 = 0.f, p2 = 0.f;
      const float4 *b = buf[w] + lane * cs;
      for (int u = 0; u < cl; ++u) {
        const float4 v = b[u];
        ir += v.x;
        ii += v.y;
        p1 += v.z;
        p2 += v.w;
      }
      xm_finish(ir, ii, p1, p2, d.rowlook, cl, (int64_t)i * r.ncol_ml + j0 + lane, ifg, amp1, amp2, coh, nullptr,
                d.fill_seed);
    }
  }
}

}  // namespace

extern "C" int s1b_crossmul_looks(const void *ref, int32_t ref_left, int32_t ref_top,
                                  int32_t ref_width, int32_t ref_height, const void *sec,
                                  int32_t sec_left, int32_t sec_top, int32_t sec_width,
                                  int32_t sec_height, int32_t left, int32_t top,
                                  int32_t nrow_ml, int32_t ncol_ml, int32_t rowlook,
                                  int32_t collook, void *ifg, float *amp1, float *amp2,
                                  float *coh, float *phase, uint64_t fill_seed, void *stream) {
  if (!ref || !sec) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_crossmul_looks: null input");
  if (rowlook < 1 || collook < 1 || nrow_ml < 0 || ncol_ml < 0)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_crossmul_looks: bad looks or size");
  if (collook > XM_MAX_COLLOOK)
    return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_crossmul_looks: collook above 4096");
  if (left < ref_left || left < sec_left || top < ref_top || top < sec_top)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_crossmul_looks: box outside the rasters");
  if ((int64_t)left + (int64_t)ncol_ml * collook > (int64_t)ref_left + ref_width ||
      (int64_t)left + (int64_t)ncol_ml * collook > (int64_t)sec_left + sec_width)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_crossmul_looks: box wider than the rasters");
  if ((int64_t)top + (int64_t)nrow_ml * rowlook > (int64_t)ref_top + ref_height ||
      (int64_t)top + (int64_t)nrow_ml * rowlook > (int64_t)sec_top + sec_height)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_crossmul_looks: box taller than the rasters");
  if (nrow_ml == 0 || ncol_ml == 0) return S1B_OK;
  XmArgs a;
  a.ref = (const float2 *)ref;
  a.sec = (const float2 *)sec;
  a.ref_off = (int64_t)(top - ref_top) * ref_width + (left - ref_left);
  a.sec_off = (int64_t)(top - sec_top) * sec_width + (left - sec_left);
  a.ref_width = ref_width;
  a.sec_width = sec_width;
  a.nrow_ml = nrow_ml;
  a.ncol_ml = ncol_ml;
  a.rowlook = rowlook;
  a.collook = collook;
  a.m_per_cta = collook >= 512 ? 1 : 512 / collook;
  a.ifg = (float2 *)ifg;
  a.amp1 = amp1;
  a.amp2 = amp2;
  a.coh = coh;
  a.phase = phase;
  a.seed = fill_seed;
  const size_t smem = (size_t)a.m_per_cta * collook * 2 * sizeof(float2);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(crossmul_looks_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  }
  const int nchunk = (ncol_ml + a.m_per_cta - 1) / a.m_per_cta;
  if (nchunk > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_crossmul_looks: too many columns");
  dim3 grid(nrow_ml, nchunk);
  crossmul_looks_kernel<<<grid, XM_THREADS, smem, (cudaStream_t)stream>>>(a);
  return s1b_launch_status();
}

extern "C" int s1b_amp_looks(const void *slc, int32_t width, int32_t height, int32_t left, int32_t top,
                             int32_t nrow0, int32_t ncol0, int32_t rowlook, int32_t collook, int32_t first,
                             float *amp, void *stream) {
  if (!slc || !amp) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_amp_looks: null argument");
  if (rowlook < 1 || collook < 1 || width < 0 || height < 0 || left < 0 || top < 0)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_amp_looks: bad looks or crop");
  const int left_sm = (left + collook - 1) / collook, top_sm = (top + rowlook - 1) / rowlook;
  const int right_sm = (left + width) / collook, bottom_sm = (top + height) / rowlook;
  const int ncol0_sm = ncol0 / collook, nrow0_sm = nrow0 / rowlook;
  if (right_sm > ncol0_sm || bottom_sm > nrow0_sm)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_amp_looks: crop outside the frame");
  const int nr = bottom_sm - top_sm, nc = right_sm - left_sm;
  if (nr <= 0 || nc <= 0) return S1B_OK;
  if (nr > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_amp_looks: too many rows");
  dim3 grid((nc + 255) / 256, nr);
  amp_looks_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((const float2 *)slc, width, left, top, left_sm, top_sm,
                                                           nr, nc, ncol0_sm, rowlook, collook, first ? 1 : 0, amp);
  return s1b_launch_status();
}

extern "C" int s1b_coherence_cc(const void *ifg, const float *amp1, const float *amp2, int32_t nrow, int32_t ncol,
                                uint64_t fill_seed, float *cc, void *stream) {
  if (!ifg || !amp1 || !amp2 || !cc) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_coherence_cc: null argument");
  if (nrow < 0 || ncol < 0) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_coherence_cc: negative size");
  if (nrow == 0 || ncol == 0) return S1B_OK;
  if (nrow > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_coherence_cc: too many rows");
  dim3 grid((ncol + 255) / 256, nrow);
  coherence_cc_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((const float2 *)ifg, amp1, amp2, nrow, ncol, fill_seed,
                                                              cc);
  return s1b_launch_status();
}

int frame_launch_box(const FrameDev &d, const FrameIO &io, cudaStream_t st) {
  frame_box_kernel<<<(d.n_pairs + 127) / 128, 128, 0, st>>>(d, io.pout);
  return s1b_launch_status();
}

int frame_launch_crossmul(const FrameDev &d, const FrameIO &io, cudaStream_t st) {
  if (d.collook > XM_MAX_COLLOOK) return s1b_fail(S1B_ERR_TOO_LARGE, "frame crossmul: collook above 4096");
  if (d.max_nrow_ml <= 0 || d.max_ncol_ml <= 0) return S1B_OK;
  if (d.fused_xmul) {  // the geocoding left the look-row sums: add the look columns
    if (d.max_nrow_ml > 65535 || d.n_pairs > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "frame crossmul: grid too large");
    frame_xm_cells_kernel<<<dim3((d.max_ncol_ml + 127) / 128, d.max_nrow_ml, d.n_pairs), 128, 0, st>>>(d, io);
    return s1b_launch_status();
  }
  const int m_per_cta = d.collook >= 512 ? 1 : 512 / d.collook;
  const size_t smem = (size_t)m_per_cta * d.collook * 2 * sizeof(float4);  // two buffers of float4
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(frame_crossmul_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  }
  const int nchunk = (d.max_ncol_ml + m_per_cta - 1) / m_per_cta;
  if (nchunk > 65535 || d.n_pairs > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "frame crossmul: grid too large");
  dim3 grid((d.max_nrow_ml + XM_ROWS - 1) / XM_ROWS, nchunk, d.n_pairs);
  frame_crossmul_kernel<<<grid, XM_THREADS, smem, st>>>(d, io, m_per_cta);
  return s1b_launch_status();
}

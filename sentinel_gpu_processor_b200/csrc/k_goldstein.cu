// Goldstein phase filter on sm_100a.
//
// Replaces goldstein_filter_cuda_host and its kernels (extract_patches,
// cuFFT forward, gaussian_filter, patchwise_normalize, spectrum_enhancement,
// cuFFT inverse, batched_overlap_add, normalize_output), reference
// csrc/src/goldstein.cu:87-408, with two kernels:
//   1. goldstein_patch_kernel -- one warp per 32x32 patch: coalesced patch
//      load into shared memory, 2-D FFT as 32-point radix-2 FFTs held in
//      registers (rows, then columns through a padded shared tile), |F|,
//      7x7 circular smoothing, patch-mean normalisation, S^alpha weighting,
//      inverse 2-D FFT, triangular weight and 1/n^2 scale; the weighted patch
//      is written to scratch.
//   2. goldstein_gather_kernel -- one thread per output pixel sums the (up to
//      16) weighted patches covering it in a fixed order and divides by the
//      summed weights.  No atomics: the result is deterministic.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "s1b.h"
#include "s1b_ctx_cache.h"
#include "s1b_device.cuh"
#include "s1b_frame.h"
#include "s1b_internal.h"

namespace {

constexpr int GN = 32;        // patch size (s1proc filter.window_size)
constexpr int GSTEP = GN / 4; // patch step, goldstein.cu:334
constexpr int GWARPS = 4;     // patches per CTA
// CTAs per SM the patch kernels are compiled for: 128 registers per thread,
// the FFT's 32 complex values in registers with a small spill (measured
// 1.14 ms per 27-pair frame against 1.41 ms at 168 registers and 3 CTAs/SM)
constexpr int GCTAS_PER_SM = 4;

// exp(2 pi i k / 32), k = 0..15, from cos/sin of 2 pi k / 32 evaluated in
// 50-digit decimal arithmetic.
__constant__ float2 c_tw[16] = {
    {1.0f, 0.0f},
    {0.9807852804032304f, 0.19509032201612828f},
    {0.9238795325112867f, 0.3826834323650898f},
    {0.8314696123025452f, 0.5555702330196022f},
    {0.7071067811865476f, 0.7071067811865476f},
    {0.5555702330196022f, 0.8314696123025452f},
    {0.3826834323650898f, 0.9238795325112867f},
    {0.19509032201612828f, 0.9807852804032304f},
    {0.0f, 1.0f},
    {-0.19509032201612828f, 0.9807852804032304f},
    {-0.3826834323650898f, 0.9238795325112867f},
    {-0.5555702330196022f, 0.8314696123025452f},
    {-0.7071067811865476f, 0.7071067811865476f},
    {-0.8314696123025452f, 0.5555702330196022f},
    {-0.9238795325112867f, 0.3826834323650898f},
    {-0.9807852804032304f, 0.19509032201612828f},
};

// The reference project's 7x7 smoothing table, goldstein.cu:43-52 (row
// ky = -3..3, column kx = -3..3).  Kept as given: the filter output depends
// on these exact values.
__constant__ float c_gauss[49] = {
    0.000004f, 0.000088f, 0.000543f, 0.000948f, 0.000543f, 0.000088f, 0.000004f,
    0.000088f, 0.001915f, 0.011776f, 0.020584f, 0.011776f, 0.001915f, 0.000088f,
    0.000543f, 0.011776f, 0.072410f, 0.126584f, 0.072410f, 0.011776f, 0.000543f,
    0.000948f, 0.020584f, 0.126584f, 0.221141f, 0.126584f, 0.020584f, 0.000948f,
    0.000543f, 0.011776f, 0.072410f, 0.126584f, 0.072410f, 0.011776f, 0.000543f,
    0.000088f, 0.001915f, 0.011776f, 0.020584f, 0.011776f, 0.001915f, 0.000088f,
    0.000004f, 0.000088f, 0.000543f, 0.000948f, 0.000543f, 0.000088f, 0.000004f};

__host__ __device__ constexpr int brev5(int i) {
  return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// One radix-2 stage (butterfly span m = 2^S) of the 32-point FFT; a template
// per stage so that every index is a compile-time constant and x stays in
// registers.  The twiddles 1 and -+i are applied as copies and swaps: the
// same values the multiplication gives for finite samples, without its
// multiplies (46 of the 80 butterflies of a transform).
template <int S, bool kInverse>
__device__ __forceinline__ void fft32_stage(float2 (&x)[GN]) {
  constexpr int m = 1 << S, half = m >> 1, stride = GN / m;
#pragma unroll
  for (int k = 0; k < GN; k += m) {
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const int tw = j * stride;
      const float2 b = x[k + j + half];
      float2 t;
      if (tw == 0) {
        t = b;
      } else if (tw == GN / 4) {  // exp(-+i pi / 2)
        t = kInverse ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
      } else {
        float2 w = c_tw[tw];
        if (!kInverse) w.y = -w.y;
        t = make_float2(w.x * b.x - w.y * b.y, w.x * b.y + w.y * b.x);
      }
      const float2 u = x[k + j];
      x[k + j] = make_float2(u.x + t.x, u.y + t.y);
      x[k + j + half] = make_float2(u.x - t.x, u.y - t.y);
    }
  }
}

// In-place 32-point DFT of x (natural order in and out), radix-2
// decimation in time.  Forward: exp(-2 pi i jk/32); inverse: exp(+...),
// unnormalised (cuFFT's convention).
template <bool kInverse>
__device__ __forceinline__ void fft32(float2 (&x)[GN]) {
#pragma unroll
  for (int i = 0; i < GN; ++i) {
    const int j = brev5(i);
    if (j > i) {
      const float2 t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  fft32_stage<1, kInverse>(x);
  fft32_stage<2, kInverse>(x);
  fft32_stage<3, kInverse>(x);
  fft32_stage<4, kInverse>(x);
  fft32_stage<5, kInverse>(x);
}

__device__ __forceinline__ float tri_weight(int t) {  // goldstein.cu:257-258
  return (float)(t < GN / 2 ? t : GN - 1 - t);
}

__device__ __forceinline__ int patch_origin(int p, int n) {  // goldstein.cu:308-313
  const int o = p * GSTEP;
  return o + GN > n ? n - GN : o;
}

// Patch p of an nrow x ncol image, by one warp with its padded 32x33 tile
// T; |F| reuses the tile once the column FFT inputs are in registers.
__device__ __forceinline__ void goldstein_patch(const float2 *__restrict__ in, float2 *__restrict__ patches,
                                                int nrow, int ncol, int n_win_j, float alpha, int p,
                                                float2 (*T)[GN + 1]) {
  const int lane = threadIdx.x & 31;
  const int i1 = patch_origin(p / n_win_j, nrow);
  const int j1 = patch_origin(p % n_win_j, ncol);
  float(*M)[GN + 1] = reinterpret_cast<float(*)[GN + 1]>(&T[0][0]);
  float2 x[GN];
  // all 32 row loads in flight at once (one L2 round trip per patch), then
  // the transpose through the tile
#pragma unroll
  for (int r = 0; r < GN; ++r) x[r] = __ldg(in + (size_t)(i1 + r) * ncol + j1 + lane);
#pragma unroll
  for (int r = 0; r < GN; ++r) T[r][lane] = x[r];
  __syncwarp();
  // forward FFT along rows (lane = row)
#pragma unroll
  for (int c = 0; c < GN; ++c) x[c] = T[lane][c];
  fft32<false>(x);
  __syncwarp();
#pragma unroll
  for (int c = 0; c < GN; ++c) T[lane][c] = x[c];
  __syncwarp();
  // forward FFT along columns (lane = column kx); x[ky] = F[ky][kx]
#pragma unroll
  for (int r = 0; r < GN; ++r) x[r] = T[r][lane];
  fft32<false>(x);
  __syncwarp();
#pragma unroll
  // |F|: spectral magnitudes of a 32 x 32 patch of interferogram samples are
  // far from float overflow, so the plain root of the squared sum serves
  for (int r = 0; r < GN; ++r) M[r][lane] = sqrtf(fmaf(x[r].x, x[r].x, x[r].y * x[r].y));
  __syncwarp();
  // 7x7 circular smoothing of |F| (goldstein.cu:105-119) and its patch sum.
  // The table is even in both offsets, g[ky][kx] = g[|ky|][|kx|], so
  //   S[y][x] = W0[y][x] + sum_{b=1..3} (Wb[y][x - b] + Wb[y][x + b]),
  //   Wb[y][x] = sum_{a=0..3} g[a][b] (M[y - a][x] + M[y + a][x])  (a = 0 once):
  // the four vertical filters Wb run down the lane's own column from a
  // sliding window of seven rows, the horizontal offsets are lane shuffles
  // (their wrap-around is the circular boundary).
  float S[GN];
  float psum = 0.f;
  {
    float win[7];  // M[y - 3 .. y + 3][lane]
#pragma unroll
    for (int k = 0; k < 6; ++k) win[k + 1] = M[(k - 3 + GN) & (GN - 1)][lane];
#pragma unroll
    for (int y = 0; y < GN; ++y) {
#pragma unroll
      for (int k = 0; k < 6; ++k) win[k] = win[k + 1];
      win[6] = M[(y + 3) & (GN - 1)][lane];
      const float p1 = win[2] + win[4], p2 = win[1] + win[5], p3 = win[0] + win[6];
      float w[4];
#pragma unroll
      for (int b = 0; b < 4; ++b)  // g[a][b] = c_gauss[(3 - a) * 7 + 3 + b]
        w[b] = fmaf(c_gauss[21 + 3 + b], win[3],
                    fmaf(c_gauss[14 + 3 + b], p1, fmaf(c_gauss[7 + 3 + b], p2, c_gauss[3 + b] * p3)));
      float s = w[0];
#pragma unroll
      for (int b = 1; b < 4; ++b)
        s += __shfl_sync(0xffffffffu, w[b], (lane - b) & (GN - 1)) + __shfl_sync(0xffffffffu, w[b], (lane + b) & (GN - 1));
      S[y] = s;
      psum += s;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) psum += __shfl_xor_sync(0xffffffffu, psum, off);
  // patch-mean normalisation and S^alpha weighting (goldstein.cu:125-176)
  const float mean = psum / (float)(GN * GN);
  const bool ok = mean > 1e-8f;
  const float inv = 1.0f / mean;
#pragma unroll
  for (int y = 0; y < GN; ++y) {
    // S^alpha through the hardware exp2/log2 (relative error ~1e-6, far
    // below the filter's float tolerance); 0^alpha = 0 for alpha > 0, and a
    // NaN weight (0^0) leaves F unscaled, as a weight of 1 would
    const float w = __powf(ok ? S[y] * inv : 0.0f, alpha);
    if (w > 0.0f) {
      x[y].x *= w;
      x[y].y *= w;
    }
  }
  // inverse FFT along columns, then rows
  fft32<true>(x);
  __syncwarp();
#pragma unroll
  for (int y = 0; y < GN; ++y) T[y][lane] = x[y];
  __syncwarp();
#pragma unroll
  for (int c = 0; c < GN; ++c) x[c] = T[lane][c];
  fft32<true>(x);
  // triangular weight and 1/n^2 (goldstein.cu:257-269); stage for a
  // coalesced store
  const float wy = tri_weight(lane);
  const float norm = 1.0f / (float)(GN * GN);
  __syncwarp();
#pragma unroll
  for (int c = 0; c < GN; ++c) {
    const float w = (tri_weight(c) + wy) * norm;
    T[lane][c] = make_float2(x[c].x * w, x[c].y * w);
  }
  __syncwarp();
  float2 *dst = patches + (size_t)p * (GN * GN);
#pragma unroll 8
  for (int r = 0; r < GN; ++r) __stcg(dst + r * GN + lane, T[r][lane]);
}

__global__ __launch_bounds__(32 * GWARPS, GCTAS_PER_SM) void goldstein_patch_kernel(
    const float2 *__restrict__ in, float2 *__restrict__ patches, int nrow, int ncol, int n_win_i,
    int n_win_j, float alpha) {
  __shared__ float2 sT[GWARPS][GN][GN + 1];
  const int warp = threadIdx.x >> 5;
  const int p = blockIdx.x * GWARPS + warp;
  if (p >= n_win_i * n_win_j) return;  // warp-uniform; only __syncwarp below
  goldstein_patch(in, patches, nrow, ncol, n_win_j, alpha, p, sT[warp]);
}

// Output pixel (y, x): fixed-order overlap-add of its covering patches.
__device__ __forceinline__ void goldstein_gather(const float2 *__restrict__ patches, float2 *__restrict__ out,
                                                 int nrow, int ncol, int n_win_i, int n_win_j, int y, int x) {
  float ax = 0.f, ay = 0.f, wsum = 0.f;
  const int pi0 = y >= GN - 1 ? (y - (GN - 1) + GSTEP - 1) / GSTEP : 0;
  const int pj0 = x >= GN - 1 ? (x - (GN - 1) + GSTEP - 1) / GSTEP : 0;
  for (int pi = pi0; pi < n_win_i; ++pi) {
    const int i1 = patch_origin(pi, nrow);
    if (i1 > y) break;
    if (y >= i1 + GN) continue;
    const int ty = y - i1;
    const float wy = tri_weight(ty);
    for (int pj = pj0; pj < n_win_j; ++pj) {
      const int j1 = patch_origin(pj, ncol);
      if (j1 > x) break;
      if (x >= j1 + GN) continue;
      const int tx = x - j1;
      const float2 v = __ldcg(patches + ((size_t)pi * n_win_j + pj) * (GN * GN) + ty * GN + tx);
      ax += v.x;
      ay += v.y;
      wsum += tri_weight(tx) + wy;
    }
  }
  if (wsum > 0.f) {  // goldstein.cu:287-291
    ax /= wsum;
    ay /= wsum;
  }
  out[(size_t)y * ncol + x] = make_float2(ax, ay);
}

__global__ __launch_bounds__(256) void goldstein_gather_kernel(const float2 *__restrict__ patches,
                                                               float2 *__restrict__ out, int nrow,
                                                               int ncol, int n_win_i, int n_win_j) {
  const int x = blockIdx.y * 256 + threadIdx.x;
  if (x >= ncol) return;
  goldstein_gather(patches, out, nrow, ncol, n_win_i, n_win_j, blockIdx.x, x);
}

__host__ __device__ inline void patch_grid(int nrow, int ncol, int &n_win_i, int &n_win_j) {  // goldstein.cu:335-340
  n_win_i = (int)ceilf((float)nrow / GSTEP) - 3;
  n_win_j = (int)ceilf((float)ncol / GSTEP) - 3;
  if (n_win_i <= 0) n_win_i = 1;
  if (n_win_j <= 0) n_win_j = 1;
}


// ------------------------------------------------------------ frame stages
// Goldstein of every pair's interferogram: blockIdx.y = pair.  Pairs too
// small to filter get filt = ifg from the gather kernel.
__global__ __launch_bounds__(32 * GWARPS, GCTAS_PER_SM) void frame_goldstein_patch_kernel(const FrameDev d, const FrameIO io) {
  __shared__ float2 sT[GWARPS][GN][GN + 1];
  const int k = blockIdx.y;
  const s1b_frame_pair_t &r = io.pout[k];
  if (!r.ok || !r.filtered) return;
  int ni, nj;
  patch_grid(r.nrow_ml, r.ncol_ml, ni, nj);
  const int warp = threadIdx.x >> 5;
  const int p = blockIdx.x * GWARPS + warp;
  if (p >= ni * nj) return;  // warp-uniform
  const FramePair &pr = d.pairs[k];
  goldstein_patch(io.ifg + pr.ml_off, io.work + pr.scratch_off, r.nrow_ml, r.ncol_ml, nj, d.alpha, p, sT[warp]);
}

__global__ __launch_bounds__(256) void frame_goldstein_gather_kernel(const FrameDev d, const FrameIO io) {
  const int k = blockIdx.z;
  const s1b_frame_pair_t &r = io.pout[k];
  const int y = blockIdx.x, x = blockIdx.y * 256 + threadIdx.x;
  if (!r.ok || y >= r.nrow_ml || x >= r.ncol_ml) return;
  const FramePair &pr = d.pairs[k];
  if (r.filtered) {
    int ni, nj;
    patch_grid(r.nrow_ml, r.ncol_ml, ni, nj);
    goldstein_gather(io.work + pr.scratch_off, io.filt + pr.ml_off, r.nrow_ml, r.ncol_ml, ni, nj, y, x);
  } else {
    const size_t o = pr.ml_off + (size_t)y * r.ncol_ml + x;
    io.filt[o] = io.ifg[o];
  }
}

}  // namespace

extern "C" size_t s1b_goldstein_scratch_bytes(int32_t nrow, int32_t ncol, int32_t n_win) {
  if (n_win != GN || nrow < GN || ncol < GN) return 0;
  int ni, nj;
  patch_grid(nrow, ncol, ni, nj);
  return (size_t)ni * nj * GN * GN * sizeof(float2);
}

extern "C" int s1b_goldstein(const void *in, void *out, int32_t nrow, int32_t ncol, int32_t n_win,
                             float alpha, void *scratch, size_t scratch_bytes, void *stream) {
  if (!in || !out) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_goldstein: null argument");
  if (n_win != GN) return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_goldstein: only n_win = 32 is implemented");
  if (nrow < GN || ncol < GN)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_goldstein: image smaller than the window");
  const size_t need = s1b_goldstein_scratch_bytes(nrow, ncol, n_win);
  if (!scratch || scratch_bytes < need)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_goldstein: scratch buffer too small");
  int ni, nj;
  patch_grid(nrow, ncol, ni, nj);
  const int64_t npatch = (int64_t)ni * nj;
  if ((npatch + GWARPS - 1) / GWARPS > 0x7fffffff || (ncol + 255) / 256 > 65535)
    return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_goldstein: image too large");
  cudaStream_t st = (cudaStream_t)stream;
  goldstein_patch_kernel<<<(unsigned)((npatch + GWARPS - 1) / GWARPS), 32 * GWARPS, 0, st>>>(
      (const float2 *)in, (float2 *)scratch, nrow, ncol, ni, nj, alpha);
  int s = s1b_launch_status();
  if (s) return s;
  dim3 grid(nrow, (ncol + 255) / 256);
  goldstein_gather_kernel<<<grid, 256, 0, st>>>((const float2 *)scratch, (float2 *)out, nrow, ncol,
                                                ni, nj);
  return s1b_launch_status();
}

// ---------------------------------------------------------------------------
// Goldstein without any device allocation.
//
// Some callers cannot allocate device memory when they filter: a plugin
// running inside a host application whose own pool allocator has already
// reserved the GPU's memory (a raw cudaMalloc then fails although the pool
// has room), or a pipeline that forbids allocation after start-up to keep a
// fixed footprint.  For them the patch scratch lives in a file-scope device
// array of fixed size that every GPU loading this library holds until the
// process exits.
namespace {

constexpr size_t kNoAllocMaxPatches = S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES;
__device__ __align__(256) float2 g_goldstein_scratch[kNoAllocMaxPatches * GN * GN];

// The array's device address, per CUDA context (see s1b_ctx_cache.h).
ContextKeyedCache<64> g_scratch_cache;

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// The calling thread's current context and its unique id, through the
// driver entry points the runtime hands out (no link against libcuda).
// ctx is null when no context is current; cacheable is false when the
// driver cannot give the id, and then nothing is cached.
int current_context(const void **ctx, uint64_t *id, bool *cacheable) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
    cudaGetLastError();
  });
  *ctx = nullptr;
  *id = 0;
  *cacheable = false;
  if (!get_current) return S1B_OK;
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS) return s1b_fail(S1B_ERR_CUDA, "s1b_goldstein_noalloc: cuCtxGetCurrent failed");
  *ctx = c;
  unsigned long long u = 0;
  if (c && get_id && get_id(c, &u) == CUDA_SUCCESS) {
    *id = u;
    *cacheable = true;
  }
  return S1B_OK;
}

// Device address of g_goldstein_scratch in the calling thread's current
// context.  The symbol name is only a host-side handle.  The address is
// looked up with cudaGetSymbolAddress the first time a context calls (which
// makes the device's primary context current when none is) and cached under
// that context's handle and id.
int noalloc_scratch(void **ptr) {
  const void *ctx;
  uint64_t id;
  bool cacheable;
  int s = current_context(&ctx, &id, &cacheable);
  if (s) return s;
  if (cacheable && g_scratch_cache.find(ctx, id, ptr)) return S1B_OK;
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_goldstein_scratch);
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  s = current_context(&ctx, &id, &cacheable);  // the context the lookup ran in
  if (s) return s;
  if (cacheable) g_scratch_cache.put(ctx, id, p);
  *ptr = p;
  return S1B_OK;
}

}  // namespace

extern "C" int s1b_goldstein_noalloc(const void *in, void *out, int32_t nrow, int32_t ncol,
                                     int32_t n_win, float alpha, void *stream) {
  if (!in || !out) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_goldstein_noalloc: null argument");
  if (n_win != GN) return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_goldstein_noalloc: only n_win = 32 is implemented");
  if (nrow < GN || ncol < GN)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_goldstein_noalloc: image smaller than the window");
  int ni, nj;
  patch_grid(nrow, ncol, ni, nj);
  const int64_t npatch = (int64_t)ni * nj;
  if (npatch > (int64_t)kNoAllocMaxPatches)
    return s1b_fail(S1B_ERR_TOO_LARGE,
                    "s1b_goldstein_noalloc: image needs more than S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES (4096) "
                    "patches of its fixed scratch (about 512 x 512 pixels); use s1b_goldstein");
  if ((ncol + 255) / 256 > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_goldstein_noalloc: image too wide");
  void *scratch = nullptr;
  int s = noalloc_scratch(&scratch);
  if (s) return s;
  // every patch slot used below is written by the patch kernel before the
  // gather reads it, so nothing left by an earlier call needs clearing
  cudaStream_t st = (cudaStream_t)stream;
  goldstein_patch_kernel<<<(unsigned)((npatch + GWARPS - 1) / GWARPS), 32 * GWARPS, 0, st>>>(
      (const float2 *)in, (float2 *)scratch, nrow, ncol, ni, nj, alpha);
  s = s1b_launch_status();
  if (s) return s;
  dim3 grid(nrow, (ncol + 255) / 256);
  goldstein_gather_kernel<<<grid, 256, 0, st>>>((const float2 *)scratch, (float2 *)out, nrow, ncol, ni, nj);
  return s1b_launch_status();
}

int frame_goldstein_patch_grid(int nrow, int ncol, int *ni, int *nj) {
  patch_grid(nrow, ncol, *ni, *nj);
  return S1B_OK;
}

int frame_launch_goldstein(const FrameDev &d, const FrameIO &io, cudaStream_t st) {
  if (d.max_nrow_ml <= 0 || d.max_ncol_ml <= 0) return S1B_OK;
  if (d.n_win != GN) return s1b_fail(S1B_ERR_UNSUPPORTED, "frame goldstein: only n_win = 32 is implemented");
  if (d.n_pairs > 65535 || (d.max_ncol_ml + 255) / 256 > 65535)
    return s1b_fail(S1B_ERR_TOO_LARGE, "frame goldstein: grid too large");
  if (d.max_patches > 0) {
    dim3 g1((d.max_patches + GWARPS - 1) / GWARPS, d.n_pairs);
    frame_goldstein_patch_kernel<<<g1, 32 * GWARPS, 0, st>>>(d, io);
    int s = s1b_launch_status();
    if (s) return s;
  }
  dim3 g2(d.max_nrow_ml, (d.max_ncol_ml + 255) / 256, d.n_pairs);
  frame_goldstein_gather_kernel<<<g2, 256, 0, st>>>(d, io);
  return s1b_launch_status();
}

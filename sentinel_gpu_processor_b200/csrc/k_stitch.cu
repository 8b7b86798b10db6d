// Burst stitching of burst interferograms into a frame (the reference's
// s1proc/interfere.py:81-180, NumPy on memmaps there).
//
// Per subswath (one CTA, bursts in order of top + bottom as Subswath.sort,
// s1proc/sario.py:239-244): the first burst is placed into the subswath
// mosaic (the union box of the first and last burst, sario.py:230-237); each
// later burst, when its pair of burst ids differs from the previous one,
// estimates the phase offset over its overlap with the mosaic:
//   m = angle(mean(conj(old) new)),  m += median(angle(conj(old) new e^{-i m}))
// (float mode: differences of phases instead of products), and is written
// rotated by -m where the mosaic is still empty (real part 0).  The offset
// carries over to later bursts without an overlap, as in the reference.
// The mean is summed in FP64 in a fixed order; the median is exact, found by
// a 32-bit radix select over the float angles (two selections for an even
// count).  Then the frame: subswaths 1..3 written in order where non-zero.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_internal.h"

namespace {

constexpr int ST_THREADS = 1024;

struct Swath {
  int32_t first, count;               // bursts [first, first + count) of the sorted table
  int32_t left, top, right, bottom;   // mosaic box
  int64_t moff;                       // mosaic, elements into the workspace
};

struct Bst {
  int64_t off;
  int32_t left, top, right, bottom, group;
};

__device__ __forceinline__ uint32_t fkey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float keyf(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

template <bool kFloat>
struct Px;

template <>
struct Px<false> {
  using T = float2;
  __device__ static bool empty(T v) { return v.x == 0.f; }  // .real == 0, as the reference masks
  __device__ static bool nonzero(T v) { return v.x != 0.f || v.y != 0.f; }
};

template <>
struct Px<true> {
  using T = float;
  __device__ static bool empty(T v) { return v == 0.f; }
  __device__ static bool nonzero(T v) { return v != 0.f; }
};

// conj(old) new (complex) or exp(i (new - old)) (phase) of an overlap pixel.
__device__ __forceinline__ float2 pdiff(float2 o, float2 n) {
  return make_float2(o.x * n.x + o.y * n.y, o.x * n.y - o.y * n.x);
}
__device__ __forceinline__ float2 pdiff(float o, float n) {
  float s, c;
  sincosf(n - o, &s, &c);
  return make_float2(c, s);
}

template <bool kFloat>
__global__ __launch_bounds__(ST_THREADS) void stitch_swath_kernel(const Bst *__restrict__ bursts,
                                                                  const Swath *__restrict__ swaths,
                                                                  const void *__restrict__ data_raw,
                                                                  void *__restrict__ mos_raw,
                                                                  double *__restrict__ offsets) {
  using T = typename Px<kFloat>::T;
  const T *data = reinterpret_cast<const T *>(data_raw);
  T *mos_all = reinterpret_cast<T *>(mos_raw);
  __shared__ double s_sum[3][ST_THREADS / 32];
  __shared__ unsigned s_hist[256];
  __shared__ unsigned s_sel[3];  // prefix, mask, rank
  __shared__ double s_bc[2];
  const Swath sw = swaths[blockIdx.x];
  const int tid = threadIdx.x;
  const int W = sw.right - sw.left;
  T *mos = mos_all + sw.moff;
  const int64_t msize = (int64_t)W * (sw.bottom - sw.top);
  for (int64_t i = tid; i < msize; i += ST_THREADS) mos[i] = T{};
  __syncthreads();
  double mpd = 0.0;  // phase offset carried from burst to burst
  int prev_group = 0, cov_top = 0, cov_bottom = 0;
  for (int q = 0; q < sw.count; ++q) {
    const Bst b = bursts[sw.first + q];
    const int bw = b.right - b.left;
    // the burst's box inside the mosaic box
    const int l = max(b.left, sw.left), r = min(b.right, sw.right);
    const int t = max(b.top, sw.top), u = min(b.bottom, sw.bottom);
    const T *src = data + b.off;
    if (q > 0 && b.group != prev_group && l < r) {
      // rows of this burst that earlier bursts covered hold the overlap
      const int ot = max(t, cov_top), ob = min(u, cov_bottom);
      const int ow = r - l;
      const int64_t on = ob > ot ? (int64_t)(ob - ot) * ow : 0;
      double sx = 0.0, sy = 0.0, sn = 0.0;
      for (int64_t i = tid; i < on; i += ST_THREADS) {
        const int y = ot + (int)(i / ow), x = l + (int)(i % ow);
        const T o = mos[(int64_t)(y - sw.top) * W + (x - sw.left)];
        const T n = src[(int64_t)(y - b.top) * bw + (x - b.left)];
        if (!Px<kFloat>::empty(o) && Px<kFloat>::nonzero(n)) {
          const float2 d = pdiff(o, n);
          sx += d.x;
          sy += d.y;
          sn += 1.0;
        }
      }
      // fixed-order block reduction: warps by shuffles, then warp sums in order
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        sx += __shfl_down_sync(0xffffffffu, sx, off);
        sy += __shfl_down_sync(0xffffffffu, sy, off);
        sn += __shfl_down_sync(0xffffffffu, sn, off);
      }
      if ((tid & 31) == 0) {
        s_sum[0][tid >> 5] = sx;
        s_sum[1][tid >> 5] = sy;
        s_sum[2][tid >> 5] = sn;
      }
      __syncthreads();
      if (tid == 0) {
        double ax = 0, ay = 0, an = 0;
        for (int w = 0; w < ST_THREADS / 32; ++w) {
          ax += s_sum[0][w];
          ay += s_sum[1][w];
          an += s_sum[2][w];
        }
        s_bc[0] = an > 0 ? atan2(ay, ax) : 0.0;
        s_bc[1] = an;
      }
      __syncthreads();
      const double mean = s_bc[0];
      const unsigned n = (unsigned)s_bc[1];
      if (n > 0) {
        // exact median of angle(d e^{-i mean}) by radix select
        const float cm = (float)cos(mean), sm = (float)sin(mean);
        float med2[2];
        const unsigned ranks[2] = {(n - 1) / 2, n / 2};
        for (int sel = 0; sel < 2; ++sel) {
          if (tid == 0) {
            s_sel[0] = 0;
            s_sel[1] = 0;
            s_sel[2] = ranks[sel];
          }
          for (int shift = 24; shift >= 0; shift -= 8) {
            for (int i = tid; i < 256; i += ST_THREADS) s_hist[i] = 0;
            __syncthreads();
            const unsigned prefix = s_sel[0], mask = s_sel[1];
            for (int64_t i = tid; i < on; i += ST_THREADS) {
              const int y = ot + (int)(i / ow), x = l + (int)(i % ow);
              const T o = mos[(int64_t)(y - sw.top) * W + (x - sw.left)];
              const T nn = src[(int64_t)(y - b.top) * bw + (x - b.left)];
              if (!Px<kFloat>::empty(o) && Px<kFloat>::nonzero(nn)) {
                const float2 d = pdiff(o, nn);
                const float a = atan2f(d.y * cm - d.x * sm, d.x * cm + d.y * sm);
                const uint32_t k = fkey(a);
                if ((k & mask) == prefix) atomicAdd(&s_hist[(k >> shift) & 255u], 1u);
              }
            }
            __syncthreads();
            if (tid == 0) {
              unsigned rank = s_sel[2], cum = 0, bin = 0;
              for (; bin < 255; ++bin) {
                if (cum + s_hist[bin] > rank) break;
                cum += s_hist[bin];
              }
              s_sel[0] |= bin << shift;
              s_sel[1] |= 255u << shift;
              s_sel[2] = rank - cum;
            }
            __syncthreads();
          }
          med2[sel] = keyf(s_sel[0]);
          __syncthreads();
        }
        // np.median: the middle value, or the mean of the two middle values
        mpd = mean + (n % 2 ? (double)med2[1] : 0.5 * ((double)med2[0] + (double)med2[1]));
      }
    }
    prev_group = b.group;
    if (tid == 0 && offsets) offsets[sw.first + q] = mpd;
    // write the burst where the mosaic is empty (the first burst: everywhere
    // in its box), rotated by -mpd
    const float cr = (float)cos(mpd), sr = (float)sin(mpd);
    const int cw = r - l;
    const int64_t cn = (u > t && cw > 0) ? (int64_t)(u - t) * cw : 0;
    for (int64_t i = tid; i < cn; i += ST_THREADS) {
      const int y = t + (int)(i / cw), x = l + (int)(i % cw);
      T &o = mos[(int64_t)(y - sw.top) * W + (x - sw.left)];
      T v = src[(int64_t)(y - b.top) * bw + (x - b.left)];
      if (q == 0) {
        o = v;
        continue;
      }
      if (!(Px<kFloat>::empty(o) && !Px<kFloat>::empty(v))) continue;
      if (mpd != 0.0) {
        if constexpr (kFloat) {
          double w = (double)v - mpd;
          if (w > kPiD) w -= 2 * kPiD;
          if (w < -kPiD) w += 2 * kPiD;
          v = (float)w;
        } else {
          v = make_float2(v.x * cr + v.y * sr, v.y * cr - v.x * sr);
        }
      }
      o = v;
    }
    __syncthreads();
    cov_top = q == 0 ? b.top : min(cov_top, b.top);
    cov_bottom = q == 0 ? b.bottom : max(cov_bottom, b.bottom);
  }
}

template <bool kFloat>
__global__ void stitch_frame_kernel(const Swath *__restrict__ swaths, int n_swaths, const void *__restrict__ mos_raw,
                                    void *__restrict__ frame_raw, int nrow0, int ncol0) {
  using T = typename Px<kFloat>::T;
  const T *mos = reinterpret_cast<const T *>(mos_raw);
  T *frame = reinterpret_cast<T *>(frame_raw);
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= ncol0) return;
  T v{};
  for (int s = n_swaths - 1; s >= 0; --s) {
    const Swath sw = swaths[s];
    if (x < sw.left || x >= sw.right || y < sw.top || y >= sw.bottom) continue;
    const T m = mos[sw.moff + (int64_t)(y - sw.top) * (sw.right - sw.left) + (x - sw.left)];
    if (Px<kFloat>::empty(m)) continue;  // the reference writes where real (or value) != 0
    v = m;
    break;
  }
  frame[(int64_t)y * ncol0 + x] = v;
}

struct Plan {
  std::vector<Bst> bursts;
  std::vector<Swath> swaths;
  int64_t mos_elems = 0;
};

int make_plan(const s1b_stitch_burst_t *in, int32_t n, Plan &p) {
  for (int sw = 1; sw <= 3; ++sw) {
    std::vector<int> idx;
    for (int i = 0; i < n; ++i)
      if (in[i].subswath == sw) idx.push_back(i);
    if (idx.empty()) continue;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
      return in[a].top + in[a].bottom < in[b].top + in[b].bottom;
    });
    Swath s;
    s.first = (int32_t)p.bursts.size();
    s.count = (int32_t)idx.size();
    const s1b_stitch_burst_t &f = in[idx.front()], &l = in[idx.back()];
    s.left = std::min(f.left, l.left);
    s.top = std::min(f.top, l.top);
    s.right = std::max(f.right, l.right);
    s.bottom = std::max(f.bottom, l.bottom);
    s.moff = p.mos_elems;
    p.mos_elems += (int64_t)(s.right - s.left) * (s.bottom - s.top);
    p.mos_elems = (p.mos_elems + 63) / 64 * 64;
    for (int i : idx) {
      const s1b_stitch_burst_t &b = in[i];
      if (b.right <= b.left || b.bottom <= b.top) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_stitch: empty burst");
      p.bursts.push_back(Bst{b.offset, b.left, b.top, b.right, b.bottom, b.group});
    }
    p.swaths.push_back(s);
  }
  return S1B_OK;
}

}  // namespace

extern "C" size_t s1b_stitch_workspace_bytes(const s1b_stitch_burst_t *bursts, int32_t n, int32_t out_float) {
  Plan p;
  if (!bursts || n < 1 || make_plan(bursts, n, p)) return 0;
  const size_t es = out_float ? 4 : 8;
  return (size_t)p.mos_elems * es + 256 + p.bursts.size() * sizeof(Bst) + 256 + p.swaths.size() * sizeof(Swath) + 256 +
         n * sizeof(double);
}

extern "C" int s1b_stitch(const s1b_stitch_burst_t *bursts, int32_t n, const void *data, int32_t out_float,
                          int32_t nrow0, int32_t ncol0, void *frame, double *offsets_host, void *workspace,
                          size_t workspace_bytes, void *stream) {
  if (!bursts || n < 1 || !data || !frame || !workspace)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_stitch: null argument");
  if (nrow0 < 1 || ncol0 < 1) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_stitch: empty frame");
  for (int i = 0; i < n; ++i) {
    const s1b_stitch_burst_t &b = bursts[i];
    if (b.subswath < 1 || b.subswath > 3)
      return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_stitch: subswath must be 1, 2 or 3");
    if (b.left < 0 || b.top < 0 || b.right > ncol0 || b.bottom > nrow0)
      return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_stitch: burst outside the frame");
  }
  Plan p;
  int s = make_plan(bursts, n, p);
  if (s) return s;
  if (workspace_bytes < s1b_stitch_workspace_bytes(bursts, n, out_float))
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_stitch: workspace too small");
  const size_t es = out_float ? 4 : 8;
  unsigned char *ws = (unsigned char *)workspace;
  void *mos = ws;
  size_t o = ((size_t)p.mos_elems * es + 255) / 256 * 256;
  Bst *d_b = (Bst *)(ws + o);
  o += (p.bursts.size() * sizeof(Bst) + 255) / 256 * 256;
  Swath *d_s = (Swath *)(ws + o);
  o += (p.swaths.size() * sizeof(Swath) + 255) / 256 * 256;
  double *d_off = (double *)(ws + o);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(d_b, p.bursts.data(), p.bursts.size() * sizeof(Bst), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_s, p.swaths.data(), p.swaths.size() * sizeof(Swath), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
  const int ns = (int)p.swaths.size();
  if (out_float)
    stitch_swath_kernel<true><<<ns, ST_THREADS, 0, st>>>(d_b, d_s, data, mos, d_off);
  else
    stitch_swath_kernel<false><<<ns, ST_THREADS, 0, st>>>(d_b, d_s, data, mos, d_off);
  s = s1b_launch_status();
  if (s) return s;
  if (nrow0 > 65535) return s1b_fail(S1B_ERR_TOO_LARGE, "s1b_stitch: frame too tall");
  dim3 grid((ncol0 + 255) / 256, nrow0);
  if (out_float)
    stitch_frame_kernel<true><<<grid, 256, 0, st>>>(d_s, ns, mos, frame, nrow0, ncol0);
  else
    stitch_frame_kernel<false><<<grid, 256, 0, st>>>(d_s, ns, mos, frame, nrow0, ncol0);
  s = s1b_launch_status();
  if (s) return s;
  if (offsets_host) {
    // offsets per burst in the caller's order (the kernel writes them in subswath order)
    std::vector<double> tmp(p.bursts.size());
    e = cudaMemcpyAsync(tmp.data(), d_off, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e));
    size_t k = 0;
    for (int sw = 1; sw <= 3; ++sw) {
      std::vector<int> idx;
      for (int i = 0; i < n; ++i)
        if (bursts[i].subswath == sw) idx.push_back(i);
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        return bursts[a].top + bursts[a].bottom < bursts[b].top + bursts[b].bottom;
      });
      for (int i : idx) offsets_host[i] = tmp[k++];
    }
  }
  return S1B_OK;
}

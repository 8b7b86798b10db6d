// Batched frame: host side of s1b_frame_* (descriptor tables, workspace and
// product layout, the launch sequence of one run, the autotuner).
//
// A run is six to eight launches on one stream with no host synchronisation:
//   init (crop rows), deramp of every burst (one launch per load width),
//   geocoding of every burst (one CTA per tile, or persistent kernels over
//   the flat tile space of the frame), per-pair box
//   and headers from the crop rows, crossmul + looks of every pair, Goldstein
//   patches and overlap-add of every pair.
// The reference runs geo2rdr once per burst and crossmul_daemon / goldstein
// per pair with files in between (csrc/src/geo2rdr.cu:316-651,
// crossmul_daemon.cu:566-975, goldstein.cu:328-408).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "s1b.h"
#include "s1b_frame.h"
#include "s1b_internal.h"

struct s1b_frame {
  int device = 0;
  std::vector<s1b_burst_plan_t> plans;
  std::vector<FrameBurst> bursts;
  std::vector<FramePair> pairs;
  s1b_burst_plan_t *d_plans = nullptr;
  FrameBurst *d_bursts = nullptr;
  FramePair *d_pairs = nullptr;
  int32_t *d_rows = nullptr;
  FrameDev dev{};
  size_t workspace_bytes = 0;
  int64_t slc_elems = 0, product_elems = 0;
  int32_t tuning[4] = {16, 0, 128, 0};  // deramp rows, deramp CTAs, geocoding columns, geocoding CTAs
  FrameDerampSplit split;               // bursts by deramp load width for the current buffers
};

namespace {

constexpr int64_t kAlign = 32;  // complex64 elements (256 bytes) between workspace regions

int64_t align_up(int64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

int cuda_fail(cudaError_t e) { return s1b_fail(S1B_ERR_CUDA, cudaGetErrorString(e)); }

// Flat tile prefixes of the current tile shapes, uploaded to the device.
int set_tiles(s1b_frame *f) {
  int64_t dt = 0, gt = 0;
  int32_t dtx = 0, dty = 0, gtx = 0, gty = 0;
  const int rows = f->tuning[0], cols = f->tuning[2];
  for (size_t b = 0; b < f->bursts.size(); ++b) {
    FrameBurst &fb = f->bursts[b];
    const s1b_burst_plan_t &p = f->plans[b];
    fb.deramp_tile0 = dt;
    fb.geo_tile0 = gt;
    const int32_t tx = (p.samples + kFrameDerampCols - 1) / kFrameDerampCols, ty = (p.lines + rows - 1) / rows;
    dt += (int64_t)tx * ty;
    dtx = std::max(dtx, tx);
    dty = std::max(dty, ty);
    const int32_t gx = (fb.ncol + cols - 1) / cols, gy = (fb.nrow + kFrameGeoRows - 1) / kFrameGeoRows;
    gt += (int64_t)gx * gy;
    gtx = std::max(gtx, gx);
    gty = std::max(gty, gy);
  }
  f->dev.n_deramp_tiles = dt;
  f->dev.n_geo_tiles = gt;
  f->dev.deramp_rows = rows;
  f->dev.deramp_tiles_x = dtx;
  f->dev.deramp_tiles_y = dty;
  f->dev.geo_cols = cols;
  f->dev.geo_tiles_x = gtx;
  f->dev.geo_tiles_y = gty;
  cudaError_t e = cudaMemcpy(f->d_bursts, f->bursts.data(), f->bursts.size() * sizeof(FrameBurst),
                             cudaMemcpyHostToDevice);
  return e == cudaSuccess ? S1B_OK : cuda_fail(e);
}

void release(s1b_frame *f) {
  cudaFree(f->d_plans);
  cudaFree(f->d_bursts);
  cudaFree(f->d_pairs);
  cudaFree(f->d_rows);
  f->d_plans = nullptr;
  f->d_bursts = nullptr;
  f->d_pairs = nullptr;
  f->d_rows = nullptr;
}

int make_io(s1b_frame *f, const void *slc, const int16_t *dem, int64_t dem_pitch, void *workspace, void *ifg,
            float *amp1, float *amp2, float *coh, void *filt, s1b_frame_pair_t *pairs, FrameIO &io) {
  if (!slc || !dem || !workspace || !ifg || !filt || !pairs)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_run: null buffer");
  if (reinterpret_cast<uintptr_t>(workspace) % 16 != 0)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_run: workspace must be 16-byte aligned");
  for (const s1b_burst_plan_t &p : f->plans)
    if (dem_pitch < p.win_right) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_run: dem_pitch below a window");
  io.slc = slc;
  io.dem = dem;
  io.dem_pitch = dem_pitch;
  io.work = (float2 *)workspace;
  io.ifg = (float2 *)ifg;
  io.amp1 = amp1;
  io.amp2 = amp2;
  io.coh = coh;
  io.filt = (float2 *)filt;
  io.pout = pairs;
  f->split.vec.clear();
  f->split.scalar.clear();
  for (size_t b = 0; b < f->bursts.size(); ++b) {
    // two samples per load: 16 bytes (complex64) or 8 (complex int16)
    const size_t es = f->dev.sample_format == S1B_SAMPLES_CI16 ? 4 : 8;
    const bool vec = f->plans[b].samples % 2 == 0 &&
                     (reinterpret_cast<uintptr_t>(io.slc) + es * (uint64_t)f->bursts[b].slc_off) % (2 * es) == 0 &&
                     reinterpret_cast<uintptr_t>(io.work + f->bursts[b].der_off) % 16 == 0;
    (vec ? f->split.vec : f->split.scalar).push_back((int32_t)b);
  }
  return S1B_OK;
}

int run_all(s1b_frame *f, const FrameIO &io, cudaStream_t st) {
  int s = frame_launch_init(f->dev, io, st);
  if (!s) s = frame_launch_deramp(f->dev, io, f->tuning[0], f->tuning[1], f->split, st);
  if (!s) s = frame_launch_geo2rdr(f->dev, io, f->tuning[2], f->tuning[3], st);
  if (!s) s = frame_launch_box(f->dev, io, st);
  if (!s) s = frame_launch_crossmul(f->dev, io, st);
  if (!s) s = frame_launch_goldstein(f->dev, io, st);
  return s;
}

// Device that owns the frame is current for the duration of a call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int s1b_frame_create(const s1b_burst_plan_t *plans, int32_t n_bursts, const int32_t *pair_ref,
                                const int32_t *pair_sec, int32_t n_pairs, int32_t rowlook, int32_t collook,
                                int32_t n_win, float alpha, uint64_t fill_seed, s1b_frame_t **frame) {
  if (!frame) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_create: null frame");
  *frame = nullptr;
  if (!plans || n_bursts < 1 || n_pairs < 1 || !pair_ref || !pair_sec)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_create: no bursts or pairs");
  if (rowlook < 1 || collook < 1) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_create: bad looks");
  if (n_win != 32) return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_frame_create: only n_win = 32 is implemented");
  s1b_frame *f = new s1b_frame();
  f->dev.fused_deramp = 1;  // the geocoding deramps its gathers (s1b_frame_set_deramp_fusion)
  if (cudaGetDevice(&f->device) != cudaSuccess) {
    delete f;
    return s1b_fail(S1B_ERR_NO_DEVICE, "s1b_frame_create: no CUDA device");
  }
  f->plans.assign(plans, plans + n_bursts);
  f->bursts.resize(n_bursts);
  int64_t slc = 0, work = 0;
  for (int b = 0; b < n_bursts; ++b) {
    const s1b_burst_plan_t &p = plans[b];
    FrameBurst &fb = f->bursts[b];
    fb.nrow = p.win_bottom - p.win_top;
    fb.ncol = p.win_right - p.win_left;
    if (fb.nrow <= 0 || fb.ncol <= 0 || p.lines < 2 || p.samples < 2) {
      delete f;
      return s1b_fail(S1B_ERR_EMPTY, "s1b_frame_create: a burst has an empty DEM window");
    }
    fb.slc_off = slc;
    slc += (int64_t)p.lines * p.samples;
    fb.der_off = work;
    // the deramped copy, or (fused deramp) the two TOPS column tables of 32 B per column
    work = align_up(work + (int64_t)std::max(p.lines, 4) * p.samples);
  }
  for (int b = 0; b < n_bursts; ++b) {
    f->bursts[b].geo_off = work;
    work = align_up(work + (int64_t)f->bursts[b].nrow * f->bursts[b].ncol);
  }
  f->pairs.resize(n_pairs);
  int64_t ml = 0;
  int max_r = 0, max_c = 0, max_p = 0;
  for (int k = 0; k < n_pairs; ++k) {
    FramePair &pr = f->pairs[k];
    pr.ref = pair_ref[k];
    pr.sec = pair_sec[k];
    if (pr.ref < 0 || pr.ref >= n_bursts || pr.sec < 0 || pr.sec >= n_bursts) {
      delete f;
      return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_create: pair burst index out of range");
    }
    // the overlap box lies inside both windows
    pr.max_nrow_ml = std::min(f->bursts[pr.ref].nrow, f->bursts[pr.sec].nrow) / rowlook + 1;
    pr.max_ncol_ml = std::min(f->bursts[pr.ref].ncol, f->bursts[pr.sec].ncol) / collook + 1;
    pr.ml_off = ml;
    ml += (int64_t)pr.max_nrow_ml * pr.max_ncol_ml;
    int ni = 0, nj = 0;
    frame_goldstein_patch_grid(pr.max_nrow_ml, pr.max_ncol_ml, &ni, &nj);
    pr.scratch_off = work;
    work = align_up(work + (int64_t)ni * nj * 32 * 32);
    max_r = std::max(max_r, pr.max_nrow_ml);
    max_c = std::max(max_c, pr.max_ncol_ml);
    max_p = std::max(max_p, ni * nj);
    // look-row sums of the fused crossmul over the union of the two windows
    const s1b_burst_plan_t &a = plans[pr.ref], &c = plans[pr.sec];
    const int top = std::min(a.win_top, c.win_top), bottom = std::max(a.win_bottom, c.win_bottom);
    pr.part_top = top / rowlook * rowlook;
    pr.part_rows = (bottom - pr.part_top + rowlook - 1) / rowlook;
    pr.part_left = std::min(a.win_left, c.win_left);
    pr.part_cols = std::max(a.win_right, c.win_right) - pr.part_left;
    pr.part_off = work;
    work = align_up(work + 2 * (int64_t)pr.part_rows * pr.part_cols);  // float4 = 2 complex64
  }
  f->slc_elems = slc;
  f->product_elems = ml;
  f->workspace_bytes = (size_t)work * 8;
  cudaError_t e = cudaMalloc(&f->d_plans, n_bursts * sizeof(s1b_burst_plan_t));
  if (e == cudaSuccess) e = cudaMalloc(&f->d_bursts, n_bursts * sizeof(FrameBurst));
  if (e == cudaSuccess) e = cudaMalloc(&f->d_pairs, n_pairs * sizeof(FramePair));
  if (e == cudaSuccess) e = cudaMalloc(&f->d_rows, 2 * n_bursts * sizeof(int32_t));
  if (e == cudaSuccess)
    e = cudaMemcpy(f->d_plans, plans, n_bursts * sizeof(s1b_burst_plan_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(f->d_pairs, f->pairs.data(), n_pairs * sizeof(FramePair), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    release(f);
    delete f;
    return cuda_fail(e);
  }
  FrameDev &d = f->dev;
  d.plans = f->d_plans;
  d.bursts = f->d_bursts;
  d.pairs = f->d_pairs;
  d.rows = f->d_rows;
  d.n_bursts = n_bursts;
  d.n_pairs = n_pairs;
  d.rowlook = rowlook;
  d.collook = collook;
  d.n_win = n_win;
  d.alpha = alpha;
  d.fill_seed = fill_seed;
  d.max_nrow_ml = max_r;
  d.max_ncol_ml = max_c;
  d.max_patches = max_p;
  // crossmul fused into the geocoding when a look row fits a geocoding tile
  d.fused_xmul = rowlook <= kFrameGeoRows ? 1 : 0;
  d.xm_tiles_x = d.xm_tiles_y = 0;
  if (d.fused_xmul)
    for (const FramePair &pr : f->pairs) {
      d.xm_tiles_x = std::max(d.xm_tiles_x, (pr.part_cols + kFrameXmCols - 1) / kFrameXmCols);
      d.xm_tiles_y = std::max(d.xm_tiles_y, (pr.part_rows + kFrameGeoRows / rowlook - 1) / (kFrameGeoRows / rowlook));
    }
  int s = set_tiles(f);
  if (s) {
    release(f);
    delete f;
    return s;
  }
  *frame = f;
  return S1B_OK;
}

extern "C" void s1b_frame_destroy(s1b_frame_t *frame) {
  if (!frame) return;
  DeviceGuard g(frame->device);
  release(frame);
  delete frame;
}

extern "C" int s1b_frame_sizes(const s1b_frame_t *f, s1b_frame_sizes_t *sizes) {
  if (!f || !sizes) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_sizes: null argument");
  sizes->workspace_bytes = f->workspace_bytes;
  sizes->slc_elems = f->slc_elems;
  sizes->product_elems = f->product_elems;
  sizes->max_nrow_ml = f->dev.max_nrow_ml;
  sizes->max_ncol_ml = f->dev.max_ncol_ml;
  return S1B_OK;
}

extern "C" int s1b_frame_burst_offset(const s1b_frame_t *f, int32_t burst, int64_t *slc_off) {
  if (!f || !slc_off || burst < 0 || burst >= (int32_t)f->bursts.size())
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_burst_offset: bad argument");
  *slc_off = f->bursts[burst].slc_off;
  return S1B_OK;
}

extern "C" int s1b_frame_pair_slot(const s1b_frame_t *f, int32_t pair, int64_t *ml_off, int32_t *max_nrow_ml,
                                   int32_t *max_ncol_ml) {
  if (!f || pair < 0 || pair >= (int32_t)f->pairs.size())
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_pair_slot: bad argument");
  if (ml_off) *ml_off = f->pairs[pair].ml_off;
  if (max_nrow_ml) *max_nrow_ml = f->pairs[pair].max_nrow_ml;
  if (max_ncol_ml) *max_ncol_ml = f->pairs[pair].max_ncol_ml;
  return S1B_OK;
}

extern "C" int s1b_frame_run(s1b_frame_t *f, const void *slc, const int16_t *dem, int64_t dem_pitch,
                             void *workspace, void *ifg, float *amp1, float *amp2, float *coh, void *filt,
                             s1b_frame_pair_t *pairs, void *stream) {
  if (!f) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_run: null frame");
  FrameIO io;
  int s = make_io(f, slc, dem, dem_pitch, workspace, ifg, amp1, amp2, coh, filt, pairs, io);
  if (s) return s;
  return run_all(f, io, (cudaStream_t)stream);
}

extern "C" int s1b_frame_tuning(const s1b_frame_t *f, int32_t tuning[4]) {
  if (!f || !tuning) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_tuning: null argument");
  std::memcpy(tuning, f->tuning, sizeof(f->tuning));
  return S1B_OK;
}

extern "C" int s1b_frame_set_deramp_fusion(s1b_frame_t *f, int32_t fused) {
  if (!f) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_set_deramp_fusion: null frame");
  f->dev.fused_deramp = fused ? 1 : 0;
  return S1B_OK;
}

extern "C" int s1b_frame_set_crossmul_fusion(s1b_frame_t *f, int32_t fused) {
  if (!f) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_set_crossmul_fusion: null frame");
  if (fused && f->dev.rowlook > kFrameGeoRows)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_frame_set_crossmul_fusion: rowlook above 128");
  if (fused && f->dev.xm_tiles_x == 0)
    for (const FramePair &pr : f->pairs) {
      f->dev.xm_tiles_x = std::max(f->dev.xm_tiles_x, (pr.part_cols + kFrameXmCols - 1) / kFrameXmCols);
      f->dev.xm_tiles_y = std::max(f->dev.xm_tiles_y, (pr.part_rows + kFrameGeoRows / f->dev.rowlook - 1) /
                                                          (kFrameGeoRows / f->dev.rowlook));
    }
  f->dev.fused_xmul = fused ? 1 : 0;
  return S1B_OK;
}

extern "C" int s1b_frame_set_sample_format(s1b_frame_t *f, int32_t format) {
  if (!f) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_set_sample_format: null frame");
  if (format != S1B_SAMPLES_C64 && format != S1B_SAMPLES_CI16)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_frame_set_sample_format: S1B_SAMPLES_C64 or S1B_SAMPLES_CI16");
  f->dev.sample_format = format;
  return S1B_OK;
}

extern "C" int s1b_frame_set_tuning(s1b_frame_t *f, const int32_t tuning[4]) {
  if (!f || !tuning) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_set_tuning: null argument");
  if (frame_max_ctas_deramp(tuning[0]) <= 0 || frame_max_ctas_geo2rdr(f->dev, tuning[2]) <= 0)
    return s1b_fail(S1B_ERR_UNSUPPORTED, "s1b_frame_set_tuning: deramp rows 8/16/32, geocoding columns 64/128/256");
  if (tuning[1] < 0 || tuning[3] < 0)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_set_tuning: negative CTA count");
  DeviceGuard g(f->device);
  std::memcpy(f->tuning, tuning, sizeof(f->tuning));
  return set_tiles(f);
}

extern "C" int s1b_frame_autotune(s1b_frame_t *f, const void *slc, const int16_t *dem, int64_t dem_pitch,
                                  void *workspace, void *ifg, float *amp1, float *amp2, float *coh, void *filt,
                                  s1b_frame_pair_t *pairs, int32_t reps, void *stream) {
  if (!f) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_autotune: null frame");
  FrameIO io;
  int s = make_io(f, slc, dem, dem_pitch, workspace, ifg, amp1, amp2, coh, filt, pairs, io);
  if (s) return s;
  if (reps < 1) reps = 1;
  cudaStream_t st = (cudaStream_t)stream;
  int sms = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, f->device);
  if (e != cudaSuccess) return cuda_fail(e);
  cudaEvent_t a, b;
  if ((e = cudaEventCreate(&a)) != cudaSuccess) return cuda_fail(e);
  if ((e = cudaEventCreate(&b)) != cudaSuccess) {
    cudaEventDestroy(a);
    return cuda_fail(e);
  }
  // time `stage` (0 deramp, 1 geocoding) with tile shape `shape` and grid `ctas`
  auto time_stage = [&](int stage, int shape, int ctas, float &ms) -> int {
    int32_t t[4];
    std::memcpy(t, f->tuning, sizeof(t));
    t[stage * 2] = shape;
    t[stage * 2 + 1] = ctas;
    int r = s1b_frame_set_tuning(f, t);
    if (r) return r;
    for (int i = 0; i <= reps; ++i) {  // the first run is a warm-up
      if (i == 1 && (e = cudaEventRecord(a, st)) != cudaSuccess) return cuda_fail(e);
      r = stage == 0 ? frame_launch_deramp(f->dev, io, shape, ctas, f->split, st)
                     : frame_launch_geo2rdr(f->dev, io, shape, ctas, st);
      if (r) return r;
    }
    if ((e = cudaEventRecord(b, st)) != cudaSuccess || (e = cudaEventSynchronize(b)) != cudaSuccess ||
        (e = cudaEventElapsedTime(&ms, a, b)) != cudaSuccess)
      return cuda_fail(e);
    return S1B_OK;
  };
  s = frame_launch_init(f->dev, io, st);
  const int shapes[2][3] = {{8, 16, 32}, {64, 128, 256}};
  for (int stage = 0; stage < 2 && !s; ++stage) {
    if (stage == 0 && f->dev.fused_deramp) {
      // nothing to tune: one launch writes the column tables the geocoding
      // candidates read
      s = frame_launch_deramp(f->dev, io, f->tuning[0], f->tuning[1], f->split, st);
      continue;
    }
    if (stage == 1 && f->dev.fused_xmul) continue;  // the fused kernel has one tile shape
    int best_shape = f->tuning[stage * 2], best_ctas = f->tuning[stage * 2 + 1];
    float best = 3.4e38f;
    for (int shape : shapes[stage]) {
      const int full = stage == 0 ? frame_max_ctas_deramp(shape) : frame_max_ctas_geo2rdr(f->dev, shape);
      const int per_sm = sms > 0 ? full / sms : 0;
      // one CTA per tile (0), then persistent grids of 1..per_sm CTAs per SM
      for (int j = 0; j <= per_sm && !s; ++j) {
        const int ctas = j * sms;
        float ms = 0.f;
        s = time_stage(stage, shape, ctas, ms);
        if (!s && ms < best) {
          best = ms;
          best_shape = shape;
          best_ctas = ctas;
        }
      }
    }
    if (!s) {
      int32_t t[4];
      std::memcpy(t, f->tuning, sizeof(t));
      t[stage * 2] = best_shape;
      t[stage * 2 + 1] = best_ctas;
      s = s1b_frame_set_tuning(f, t);
      // the geocoding candidates read the deramped bursts of the chosen deramp
      if (!s && stage == 0) s = frame_launch_deramp(f->dev, io, f->tuning[0], f->tuning[1], f->split, st);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (!s && (e = cudaStreamSynchronize(st)) != cudaSuccess) s = cuda_fail(e);
  return s;
}

extern "C" int s1b_frame_profile(s1b_frame_t *f, const void *slc, const int16_t *dem, int64_t dem_pitch,
                                 void *workspace, void *ifg, float *amp1, float *amp2, float *coh, void *filt,
                                 s1b_frame_pair_t *pairs, float *stage_ms, void *stream) {
  if (!f || !stage_ms) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_frame_profile: null argument");
  FrameIO io;
  int s = make_io(f, slc, dem, dem_pitch, workspace, ifg, amp1, amp2, coh, filt, pairs, io);
  if (s) return s;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t ev[7];
  int made = 0;
  cudaError_t e = cudaSuccess;
  for (; made < 7 && e == cudaSuccess; ++made) e = cudaEventCreate(&ev[made]);
  if (e != cudaSuccess) {
    for (int i = 0; i < made - 1; ++i) cudaEventDestroy(ev[i]);
    return cuda_fail(e);
  }
  // stages: [init + deramp, geocoding, box, crossmul, Goldstein] between events
  s = frame_launch_init(f->dev, io, st);
  if (!s) e = cudaEventRecord(ev[0], st);
  if (!s && e == cudaSuccess) s = frame_launch_deramp(f->dev, io, f->tuning[0], f->tuning[1], f->split, st);
  if (!s && e == cudaSuccess) e = cudaEventRecord(ev[1], st);
  if (!s && e == cudaSuccess) s = frame_launch_geo2rdr(f->dev, io, f->tuning[2], f->tuning[3], st);
  if (!s && e == cudaSuccess) e = cudaEventRecord(ev[2], st);
  if (!s && e == cudaSuccess) s = frame_launch_box(f->dev, io, st);
  if (!s && e == cudaSuccess) e = cudaEventRecord(ev[3], st);
  if (!s && e == cudaSuccess) s = frame_launch_crossmul(f->dev, io, st);
  if (!s && e == cudaSuccess) e = cudaEventRecord(ev[4], st);
  if (!s && e == cudaSuccess) s = frame_launch_goldstein(f->dev, io, st);
  if (!s && e == cudaSuccess) e = cudaEventRecord(ev[5], st);
  if (!s && e == cudaSuccess) e = cudaEventSynchronize(ev[5]);
  for (int i = 0; i < 5 && !s && e == cudaSuccess; ++i) e = cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
  for (int i = 0; i < 7; ++i) cudaEventDestroy(ev[i]);
  if (!s && e != cudaSuccess) s = cuda_fail(e);
  return s;
}

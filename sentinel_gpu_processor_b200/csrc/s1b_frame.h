// Batched frame: device descriptor tables shared by the frame kernels and the
// host orchestrator (frame.cpp).  Internal; the public surface is
// s1b_frame_* in s1b.h.
#ifndef S1B_FRAME_H
#define S1B_FRAME_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "s1b.h"

// One burst of a frame, geocoded onto the frame's DEM grid.
struct FrameBurst {
  int64_t slc_off;       // first complex64 element of the burst in the caller's SLC buffer
  int64_t der_off;       // its deramped copy, complex64 elements into the workspace
  int64_t geo_off;       // its geocoded DEM window, complex64 elements into the workspace
  int64_t deramp_tile0;  // first index of the burst in the flat deramp tile space
  int64_t geo_tile0;     // first index of the burst in the flat geocoding tile space
  int32_t nrow, ncol;    // DEM window
};

// One interferometric pair and the slots of its products.
struct FramePair {
  int32_t ref, sec;                  // burst indices
  int32_t max_nrow_ml, max_ncol_ml;  // slot capacity (multilooked pixels)
  int64_t ml_off;                    // first element of its slot in every product array
  int64_t scratch_off;               // Goldstein patches, complex64 elements into the workspace
  // Look-row sums of the crossmul fused into the geocoding: one float4 per
  // column and look row over the union of the two DEM windows, rows aligned
  // to the looks on the RSC grid (row part_top, column part_left first).
  int64_t part_off;                  // complex64 elements into the workspace
  int32_t part_top, part_left;       // RSC grid row (a multiple of rowlook) and column of element 0
  int32_t part_rows, part_cols;      // look rows, columns
};

// Everything a frame kernel needs, passed by value.
struct FrameDev {
  const s1b_burst_plan_t *plans;
  const FrameBurst *bursts;
  const FramePair *pairs;
  int32_t *rows;  // crop rows [2 * n_bursts]: first, last (exclusive)
  int32_t n_bursts, n_pairs;
  int64_t n_deramp_tiles, n_geo_tiles;
  int32_t rowlook, collook, n_win;
  float alpha;
  uint64_t fill_seed;
  int32_t max_nrow_ml, max_ncol_ml, max_patches;
  int32_t deramp_rows, geo_cols;  // tile shapes the launches use
  int32_t deramp_tiles_x, deramp_tiles_y;  // deramp tiles of the largest burst, per axis
  int32_t geo_tiles_x, geo_tiles_y;        // geocoding tiles of the largest window, per axis
  int32_t sample_format;                   // S1B_SAMPLES_C64 or S1B_SAMPLES_CI16
  int32_t fused_deramp;                    // 1: geocoding deramps its gathers (column tables only)
  int32_t cull_geo;                        // 1: geocoding culls blocks outside the valid lines (set per launch)
  int32_t fused_xmul;                      // 1: geocoding forms the crossmul look-row sums (no geocoded windows)
  int32_t xm_tiles_x, xm_tiles_y;          // fused geocoding + crossmul tiles of the largest pair, per axis
};

// Run-time buffers of one frame launch sequence.
struct FrameIO {
  const void *slc;  // complex64 or complex int16 samples (FrameDev::sample_format)
  const int16_t *dem;
  int64_t dem_pitch;
  float2 *work;  // workspace viewed as complex64
  float2 *ifg;
  float *amp1, *amp2, *coh;
  float2 *filt;
  s1b_frame_pair_t *pout;
};

// Bursts of a frame by deramp load width: rows that start on 16 bytes (even
// samples, aligned burst) take 16-byte loads.  Host side, per launch.
struct FrameDerampSplit {
  std::vector<int32_t> vec, scalar;
};

// A list of burst indices passed to a kernel by value.
constexpr int kFrameListMax = 240;
struct FrameBurstList {
  int32_t n;
  int32_t idx[kFrameListMax];
};

// Tile-space helpers shared by host and device.
constexpr int kFrameDerampCols = 512;  // columns of a deramp tile (256 threads x 2)
constexpr int kFrameGeoRows = 128;     // rows of a geocoding tile (column walk length)
constexpr int kFrameXmCols = 128;      // columns of a geocoding + crossmul tile

// Launchers (k_geo2rdr.cu, k_crossmul.cu, k_goldstein.cu).  `ctas` is the
// persistent grid; 0 launches one CTA per tile over (tile x, tile y, burst).
int frame_launch_init(const FrameDev &d, const FrameIO &io, cudaStream_t st);
int frame_launch_deramp(const FrameDev &d, const FrameIO &io, int rows_per_tile, int ctas,
                        const FrameDerampSplit &split, cudaStream_t st);
int frame_launch_geo2rdr(const FrameDev &d, const FrameIO &io, int cols_per_tile, int ctas, cudaStream_t st);
int frame_max_ctas_deramp(int rows_per_tile);
int frame_max_ctas_geo2rdr(const FrameDev &d, int cols_per_tile);
int frame_launch_box(const FrameDev &d, const FrameIO &io, cudaStream_t st);
int frame_launch_crossmul(const FrameDev &d, const FrameIO &io, cudaStream_t st);
int frame_launch_goldstein(const FrameDev &d, const FrameIO &io, cudaStream_t st);
int frame_goldstein_patch_grid(int nrow, int ncol, int *ni, int *nj);

#endif

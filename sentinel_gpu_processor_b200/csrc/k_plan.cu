// Burst geometry prep on the GPU: footprint, DEM window and TOPS centre
// coefficients of many bursts in one launch (s1b_burst_geometry), with the
// functions of the host planner (s1b_geom.h).  The reference computes these
// on the host per burst (csrc/src/bounds.cu:237-317, geo2rdr.cu:387-400,
// 469-542, 569-586).  This file is compiled without FMA contraction
// (-fmad=false), so its FP64 arithmetic rounds operation by operation as the
// host planner's does; the transcendental functions are CUDA's.
#include <cuda_runtime.h>

#include "s1b.h"
#include "s1b_device.cuh"
#include "s1b_geom.h"
#include "s1b_internal.h"

namespace {

__global__ void burst_geometry_kernel(const s1b_orbit_poly_t *__restrict__ orbits, int32_t n_orbits,
                                      const double *__restrict__ tables, const int32_t *__restrict__ table_records,
                                      int32_t n_tables, int32_t max_records,
                                      const s1b_burst_geometry_in_t *__restrict__ in, int32_t n, s1b_rsc_t rsc,
                                      int32_t has_rsc, s1b_burst_geometry_t *__restrict__ out) {
  using namespace s1b_geom;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const s1b_burst_geometry_in_t b = in[i];
  s1b_burst_geometry_t o = {};
  o.status = 1;
  if (b.orbit >= 0 && b.orbit < n_orbits && b.fm_table >= 0 && b.fm_table < n_tables && b.dc_table >= 0 &&
      b.dc_table < n_tables && b.lines >= 2 && b.samples >= 2 && b.prf > 0 && b.range_sampling_rate > 0) {
    const s1b_orbit_poly_t &orb = orbits[b.orbit];
    const double dtaz = 1. / b.prf;                            // geo2rdr.cu:591
    const double tend = b.tstart + (b.lines - 1) * dtaz;       // 592
    const double rngstart = b.slant_range_time * kSol / 2.0;   // 594
    const double dmrg = kSol / 2.0 / b.range_sampling_rate;    // 595
    const double rngend = rngstart + (b.samples - 1) * dmrg;
    footprint(orb, b.tstart, tend, rngstart, rngend, b.hmin, b.hmax, o.latlon_box);
    // packed records (time, t0, c0, c1, c2); counts clamped to the array
    auto view = [&](int t) {
      const double *r = tables + (size_t)t * max_records * 5;
      int nr = table_records[t];
      nr = nr < 1 ? 1 : (nr > max_records ? max_records : nr);
      return PolyView{nr, 5, r, r + 1, r + 2, r + 3, r + 4};
    };
    tops_centre(orb, view(b.fm_table), view(b.dc_table), b.tstart + b.lines * b.azimuth_time_interval / 2,
                b.radar_frequency, b.azimuth_steering_rate, b.slant_range_time, &o.ks, o.fm, o.dc, &o.etac0);
    if (has_rsc) dem_window(o.latlon_box, rsc, o.win);
    o.status = 0;
  }
  out[i] = o;
}

}  // namespace

extern "C" int s1b_burst_geometry(const s1b_orbit_poly_t *orbits, int32_t n_orbits, const double *tables,
                                  const int32_t *table_records, int32_t n_tables, int32_t max_records,
                                  const s1b_burst_geometry_in_t *bursts, int32_t n, const s1b_rsc_t *rsc,
                                  s1b_burst_geometry_t *out, void *stream) {
  if (n < 0 || (n > 0 && (!orbits || !tables || !table_records || !bursts || !out)))
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_burst_geometry: null argument");
  if (n_orbits < 1 || n_tables < 1 || max_records < 1)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_burst_geometry: no orbits or tables");
  if (n == 0) return S1B_OK;
  const s1b_rsc_t r = rsc ? *rsc : s1b_rsc_t{};
  burst_geometry_kernel<<<(n + 63) / 64, 64, 0, (cudaStream_t)stream>>>(
      orbits, n_orbits, tables, table_records, n_tables, max_records, bursts, n, r, rsc ? 1 : 0, out);
  return s1b_launch_status();
}

// Host-side planning for one burst: orbit polynomials, footprint bounds,
// TOPS coefficients, DEM window, crossmul box.  Everything here is what the
// reference geo2rdr / crossmul_daemon executables compute on the CPU before
// launching kernels; the formulas are kept so results agree with them.
#include <cmath>
#include <cstring>

#include "s1b.h"
#include "s1b_geom.h"
#include "s1b_internal.h"

namespace {

using namespace s1b_geom;

// Confluent divided differences of the 4-point Hermite data in the
// normalised time s = (t - tc) / h, converted to monomial coefficients in
// (t - tc).  The interpolant is the unique degree-7 polynomial matching the
// four positions and velocities, which is what orbithermite evaluates in
// Lagrange form.
void window_poly(const double *t4, const double *x4, const double *v4, double tc, double h,
                 double out[3][8]) {
  long double z[8];
  for (int i = 0; i < 4; ++i) z[2 * i] = z[2 * i + 1] = ((long double)t4[i] - tc) / h;
  for (int comp = 0; comp < 3; ++comp) {
    long double q[8][8] = {};
    for (int i = 0; i < 4; ++i) q[2 * i][0] = q[2 * i + 1][0] = x4[3 * i + comp];
    for (int j = 1; j < 8; ++j) {
      for (int i = j; i < 8; ++i) {
        if (j == 1 && (i & 1))
          q[i][1] = (long double)v4[3 * (i / 2) + comp] * h;
        else
          q[i][j] = (q[i][j - 1] - q[i - 1][j - 1]) / (z[i] - z[i - j]);
      }
    }
    long double poly[8] = {}, basis[8] = {1.0L};
    for (int k = 0; k < 8; ++k) {
      for (int m = 0; m < 8; ++m) poly[m] += q[k][k] * basis[m];
      long double nb[8] = {};
      for (int m = 0; m < 8; ++m) {
        if (m > 0) nb[m] += basis[m - 1];
        nb[m] -= z[k] * basis[m];
      }
      std::memcpy(basis, nb, sizeof(basis));
    }
    long double scale = 1.0L;
    for (int k = 0; k < 8; ++k) {
      out[comp][k] = (double)(poly[k] / scale);
      scale *= h;
    }
  }
}

void eval_host(const s1b_orbit_poly_t &p, double t, double x[3], double v[3], double a[3]) {
  eval_poly(p, t, x, v, a);
}

PolyView view(const s1b_poly_table_t *tab) { return PolyView{tab->n, 1, tab->time, tab->t0, tab->c0, tab->c1, tab->c2}; }

}  // namespace

extern "C" int s1b_orbit_poly(const s1b_orbit_t *orbit, s1b_orbit_poly_t *poly) {
  if (!orbit || !poly || !orbit->t || !orbit->x || !orbit->v) return S1B_ERR_INVALID_ARGUMENT;
  const int n = orbit->n;
  if (n < 4) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "orbit needs at least 4 state vectors");
  if (n > S1B_MAX_STATE_VECTORS)
    return s1b_fail(S1B_ERR_TOO_LARGE, "orbit has more than S1B_MAX_STATE_VECTORS state vectors");
  const double dt = orbit->t[1] - orbit->t[0];
  if (!(dt > 0)) return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "orbit times must increase");
  std::memset(poly, 0, sizeof(*poly));
  poly->n_state = n;
  poly->n_win = n - 3;
  poly->t0 = orbit->t[0];
  poly->inv_dt = 1.0 / dt;
  for (int w = 1; w <= n - 3; ++w) {
    const double *t4 = orbit->t + (w - 1);
    const double tc = 0.5 * (t4[1] + t4[2]);
    const double h = (t4[3] - t4[0]) / 3.0;
    poly->tc[w - 1] = tc;
    window_poly(t4, orbit->x + 3 * (w - 1), orbit->v + 3 * (w - 1), tc, h, poly->c[w - 1]);
  }
  return S1B_OK;
}

extern "C" int s1b_orbit_eval_host(const s1b_orbit_poly_t *orbit, const double *t, int64_t n,
                                   double *satx, double *satv) {
  if (!orbit || (n > 0 && (!t || !satx || !satv))) return S1B_ERR_INVALID_ARGUMENT;
  for (int64_t i = 0; i < n; ++i) eval_host(*orbit, t[i], satx + 3 * i, satv + 3 * i, nullptr);
  return S1B_OK;
}

extern "C" int s1b_bounds(const s1b_orbit_poly_t *orb, double start_time, double end_time,
                          double start_rng, double end_rng, double hmin, double hmax,
                          double latlons[4]) {
  if (!orb || !latlons) return S1B_ERR_INVALID_ARGUMENT;
  footprint(*orb, start_time, end_time, start_rng, end_rng, hmin, hmax, latlons);
  return S1B_OK;
}

extern "C" int s1b_burst_plan(const s1b_radar_t *radar, const s1b_orbit_t *orbit,
                              const s1b_poly_table_t *fm, const s1b_poly_table_t *dc,
                              const s1b_burst_t *burst, const s1b_rsc_t *rsc,
                              s1b_burst_plan_t *plan) {
  if (!radar || !orbit || !fm || !dc || !burst || !plan)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "s1b_burst_plan: null argument");
  if (fm->n < 1 || dc->n < 1)
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "empty FM-rate or Doppler table");
  if (radar->lines_per_burst < 2 || radar->samples_per_burst < 2 || !(radar->prf > 0) ||
      !(radar->range_sampling_rate > 0) || !(radar->wvl > 0))
    return s1b_fail(S1B_ERR_INVALID_ARGUMENT, "invalid radar parameters");
  int st = s1b_orbit_poly(orbit, &plan->orbit);
  if (st != S1B_OK) return st;
  s1b_burst_plan_t &p = *plan;
  const int L = radar->lines_per_burst, S = radar->samples_per_burst;
  p.lines = L;
  p.samples = S;
  p.first_valid_line = burst->first_valid_line;
  p.last_valid_line = burst->last_valid_line;
  p.first_valid_sample = burst->first_valid_sample;
  p.last_valid_sample = burst->last_valid_sample;
  p.ati = radar->azimuth_time_interval;
  p.tstart = burst->azimuth_time;
  p.dtaz = 1. / radar->prf;                                  // geo2rdr.cu:591
  const double tend = p.tstart + (L - 1) * p.dtaz;           // 592
  p.tmid = (p.tstart + tend) * 0.5;                          // 593
  p.rngstart = radar->slant_range_time * kSol / 2.0;         // 594
  p.dmrg = kSol / 2.0 / radar->range_sampling_rate;          // 595
  p.slant_range_time = radar->slant_range_time;
  p.range_sampling_rate = radar->range_sampling_rate;
  p.wvl = radar->wvl;
  p.k4pi_wvl = 4.0 * kPi / radar->wvl;
  eval_host(p.orbit, p.tmid, p.xmid, p.vmid, p.amid);
  // TOPS steering ks, FM-rate and Doppler at the burst centre, etac at the
  // first range sample (geo2rdr.cu:477-541)
  tops_centre(p.orbit, view(fm), view(dc), p.tstart + L * p.ati / 2, radar->radar_frequency,
              radar->azimuth_steering_rate, radar->slant_range_time, &p.ks, p.fm, p.dc, &p.etac0);
  // Footprint and DEM window (geo2rdr.cu:387-400, 569-586).
  const double rngend = p.rngstart + (S - 1) * p.dmrg;
  st = s1b_bounds(&p.orbit, p.tstart, tend, p.rngstart, rngend, radar->hmin, radar->hmax,
                  p.latlon_box);
  if (st != S1B_OK) return st;
  p.win_left = p.win_top = p.win_right = p.win_bottom = 0;
  p.rsc_nlat = p.rsc_nlon = 0;
  p.lat0 = p.lon0 = p.dlat = p.dlon = 0.0;
  if (!rsc) return S1B_OK;
  int32_t win[4];
  dem_window(p.latlon_box, *rsc, win);
  const int left = win[0], top = win[1], right = win[2], bottom = win[3];
  p.win_left = left;
  p.win_top = top;
  p.win_right = right;
  p.win_bottom = bottom;
  p.rsc_nlat = rsc->nlat;
  p.rsc_nlon = rsc->nlon;
  p.dlat = rsc->dlat;
  p.dlon = rsc->dlon;
  p.lat0 = rsc->latmax + rsc->dlat * top;   // geo2rdr.cu:611
  p.lon0 = rsc->lonmin + rsc->dlon * left;  // geo2rdr.cu:612
  if (left >= right || top >= bottom) return S1B_ERR_EMPTY;
  return S1B_OK;
}

extern "C" int s1b_crossmul_box(const int32_t *h1, const int32_t *h2, int32_t rowlook,
                                int32_t collook, int32_t use_union, int32_t *box,
                                int32_t *hdr) {
  if (!h1 || !h2 || !box || rowlook < 1 || collook < 1) return S1B_ERR_INVALID_ARGUMENT;
  int left, right, top, bottom;
  if (!use_union) {  // crossmul_daemon.cu:612-620
    left = h1[2] > h2[2] ? h1[2] : h2[2];
    right = h1[4] < h2[4] ? h1[4] : h2[4];
    top = h1[3] > h2[3] ? h1[3] : h2[3];
    bottom = h1[5] < h2[5] ? h1[5] : h2[5];
  } else {  // crossmul.cu:191-198
    left = h1[2] < h2[2] ? h1[2] : h2[2];
    right = h1[4] > h2[4] ? h1[4] : h2[4];
    top = h1[3] < h2[3] ? h1[3] : h2[3];
    bottom = h1[5] > h2[5] ? h1[5] : h2[5];
  }
  left = (left + collook - 1) / collook * collook;
  right = right / collook * collook;
  top = (top + rowlook - 1) / rowlook * rowlook;
  bottom = bottom / rowlook * rowlook;
  box[0] = left;
  box[1] = top;
  box[2] = right;
  box[3] = bottom;
  if (hdr) {  // crossmul_daemon.cu:660-666
    hdr[0] = h1[0] / rowlook;
    hdr[1] = h1[1] / collook;
    hdr[2] = left / collook;
    hdr[3] = top / rowlook;
    hdr[4] = right / collook;
    hdr[5] = bottom / rowlook;
  }
  const bool empty = use_union ? ((bottom - top) / rowlook == 0 || (right - left) / collook == 0)
                               : (bottom - top <= 0 || right - left <= 0);
  return empty ? S1B_ERR_EMPTY : S1B_OK;
}

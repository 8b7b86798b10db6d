// Host-side planning for one burst: orbit polynomials, footprint bounds,
// TOPS coefficients, DEM window, crossmul box.  Everything here is what the
// reference geo2rdr / crossmul_daemon executables compute on the CPU before
// launching kernels; the formulas are kept so results agree with them.
#include <cmath>
#include <cstring>

#include "s1b.h"
#include "s1b_internal.h"

namespace {

constexpr double kRa = 6378137.0;           // WGS84 semi-major axis, orbit.hpp:7
constexpr double kRe2 = 0.00669437999015;   // WGS84 e^2, orbit.hpp:10
constexpr double kSol = 299792458.0;        // geo2rdr.cu:27
constexpr double kPi = 3.14159265358979323846;

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 unit(V3 a) {
  double n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x / n, a.y / n, a.z / n};
}

// ECEF -> geodetic by the single Bowring step the reference uses
// (orbit.cu:37-70); the DEM window depends on it through int() truncation.
V3 ecef_to_llh(V3 p) {
  const double q2 = 1.0 / (1.0 - kRe2);
  const double q = std::sqrt(q2);
  const double q3 = q2 - 1.0;
  const double b = kRa * std::sqrt(1 - kRe2);
  double lon = std::atan2(p.y, p.x);
  if (p.y < 0 && lon > 0) lon -= kPi;
  if (p.y > 0 && lon < 0) lon += kPi;
  const double rp = std::sqrt(p.x * p.x + p.y * p.y);
  const double theta = std::atan((p.z / rp) * q);
  const double tant = (p.z + q3 * b * std::pow(std::sin(theta), 3)) /
                      (rp - kRe2 * kRa * std::pow(std::cos(theta), 3));
  const double lat = std::atan(tant);
  const double re = kRa / std::sqrt(1.0 - kRe2 * std::sin(lat) * std::sin(lat));
  const double h = rp / std::cos(lat) - re;
  return {lat / kPi * 180, lon / kPi * 180, h};
}

// Geodesic heading from (lat1, lon1) to (lat2, lon2) on the ellipsoid by
// Sodano's non-iterative inverse solution, the method of bounds.cu:112-199.
double geodesic_heading(double lat1, double lon1, double lat2, double lon2) {
  const double e = std::sqrt(kRe2);
  const double sq = std::sqrt(1.0 - kRe2);
  const double f = 1.0 - sq;
  const double ep = e * f / (kRe2 - f);
  const double n = f / kRe2;
  const double base = 16.0 * kRe2 * n * n;
  const double k1 = (base + ep * ep) / (ep * ep);
  const double k2 = base / (base + ep * ep);
  const double k3 = base / (ep * ep);
  const double k4 = (16.0 * n - ep * ep) / (base + ep * ep);
  const double k5 = 16.0 / (kRe2 * (base + ep * ep));
  const double d2r = kPi / 180.0;
  const double tan1 = std::tan(lat1 * d2r), tan2 = std::tan(lat2 * d2r);
  const double dl = std::fabs(lon2 * d2r - lon1 * d2r);
  const double dl_signed = lon2 * d2r - lon1 * d2r;
  double slon = std::sin(dl);
  const double clon = std::cos(dl);
  const double tb1 = sq * tan1, tb2 = sq * tan2;
  const double cb1 = 1.0 / std::sqrt(1.0 + tb1 * tb1);
  const double cb2 = 1.0 / std::sqrt(1.0 + tb2 * tb2);
  const double sb1 = tb1 * cb1, sb2 = tb2 * cb2;
  const double ac = sb1 * sb2, bc = cb1 * cb2;
  const double cphi = ac + bc * clon;
  const double sgn = (slon > 0) - (slon < 0);
  const double sphi = sgn * std::sqrt(1.0 - std::fmin(cphi * cphi, 1.0));
  const double phi = std::fabs(std::atan2(sphi, cphi));
  if (!(kRa * std::fabs(phi) > 1e-6)) return 0.0;
  const double ca = (bc * slon) / sphi;
  const double cb = ca * ca;
  const double cc = (cphi * (1.0 - cb)) / k1;
  const double cd = (-2.0 * ac) / k1;
  const double ce = -ac * k2;
  const double cf = k3 * cc;
  const double cg = phi * phi / sphi;
  const double x = ((phi * (k4 + cb) + sphi * (cc + cd) + cg * (cf + ce)) * ca) / k5;
  const double lam = dl + x;
  const double t2 = tb2 * cb1 - std::cos(lam) * sb1;
  const double s = (dl_signed > 0) - (dl_signed < 0);
  slon = std::sin(lam) * s;
  return std::atan2(slon, t2);
}

// Radius of curvature along heading `hdg` at geodetic latitude `lat` (rad):
// bounds.cu:33-45.
double radius_along(double lat, double hdg) {
  const double s2 = std::pow(std::sin(lat), 2);
  const double re = kRa / std::sqrt(1.0 - kRe2 * s2);
  const double rn = kRa * (1.0 - kRe2) / std::pow(1.0 - kRe2 * s2, 1.5);
  return (re * rn) / (re * std::pow(std::cos(hdg), 2) + rn * std::pow(std::sin(hdg), 2));
}

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
  int w = s1b_orbit_window(p, t);
  const double tau = t - p.tc[w - 1];
  for (int comp = 0; comp < 3; ++comp) {
    const double *c = p.c[w - 1][comp];
    double f = c[7], d = 0.0, dd = 0.0;
    for (int k = 6; k >= 0; --k) {
      dd = dd * tau + d;
      d = d * tau + f;
      f = f * tau + c[k];
    }
    x[comp] = f;
    v[comp] = d;
    if (a) a[comp] = 2.0 * dd;
  }
}

// Poly-table linear interpolation at time tc: geo2rdr.cu:485-527 (the first
// record with the smallest |time - tc| anchors the interpolation).
void interp_table(const s1b_poly_table_t *tab, double tc, double out[4]) {
  const int n = tab->n;
  int idx = 0;
  double mind = 1e10;
  for (int i = 0; i < n; ++i) {
    double d = std::fabs(tab->time[i] - tc);
    if (mind > d) {
      mind = d;
      idx = i;
    }
  }
  const double *cols[4] = {tab->t0, tab->c0, tab->c1, tab->c2};
  if (tab->time[idx] < tc && idx < n - 1) {
    double f = (tc - tab->time[idx]) / (tab->time[idx + 1] - tab->time[idx]);
    for (int k = 0; k < 4; ++k) out[k] = cols[k][idx] + f * (cols[k][idx + 1] - cols[k][idx]);
  } else if (tab->time[idx] > tc && idx > 0) {
    double f = (tc - tab->time[idx - 1]) / (tab->time[idx] - tab->time[idx - 1]);
    for (int k = 0; k < 4; ++k) out[k] = cols[k][idx - 1] + f * (cols[k][idx] - cols[k][idx - 1]);
  } else {
    for (int k = 0; k < 4; ++k) out[k] = cols[k][idx];
  }
}

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
  // Heading of the ground track and the local radius of curvature along it
  // (bounds.cu:247-258), then each (range, time, height) corner placed by
  // the law of cosines in the TCN frame of the satellite (bounds.cu:260-284).
  double xs[3], vs_[3], xe[3], ve[3], xm[3], vm[3];
  eval_host(*orb, start_time, xs, vs_, nullptr);
  eval_host(*orb, end_time, xe, ve, nullptr);
  eval_host(*orb, (start_time + end_time) / 2., xm, vm, nullptr);
  V3 ls = ecef_to_llh({xs[0], xs[1], xs[2]});
  V3 le = ecef_to_llh({xe[0], xe[1], xe[2]});
  const double hdg = geodesic_heading(ls.x, ls.y, le.x, le.y);
  V3 lm = ecef_to_llh({xm[0], xm[1], xm[2]});
  const double rcurv = radius_along(lm.x * kPi / 180.0, hdg);
  double lat[8], lon[8];
  for (int i = 0; i < 8; ++i) {
    const double r = i < 4 ? start_rng : end_rng;
    const double t = (i % 4 < 2) ? start_time : end_time;
    const double h = (i % 2 == 0) ? hmin : hmax;
    double x[3], v[3];
    eval_host(*orb, t, x, v, nullptr);
    const V3 pos{x[0], x[1], x[2]}, vel{v[0], v[1], v[2]};
    const V3 llh = ecef_to_llh(pos);
    const V3 vhat = unit(vel);
    const V3 sat_llh = ecef_to_llh(pos);
    const double la = sat_llh.x * kPi / 180.0, lo = sat_llh.y * kPi / 180.0;
    const V3 nhat{-std::cos(la) * std::cos(lo), -std::cos(la) * std::sin(lo), -std::sin(la)};
    const V3 chat = unit(cross(nhat, vel));  // right-looking
    const V3 that = unit(cross(chat, nhat));
    const double aa = rcurv + llh.z;
    const double bb = rcurv + h;
    const double cost = 0.5 * ((aa / r + r / aa - bb / aa * bb / r));
    const double sint = std::sqrt(1. - cost * cost);
    const double gamm = cost * r;
    const double alpha = (0.0 * r - gamm * dot(nhat, vhat)) / dot(vhat, that);
    const double beta = std::sqrt((r * sint) * (r * sint) - alpha * alpha);
    const V3 tgt = pos + (gamm * nhat + alpha * that + beta * chat);
    const V3 g = ecef_to_llh(tgt);
    lat[i] = g.x;
    lon[i] = g.y;
  }
  double mn[2] = {lat[0], lon[0]}, mx[2] = {lat[0], lon[0]};
  for (int i = 1; i < 8; ++i) {
    if (mn[0] > lat[i]) mn[0] = lat[i];
    if (mx[0] < lat[i]) mx[0] = lat[i];
    if (mn[1] > lon[i]) mn[1] = lon[i];
    if (mx[1] < lon[i]) mx[1] = lon[i];
  }
  latlons[0] = mn[0];
  latlons[1] = mx[0];
  latlons[2] = mn[1];
  latlons[3] = mx[1];
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
  // TOPS steering: ks at the burst centre (geo2rdr.cu:477-483).
  const double tcen = p.tstart + L * p.ati / 2;
  double xc[3], vc[3];
  eval_host(p.orbit, tcen, xc, vc, nullptr);
  const double vs = std::sqrt(vc[0] * vc[0] + vc[1] * vc[1] + vc[2] * vc[2]);
  p.ks = 2.0 * vs * radar->radar_frequency / kSol * radar->azimuth_steering_rate * kPi / 180.0;
  interp_table(fm, tcen, p.fm);
  interp_table(dc, tcen, p.dc);
  {  // etac at the first range sample (geo2rdr.cu:533-541, i = 0)
    const double dt1 = radar->slant_range_time - p.fm[0];
    const double ka = p.fm[1] + dt1 * (p.fm[2] + p.fm[3] * dt1);
    const double dt2 = radar->slant_range_time - p.dc[0];
    const double fnc = p.dc[1] + dt2 * (p.dc[2] + p.dc[3] * dt2);
    p.etac0 = -fnc / ka;
  }
  // Footprint and DEM window (geo2rdr.cu:387-400, 569-586).
  const double rngend = p.rngstart + (S - 1) * p.dmrg;
  st = s1b_bounds(&p.orbit, p.tstart, tend, p.rngstart, rngend, radar->hmin, radar->hmax,
                  p.latlon_box);
  if (st != S1B_OK) return st;
  p.win_left = p.win_top = p.win_right = p.win_bottom = 0;
  p.rsc_nlat = p.rsc_nlon = 0;
  p.lat0 = p.lon0 = p.dlat = p.dlon = 0.0;
  if (!rsc) return S1B_OK;
  const double latmin = p.latlon_box[0], latmax = p.latlon_box[1];
  const double lonmin = p.latlon_box[2], lonmax = p.latlon_box[3];
  int left = (int)((lonmin - rsc->lonmin) / rsc->dlon);
  int top = (int)((latmax - rsc->latmax) / rsc->dlat);
  int right = (int)((lonmax - rsc->lonmin) / rsc->dlon + 1);
  int bottom = (int)((latmin - rsc->latmax) / rsc->dlat + 1);
  left = left > 0 ? left : 0;
  top = top > 0 ? top : 0;
  right = right < rsc->nlon ? right : rsc->nlon;
  bottom = bottom < rsc->nlat ? bottom : rsc->nlat;
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

// Burst geometry shared by the host planner (plan.cpp) and the device
// kernel of s1b_burst_geometry (k_plan.cu): orbit polynomial evaluation,
// the one-step ECEF -> geodetic conversion, the footprint of a burst from
// its corner geometry, the FM-rate / Doppler table interpolation at the
// burst centre and the DEM window.  What the reference computes on the host
// before its kernels run (csrc/src/bounds.cu:33-317, orbit.cu:37-70,
// geo2rdr.cu:387-400, 469-542, 569-586); the DEM window depends on these
// values through int() truncation, so the formulas and their order follow it.
#ifndef S1B_GEOM_H
#define S1B_GEOM_H

#include <math.h>

#include "s1b.h"
#include "s1b_internal.h"

namespace s1b_geom {

constexpr double kRa = 6378137.0;          // WGS84 semi-major axis, orbit.hpp:7
constexpr double kRe2 = 0.00669437999015;  // WGS84 e^2, orbit.hpp:10
constexpr double kSol = 299792458.0;       // geo2rdr.cu:27
constexpr double kPi = 3.14159265358979323846;

struct V3 {
  double x, y, z;
};
S1B_HD V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
S1B_HD V3 scale(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
S1B_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
S1B_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
S1B_HD V3 unit(V3 a) {
  const double n = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x / n, a.y / n, a.z / n};
}

// Orbit position, velocity and (optionally) acceleration at time t from the
// window polynomial (Horner's scheme carrying two derivatives).
S1B_HD void eval_poly(const s1b_orbit_poly_t &p, double t, double x[3], double v[3], double a[3]) {
  const int w = s1b_orbit_window(p, t);
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

// ECEF -> geodetic by the single Bowring step the reference uses
// (orbit.cu:37-70).  Returns (lat deg, lon deg, h m).
S1B_HD V3 ecef_to_llh(V3 p) {
  const double q2 = 1.0 / (1.0 - kRe2);
  const double q = sqrt(q2);
  const double q3 = q2 - 1.0;
  const double b = kRa * sqrt(1 - kRe2);
  double lon = atan2(p.y, p.x);
  if (p.y < 0 && lon > 0) lon -= kPi;
  if (p.y > 0 && lon < 0) lon += kPi;
  const double rp = sqrt(p.x * p.x + p.y * p.y);
  const double theta = atan((p.z / rp) * q);
  const double tant = (p.z + q3 * b * pow(sin(theta), 3)) / (rp - kRe2 * kRa * pow(cos(theta), 3));
  const double lat = atan(tant);
  const double re = kRa / sqrt(1.0 - kRe2 * sin(lat) * sin(lat));
  const double h = rp / cos(lat) - re;
  return {lat / kPi * 180, lon / kPi * 180, h};
}

// Geodesic heading from (lat1, lon1) to (lat2, lon2) on the ellipsoid by
// Sodano's non-iterative inverse solution, the method of bounds.cu:112-199.
S1B_HD double geodesic_heading(double lat1, double lon1, double lat2, double lon2) {
  const double e = sqrt(kRe2);
  const double sq = sqrt(1.0 - kRe2);
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
  const double tan1 = tan(lat1 * d2r), tan2 = tan(lat2 * d2r);
  const double dl = fabs(lon2 * d2r - lon1 * d2r);
  const double dl_signed = lon2 * d2r - lon1 * d2r;
  double slon = sin(dl);
  const double clon = cos(dl);
  const double tb1 = sq * tan1, tb2 = sq * tan2;
  const double cb1 = 1.0 / sqrt(1.0 + tb1 * tb1);
  const double cb2 = 1.0 / sqrt(1.0 + tb2 * tb2);
  const double sb1 = tb1 * cb1, sb2 = tb2 * cb2;
  const double ac = sb1 * sb2, bc = cb1 * cb2;
  const double cphi = ac + bc * clon;
  const double sgn = (slon > 0) - (slon < 0);
  const double sphi = sgn * sqrt(1.0 - fmin(cphi * cphi, 1.0));
  const double phi = fabs(atan2(sphi, cphi));
  if (!(kRa * fabs(phi) > 1e-6)) return 0.0;
  const double ca = (bc * slon) / sphi;
  const double cb = ca * ca;
  const double cc = (cphi * (1.0 - cb)) / k1;
  const double cd = (-2.0 * ac) / k1;
  const double ce = -ac * k2;
  const double cf = k3 * cc;
  const double cg = phi * phi / sphi;
  const double x = ((phi * (k4 + cb) + sphi * (cc + cd) + cg * (cf + ce)) * ca) / k5;
  const double lam = dl + x;
  const double t2 = tb2 * cb1 - cos(lam) * sb1;
  const double s = (dl_signed > 0) - (dl_signed < 0);
  slon = sin(lam) * s;
  return atan2(slon, t2);
}

// Radius of curvature along heading `hdg` at geodetic latitude `lat` (rad):
// bounds.cu:33-45.
S1B_HD double radius_along(double lat, double hdg) {
  const double s2 = pow(sin(lat), 2);
  const double re = kRa / sqrt(1.0 - kRe2 * s2);
  const double rn = kRa * (1.0 - kRe2) / pow(1.0 - kRe2 * s2, 1.5);
  return (re * rn) / (re * pow(cos(hdg), 2) + rn * pow(sin(hdg), 2));
}

// Footprint [latmin, latmax, lonmin, lonmax] of a burst at heights
// hmin..hmax (bounds.cu:237-317): the heading of the ground track and the
// local radius of curvature along it (247-258), then each (range, time,
// height) corner placed by the law of cosines in the satellite's TCN frame
// (260-284), right-looking.
S1B_HD void footprint(const s1b_orbit_poly_t &orb, double start_time, double end_time, double start_rng,
                      double end_rng, double hmin, double hmax, double latlons[4]) {
  double xs[3], vs_[3], xe[3], ve[3], xm[3], vm[3];
  eval_poly(orb, start_time, xs, vs_, nullptr);
  eval_poly(orb, end_time, xe, ve, nullptr);
  eval_poly(orb, (start_time + end_time) / 2., xm, vm, nullptr);
  const V3 ls = ecef_to_llh({xs[0], xs[1], xs[2]});
  const V3 le = ecef_to_llh({xe[0], xe[1], xe[2]});
  const double hdg = geodesic_heading(ls.x, ls.y, le.x, le.y);
  const V3 lm = ecef_to_llh({xm[0], xm[1], xm[2]});
  const double rcurv = radius_along(lm.x * kPi / 180.0, hdg);
  double lat[8], lon[8];
  for (int i = 0; i < 8; ++i) {
    const double r = i < 4 ? start_rng : end_rng;
    const double t = (i % 4 < 2) ? start_time : end_time;
    const double h = (i % 2 == 0) ? hmin : hmax;
    double x[3], v[3];
    eval_poly(orb, t, x, v, nullptr);
    const V3 pos{x[0], x[1], x[2]}, vel{v[0], v[1], v[2]};
    const V3 llh = ecef_to_llh(pos);
    const V3 vhat = unit(vel);
    const V3 sat_llh = ecef_to_llh(pos);
    const double la = sat_llh.x * kPi / 180.0, lo = sat_llh.y * kPi / 180.0;
    const V3 nhat{-cos(la) * cos(lo), -cos(la) * sin(lo), -sin(la)};
    const V3 chat = unit(cross(nhat, vel));  // right-looking
    const V3 that = unit(cross(chat, nhat));
    const double aa = rcurv + llh.z;
    const double bb = rcurv + h;
    const double cost = 0.5 * ((aa / r + r / aa - bb / aa * bb / r));
    const double sint = sqrt(1. - cost * cost);
    const double gamm = cost * r;
    const double alpha = (0.0 * r - gamm * dot(nhat, vhat)) / dot(vhat, that);
    const double beta = sqrt((r * sint) * (r * sint) - alpha * alpha);
    const V3 tgt = add(pos, add(add(scale(gamm, nhat), scale(alpha, that)), scale(beta, chat)));
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
}

// Records of an FM-rate or Doppler table: record i has time, t0, c0, c1, c2
// at time[i * stride] ... c2[i * stride] (separate arrays: stride 1; packed
// 5-double records: stride 5).
struct PolyView {
  int n, stride;
  const double *time, *t0, *c0, *c1, *c2;
};

// Linear interpolation of the table at time tc: geo2rdr.cu:485-527 (the
// first record with the smallest |time - tc| anchors the interpolation).
S1B_HD void interp_table(const PolyView &tab, double tc, double out[4]) {
  const int n = tab.n, st = tab.stride;
  int idx = 0;
  double mind = 1e10;
  for (int i = 0; i < n; ++i) {
    const double d = fabs(tab.time[i * st] - tc);
    if (mind > d) {
      mind = d;
      idx = i;
    }
  }
  const double *cols[4] = {tab.t0, tab.c0, tab.c1, tab.c2};
  const double ti = tab.time[idx * st];
  if (ti < tc && idx < n - 1) {
    const double f = (tc - ti) / (tab.time[(idx + 1) * st] - ti);
    for (int k = 0; k < 4; ++k) out[k] = cols[k][idx * st] + f * (cols[k][(idx + 1) * st] - cols[k][idx * st]);
  } else if (ti > tc && idx > 0) {
    const double tp = tab.time[(idx - 1) * st];
    const double f = (tc - tp) / (ti - tp);
    for (int k = 0; k < 4; ++k) out[k] = cols[k][(idx - 1) * st] + f * (cols[k][idx * st] - cols[k][(idx - 1) * st]);
  } else {
    for (int k = 0; k < 4; ++k) out[k] = cols[k][idx * st];
  }
}

// TOPS quantities at the burst centre tc (geo2rdr.cu:477-541): the steering
// ks = 2 |V(tc)| f0 / c * psi_dot * pi / 180, the interpolated FM-rate and
// Doppler polynomials, and etac at the first range sample.
S1B_HD void tops_centre(const s1b_orbit_poly_t &orb, const PolyView &fm_tab, const PolyView &dc_tab, double tc,
                        double radar_frequency, double steering_rate, double slant_range_time, double *ks,
                        double fm[4], double dc[4], double *etac0) {
  double xc[3], vc[3];
  eval_poly(orb, tc, xc, vc, nullptr);
  const double vs = sqrt(vc[0] * vc[0] + vc[1] * vc[1] + vc[2] * vc[2]);
  *ks = 2.0 * vs * radar_frequency / kSol * steering_rate * kPi / 180.0;
  interp_table(fm_tab, tc, fm);
  interp_table(dc_tab, tc, dc);
  const double dt1 = slant_range_time - fm[0];
  const double ka = fm[1] + dt1 * (fm[2] + fm[3] * dt1);
  const double dt2 = slant_range_time - dc[0];
  const double fnc = dc[1] + dt2 * (dc[2] + dc[3] * dt2);
  *etac0 = -fnc / ka;
}

// DEM window [left, right) x [top, bottom) of a footprint on the RSC grid:
// C int() truncation of each end, then clamped (geo2rdr.cu:569-586).
S1B_HD void dem_window(const double latlons[4], const s1b_rsc_t &rsc, int32_t win[4]) {
  int left = (int)((latlons[2] - rsc.lonmin) / rsc.dlon);
  int top = (int)((latlons[1] - rsc.latmax) / rsc.dlat);
  int right = (int)((latlons[3] - rsc.lonmin) / rsc.dlon + 1);
  int bottom = (int)((latlons[0] - rsc.latmax) / rsc.dlat + 1);
  win[0] = left > 0 ? left : 0;
  win[1] = top > 0 ? top : 0;
  win[2] = right < rsc.nlon ? right : rsc.nlon;
  win[3] = bottom < rsc.nlat ? bottom : rsc.nlat;
}

}  // namespace s1b_geom

#endif

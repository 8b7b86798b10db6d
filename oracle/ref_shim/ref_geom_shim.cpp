// extern "C" entry points over the reference's host/device geometry
// functions (csrc/src/orbit.cu, csrc/src/bounds.cu) compiled as plain host
// C++.  Test infrastructure only: oracle/build_ref.py links this file with
// the reference sources into oracle/_ref/libref_geom.so, which pins the
// float64 geometry oracle (oracle/geometry.py) to the reference itself.
#include <cstddef>
#include <string>
#include "orbit.hpp"
#include "bounds.hpp"

extern "C" {

void ref_llh2xyz(const double *llh, double *xyz, long n) {
  for (long i = 0; i < n; ++i) {
    double a[3] = {llh[3 * i], llh[3 * i + 1], llh[3 * i + 2]};
    llh2xyz(a, xyz + 3 * i);
  }
}

void ref_xyz2llh(const double *xyz, double *llh, long n) {
  for (long i = 0; i < n; ++i) {
    double a[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    xyz2llh(a, llh + 3 * i);
  }
}

void ref_intp_orbit(long nstatvec, double *tt, double *xx, double *vv,
                    const double *t, long n, double *satx, double *satv) {
  for (long i = 0; i < n; ++i)
    intp_orbit((std::size_t)nstatvec, tt, xx, vv, t[i], satx + 3 * i, satv + 3 * i);
}

void ref_orbitrangetime(long nstatvec, double *tt, double *xx, double *vv,
                        const double *xyz, long n, double tline0,
                        double *satx0, double *satv0, double *tline,
                        double *dr) {
  for (long i = 0; i < n; ++i) {
    double p[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    double tl = 0.0;
    orbitrangetime((std::size_t)nstatvec, tt, xx, vv, p, tline0, satx0, satv0,
                   tl, dr + 3 * i);
    tline[i] = tl;
  }
}

void ref_bounds(double start_time, double end_time, double start_rng,
                double end_rng, double hmin, double hmax, double *tt,
                double *xx, double *vv, long nstatvec, double *latlons) {
  bounds(start_time, end_time, start_rng, end_rng, hmin, hmax, tt, xx, vv,
         (std::size_t)nstatvec, latlons, std::string("RIGHT"));
}
}

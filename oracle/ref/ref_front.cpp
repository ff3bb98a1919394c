// ref_front.cpp -- builds the reference's master/slave burst matching into
// oracle/_ref/libref_front.so.  Test infrastructure: it produces reference
// outputs for the golden fixtures, nothing else links it.
//
// The build recipe extracts Func.cpp:1133-1746 verbatim into
// oracle/_ref/gen/func_geo.inc (carriage returns stripped): getLatitude,
// getLontitude, Locating, Geodetic2Geographic, getXyz, getVelocity,
// getAcceleration, xyz2aztime, polyval1d, getxyz, getxyzdot, eq_in, solve33,
// lp2xyz, lp2ell and ComputerBurstOverlap.  This file compiles them against
// minimal stand-ins for the reference's types (DataTypes.h) and the WGS84
// constants of its ellipsoid class (DataTypes.cpp:177-183).
// ComputerBurstOverlap ends without a return statement; the recipe adds
// `return true;` before its closing brace (g++ traps there otherwise), and
// only its output arguments are read.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

using namespace std;

#include "Constants.h"

// the reference pauses a console on errors; a test run has none
#define system(cmd) 0

struct S1PreciseOrbit {
  int NumPoints = 0;
  int NumCoeff = 0;
  double *orbitAzTime = nullptr;
  double *coef_x = nullptr, *coef_y = nullptr, *coef_z = nullptr;
};

struct SubSwathInfo {
  double firstLineTime = 0, lastLineTime = 0;
  double slrTimeToFirstPixel = 0, slrTimeToLastPixel = 0;
  double azimuthTimeInterval = 0, prf = 0, rangeSamplingRate = 0;
  int numOfBursts = 0, linesPerBurst = 0, samplesPerBurst = 0;
  double burstFirstLineTime[16] = {};
  int numOfGeoLines = 0, numOfGeoPointsPerLine = 0;
  double *azimuthTime = nullptr, *slantRangeTime = nullptr;
  double *latitude = nullptr, *longitude = nullptr;
};

struct SentinelTOPS {
  int NumSubSwath = 1;
  SubSwathInfo *SubSwath = nullptr;
};

class ellipsoid_WGS84 {
 public:
  double e2, e2b, a, b;
  ellipsoid_WGS84() {
    a = 6378137.0;
    b = 6356752.3142451794975639665996337;
    e2 = 1.0 - (b / a) * (b / a);
    e2b = e2 / (1 - e2);
  }
};

void Locating(SentinelTOPS &S1, double aztime, double rgtime, int SubSwathID, int *Index,
              double *coef);

#include "func_geo.inc"

// One image of the pair, as plain arrays (bursts, geolocation grid, orbit
// polynomial of its state vectors).
struct RefImage {
  int n_bursts, lines_per_burst, samples_per_burst;
  double dt, prf, rsr, slr_first, slr_last, first_line_time, last_line_time;
  const double *burst_first_line_time;
  int geo_lines, geo_points;
  const double *az_time, *slr_time, *lat, *lon;
  int n_points, n_coef;
  const double *orbit_t, *cx, *cy, *cz;
};

static void fill(const RefImage &r, SubSwathInfo &s, S1PreciseOrbit &o) {
  s.firstLineTime = r.first_line_time;
  s.lastLineTime = r.last_line_time;
  s.slrTimeToFirstPixel = r.slr_first;
  s.slrTimeToLastPixel = r.slr_last;
  s.azimuthTimeInterval = r.dt;
  s.prf = r.prf;
  s.rangeSamplingRate = r.rsr;
  s.numOfBursts = r.n_bursts;
  s.linesPerBurst = r.lines_per_burst;
  s.samplesPerBurst = r.samples_per_burst;
  for (int b = 0; b < r.n_bursts && b < 16; b++) s.burstFirstLineTime[b] = r.burst_first_line_time[b];
  s.numOfGeoLines = r.geo_lines;
  s.numOfGeoPointsPerLine = r.geo_points;
  s.azimuthTime = const_cast<double *>(r.az_time);
  s.slantRangeTime = const_cast<double *>(r.slr_time);
  s.latitude = const_cast<double *>(r.lat);
  s.longitude = const_cast<double *>(r.lon);
  o.NumPoints = r.n_points;
  o.NumCoeff = r.n_coef;
  o.orbitAzTime = const_cast<double *>(r.orbit_t);
  o.coef_x = const_cast<double *>(r.cx);
  o.coef_y = const_cast<double *>(r.cy);
  o.coef_z = const_cast<double *>(r.cz);
}

extern "C" {

// ComputerBurstOverlap on one sub-swath; out[4] = M_burst0, M_burstN,
// S_burst0, S_burstN (left at -1 where the reference sets nothing).
void ref_burst_overlap(int burst0, int burstN, const RefImage *m, const RefImage *s, int *out) {
  SubSwathInfo ms, ss;
  S1PreciseOrbit mo, so;
  fill(*m, ms, mo);
  fill(*s, ss, so);
  SentinelTOPS M, S;
  M.SubSwath = &ms;
  S.SubSwath = &ss;
  out[0] = out[1] = out[2] = out[3] = -1;
  ComputerBurstOverlap(burst0, burstN, out[0], out[1], out[2], out[3], M, S, 1, mo, so);
}

// lp2ell of 1-based (line, pixel) of one burst, from xyz (in/out).
long ref_lp2ell(double line, double pixel, const RefImage *im, int burst, double *xyz) {
  SubSwathInfo s;
  S1PreciseOrbit o;
  fill(*im, s, o);
  ellipsoid_WGS84 ell;
  return lp2ell(line, pixel, ell, s, burst, o, xyz);
}

// xyz2aztime on an image's orbit from t0 (the reference passes the middle
// orbit time, an int parameter).
double ref_xyz2aztime(const double *xyz, const RefImage *im, double t0) {
  double p[3] = {xyz[0], xyz[1], xyz[2]};
  return xyz2aztime(p, im->n_coef, const_cast<double *>(im->cx), const_cast<double *>(im->cy),
                    const_cast<double *>(im->cz), t0, im->orbit_t[im->n_points / 2]);
}

// getLatitude / getLontitude on an image's geolocation grid.
void ref_grid_latlon(const RefImage *im, double aztime, double rgtime, double *latlon) {
  SubSwathInfo s;
  S1PreciseOrbit o;
  fill(*im, s, o);
  SentinelTOPS S;
  S.SubSwath = &s;
  latlon[0] = getLatitude(S, aztime, rgtime, 0);
  latlon[1] = getLontitude(S, aztime, rgtime, 0);
}

}  // extern "C"

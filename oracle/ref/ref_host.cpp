// ref_host.cpp -- builds the reference's host precomputes of the burst-pair
// path into oracle/_ref/libref_host.so.  Test infrastructure: it produces
// reference outputs for the golden fixtures, nothing else links it.
//
// Func.cpp cannot be compiled as a whole here (it needs GDAL and tinyxml2 and
// is Win32 code), so the build recipe extracts the functions of the path
// verbatim from it into oracle/_ref/gen/ (carriage returns stripped) and this
// file compiles them against minimal stand-ins for the reference's types:
//   func_fns.inc        matTxmat, choles, solvechol, invertchol, Polyfit_Orbit
//                       (Func.cpp:940-1126), getVelocity (1284-1314),
//                       computeDC (1828-1865), InKernelInit (2105-2158),
//                       getLineIdxInMetaData (2766-2820),
//                       EstOverlapSize, GetSpectralSep (2935-2976)
//   func_deramp_dc.inc  ComputeDerampPara, per-burst DC polynomials and the
//                       Doppler centroid rows (Func.cpp:1938-1971)
//   func_deramp_kt.inc  ComputeDerampPara, FM rate, reference time and the
//                       Doppler rate kt (Func.cpp:2018-2093)
// The two ComputeDerampPara pieces run inside one function whose locals carry
// the reference's names; the XML parsing between and before them is replaced
// by the caller's DC and FM-rate lists.  Constants.h (PI, SOL, sinc, rect,
// sqr, abs3D, deg2rad) is included from the reference tree.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

using namespace std;

#include "Constants.h"

// ---- stand-ins for the members of DataTypes.h the extracted code touches
struct Polynomial {
  double aztime, t0, c0, c1, c2;
};

struct ResampleTable {
  float *KernelAz = nullptr;
  float *KernelRg = nullptr;
};

struct S1PreciseOrbit {
  int NumPoints = 0;
  int NumCoeff = 0;
  double *orbitAzTime = nullptr;
  double *x_pos = nullptr, *y_pos = nullptr, *z_pos = nullptr;
  double *coef_x = nullptr, *coef_y = nullptr, *coef_z = nullptr;
};

struct SubSwathInfo {
  double firstLineTime = 0, lastLineTime = 0;
  double slrTimeToFirstPixel = 0;
  double azimuthTimeInterval = 0;
  double rangePixelSpacing = 0;
  double wavelength = 0;
  double azimuthSteeringRate = 0;
  int firstValidPixel = 0;
  int numOfBursts = 0, linesPerBurst = 0, samplesPerBurst = 0, numOfLines = 0;
  double burstFirstLineTime[16] = {};
  double burstLastLineTime[16] = {};
  double *rangeDependDopplerRate = nullptr;
  double *dopplerRate = nullptr;
  double *referenceTime = nullptr;
  double *dopplerCentroid = nullptr;
};

struct SentinelTOPS {
  int NumSubSwath = 1;
  SubSwathInfo *SubSwath = nullptr;
};

#include "func_fns.inc"

static void deramp_para_core(SentinelTOPS &S1, S1PreciseOrbit &PreciseOrbit,
                             Polynomial *DCEstimateList, int n_dc, const Polynomial *fm_list,
                             int n_fm) {
  const int i = 0;
  int numbers = n_dc;
#include "func_deramp_dc.inc"
  numbers = n_fm;
  Polynomial *azFmRateList = new Polynomial[numbers];
  for (int k = 0; k < numbers; k++) azFmRateList[k] = fm_list[k];
#include "func_deramp_kt.inc"
}

// ---- C entry points for the golden-fixture script
extern "C" {

int ref_lut(int npoints, double prf, double abw, double rsr2x, float *kaz, float *krg) {
  ResampleTable t;
  if (!InKernelInit(t, npoints, prf, abw, rsr2x)) return 1;
  memcpy(kaz, t.KernelAz, sizeof(float) * npoints * (Interval + 1));
  memcpy(krg, t.KernelRg, sizeof(float) * npoints * (Interval + 1));
  delete[] t.KernelAz;
  delete[] t.KernelRg;
  return 0;
}

// Returns the number of coefficients written to cx, cy, cz.
int ref_polyfit_orbit(int n, double *t, double *x, double *y, double *z, double *cx, double *cy,
                      double *cz) {
  S1PreciseOrbit o;
  o.NumPoints = n;
  o.orbitAzTime = t;
  o.x_pos = x;
  o.y_pos = y;
  o.z_pos = z;
  Polyfit_Orbit(o);
  for (int k = 0; k < o.NumCoeff; k++) {
    cx[k] = o.coef_x[k];
    cy[k] = o.coef_y[k];
    cz[k] = o.coef_z[k];
  }
  delete[] o.coef_x;
  delete[] o.coef_y;
  delete[] o.coef_z;
  return o.NumCoeff;
}

// One sub-swath's deramp rows [n_bursts][samples]: dc, FM rate, reference
// time and kt.  Orbit: fitted coefficients and the state-vector times.
int ref_deramp_params(int n_bursts, int lines_per_burst, int samples_per_burst,
                      int first_valid_pixel, double slr_time_first_pixel,
                      double range_pixel_spacing, double azimuth_time_interval,
                      double first_line_time, double last_line_time, double steering_rate_deg,
                      double wavelength, const double *burst_first, const double *burst_last,
                      Polynomial *dc_list, int n_dc, const Polynomial *fm_list, int n_fm,
                      double *orb_t, int orb_npts, double *cx, double *cy, double *cz,
                      int ncoef, double *dc, double *fm, double *tref, double *kt) {
  if (n_bursts < 1 || n_bursts > 16 || n_fm < n_bursts) return 1;
  SubSwathInfo sw;
  sw.firstLineTime = first_line_time;
  sw.lastLineTime = last_line_time;
  sw.slrTimeToFirstPixel = slr_time_first_pixel;
  sw.azimuthTimeInterval = azimuth_time_interval;
  sw.rangePixelSpacing = range_pixel_spacing;
  sw.wavelength = wavelength;
  sw.azimuthSteeringRate = steering_rate_deg;
  sw.firstValidPixel = first_valid_pixel;
  sw.numOfBursts = n_bursts;
  sw.linesPerBurst = lines_per_burst;
  sw.samplesPerBurst = samples_per_burst;
  for (int b = 0; b < n_bursts; b++) {
    sw.burstFirstLineTime[b] = burst_first[b];
    sw.burstLastLineTime[b] = burst_last[b];
  }
  SentinelTOPS S1;
  S1.SubSwath = &sw;
  S1PreciseOrbit orb;
  orb.NumPoints = orb_npts;
  orb.orbitAzTime = orb_t;
  orb.NumCoeff = ncoef;
  orb.coef_x = cx;
  orb.coef_y = cy;
  orb.coef_z = cz;
  deramp_para_core(S1, orb, dc_list, n_dc, fm_list, n_fm);
  const size_t n = (size_t)n_bursts * samples_per_burst;
  memcpy(dc, sw.dopplerCentroid, n * sizeof(double));
  memcpy(fm, sw.rangeDependDopplerRate, n * sizeof(double));
  memcpy(tref, sw.referenceTime, n * sizeof(double));
  memcpy(kt, sw.dopplerRate, n * sizeof(double));
  delete[] sw.dopplerCentroid;
  delete[] sw.rangeDependDopplerRate;
  delete[] sw.referenceTime;
  delete[] sw.dopplerRate;
  return 0;
}

int ref_overlap_size(int n_bursts, const double *first, const double *last, double dt, int *ov,
                     int *total, int *maximum) {
  if (n_bursts < 2 || n_bursts > 16) return 1;
  SubSwathInfo sw;
  sw.azimuthTimeInterval = dt;
  for (int b = 0; b < n_bursts; b++) {
    sw.burstFirstLineTime[b] = first[b];
    sw.burstLastLineTime[b] = last[b];
  }
  EstOverlapSize(sw, ov, 0, n_bursts - 1, *total, *maximum);
  return 0;
}

double ref_spectral_sep(int n_bursts, int samples_per_burst, int lines_per_burst, double dt,
                        double *kt) {
  SubSwathInfo sw;
  sw.numOfBursts = n_bursts;
  sw.samplesPerBurst = samples_per_burst;
  sw.linesPerBurst = lines_per_burst;
  sw.azimuthTimeInterval = dt;
  sw.dopplerRate = kt;
  return GetSpectralSep(sw);
}

// getLineIdxInMetaData of a sub-swath with these burst times
int ref_line_idx(int n_bursts, int lines_per_burst, const double *first, const double *last,
                 double dt, int num_lines, double t, int burst0, int burstN) {
  if (n_bursts < 1 || n_bursts > 16) return -2;
  SubSwathInfo sw;
  sw.numOfBursts = n_bursts;
  sw.linesPerBurst = lines_per_burst;
  sw.numOfLines = num_lines;
  sw.azimuthTimeInterval = dt;
  for (int b = 0; b < n_bursts; b++) {
    sw.burstFirstLineTime[b] = first[b];
    sw.burstLastLineTime[b] = last[b];
  }
  return getLineIdxInMetaData(sw, t, burst0, burstN);
}

}  // extern "C"

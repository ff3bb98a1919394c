/*
 * tops_oracle.h -- CPU FP64 restatement of the reference TOPS burst-pair path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py
 * may load it.  Nothing in the product links, calls or falls back to it.
 *
 * Every function names the reference file:line it restates (paths are
 * relative to the a787854/InSAR-on-Sentinel-1-TOPS-data project root).
 * Deliberate deviations from the reference (all documented per function):
 *   - phases are kept in FP64 (the reference stores the deramp phase as
 *     float, DerampAndResample.cu:163-164); an emulation switch restores the
 *     float storage so the oracle can be pinned against the reference build;
 *   - coherence pads are zero (the reference leaves them uninitialised,
 *     EstCoh.cu:581-583, 823);
 *   - all sums are FP64 (the reference uses FP32 prefix sums and trees).
 *
 * Data conventions: CInt16 = interleaved int16 (re, im); complex64 =
 * interleaved float; complex128 = interleaved double; all row-major.
 */
#ifndef TOPS_ORACLE_H
#define TOPS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_LUT_BINS 2048

/* Func.cpp:2105-2158 (InKernelInit) with Constants.h:12-30 (sinc, rect).
 * kaz, krg: [ORC_LUT_BINS][npoints] float, row-normalised. */
void orc_lut(int npoints, double prf, double abw, double rsr2x, float *kaz, float *krg);

/* Func.cpp:1050-1126 (Polyfit_Orbit) with matTxmat/choles/solvechol
 * (Func.cpp:940-1013).  Returns the number of coefficients per axis. */
int orc_polyfit_orbit(int npts, const double *t, const double *x, const double *y,
                      const double *z, double *cx, double *cy, double *cz);

/* Func.cpp:1284-1314 (getVelocity): velocity from orbit polynomials at the
 * normalised time t = (t_abs - t_mid) / 10. */
void orc_orbit_velocity(double t, const double *cx, const double *cy, const double *cz,
                        int n, double v[3]);

typedef struct { double aztime, t0, c0, c1, c2; } orc_poly;

/* Func.cpp:1828-1865 (computeDC): linear interpolation of DC estimates. */
void orc_compute_dc(double aztime, const orc_poly *list, int n, orc_poly *res);

typedef struct {
  int n_bursts, samples_per_burst, lines_per_burst, first_valid_pixel;
  double slr_time_first_pixel, range_pixel_spacing, azimuth_time_interval;
  double first_line_time, last_line_time, steering_rate_deg, wavelength;
  const double *burst_first_line_time, *burst_last_line_time;
  const orc_poly *dc_list; int n_dc;
  const orc_poly *fm_list; int n_fm;
  const double *orb_cx, *orb_cy, *orb_cz; int orb_ncoef; double orb_mid_time;
} orc_deramp_in;

/* Func.cpp:1938-2091 (the formula loops of ComputeDerampPara).  Outputs are
 * [n_bursts][samples_per_burst]: Doppler centroid, range-dependent FM rate,
 * reference time and the TOPS Doppler rate kt. */
void orc_deramp_params(const orc_deramp_in *in, double *dc, double *fmrate,
                       double *reftime, double *kt);

/* Func.cpp:2935-2960 (EstOverlapSize). */
void orc_overlap_size(int n_bursts, const double *first_time, const double *last_time,
                      double dt, int *ov, int *total, int *maximum);

/* Func.cpp:2962-2976 (GetSpectralSep); kt is [n_bursts][W]. */
double orc_spectral_sep(int n_bursts, int W, int L, double dt, const double *kt);

/* Stitch_OneSubswath + getLineIdxInMetaData (Func.cpp:2766-2933): for each
 * output line, the row of the burst stack burst0..burstN it copies; returns
 * the line count, or -1 where the reference stops (no burst covers a line)
 * or a row falls outside the stack; map may be NULL (count only). */
int orc_stitch_line_map(int n_bursts, int lines_per_burst, const double *first_time,
                        const double *last_time, double dt, double first_line_time,
                        const int *first_valid, const int *last_valid, int burst0, int burstN,
                        int *map, int capacity);

/* Geometric coregistration of one burst: Geocoreg_cuda.cu:87-323 (llh2xyz,
 * SolveNewtonEq, getPos/getVelo/getAcc, ell2lpGeo), 548-605 (WeighthSet,
 * AMatrixSet), 822-851 (normal equations + Cholesky solve, restated with
 * Func.cpp:959-1013).  Index 0 = master, 1 = slave. */
typedef struct {
  int dem_lines, dem_pixels;
  double lat0, lon0, dlat, dlon;   /* degrees; row r is lat0 - r*dlat */
  double nodata;
  int xmin, xmax, ymin, ymax;      /* master burst box (full-image lines) */
  double dt[2], first_line_time[2], slr_time[2], range_spacing[2];
  double mid_time[2], azi_init[2];
  int line_offset[2];
  const double *cx[2], *cy[2], *cz[2];
  int ncoef[2];
} orc_geo_in;

/* Returns 0 on success, 1 if the normal matrix is not positive definite.
 * pix (optional, may be NULL): [4][dem_lines*dem_pixels] master line,
 * master pixel, slave line, slave pixel (-99999999 for nodata). */
int orc_geocoreg(const orc_geo_in *in, const float *dem, double *cpm_az, double *cpm_rg,
                 double *pix, long *n_valid);

/* cuConstants.cuh:53-65 (normalizeWarp, my_polyval). */
double orc_normalize_warp(double v, double lo, double hi);
double orc_polyval(double l, double p, const double *c);

/* Deramp + demodulation + 12-point sinc resample + reramp of one burst:
 * DerampAndResample.cu:108-183 (GetIndexes, DerampDemod_Shared) and
 * 349-520 (Interpolation_12p). */
typedef struct {
  const int16_t *slave; long slave_stride;   /* complex elements per row */
  int mbox[4], sbox[4];                      /* {x0, x1, y0, y1} inclusive */
  double cpm_az[6], cpm_rg[6], az_shift;
  const float *kaz, *krg; int npoints;
  int s_burst_idx, s_lines_per_burst;
  double dt;
  const double *kt, *tref, *fdc;             /* indexed by sample x */
  int f32_phase;   /* 1: store the deramp phase as float like the reference */
} orc_resample_in;

/* out: complex128 [mLines][mPixels].  Returns counts of (outside, edge,
 * interior) pixels through cnt[3] when cnt != NULL. */
void orc_resample(const orc_resample_in *in, double *out, long cnt[3]);

/* Same, but only for master rows [row0, row0 + nrows); out holds those rows. */
void orc_resample_rows(const orc_resample_in *in, int row0, int nrows, double *out);

/* Windowed coherence of one burst: EstCoh.cu:101-139 (CohMatSet), 413-456
 * (Cohbasic) and 359-411 (CpCoh2, same mask).  Zero padding.  coh: double
 * [lines][pixels]. */
void orc_coherence(const int16_t *master, const float *slave, int lines, int pixels,
                   int win_rg, int win_az, double *coh);

/* ESD shifts over burst overlaps: EstESD.cu:62-161, 243-259, 297-546,
 * 914-1252.  Inputs are the concatenated overlap bands [sum(ov)][W].
 * shift[n_ov] in pixels; sums (optional) [n_ov][2] complex phasor sums;
 * n_used (optional) pixels that passed the coherence mask. */
void orc_esd(const int16_t *mF, const int16_t *mB, const float *sF, const float *sB,
             const int *ov, int n_ov, int W, int win_az, int win_rg, double thr,
             double spec_sep, double dt, double *shift, double *sums, long *n_used);

/* Number of OpenMP threads the oracle uses (for the cpu_baseline report). */
int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif

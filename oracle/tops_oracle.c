/*
 * tops_oracle.c -- CPU FP64 restatement of the reference TOPS burst-pair path.
 *
 * TEST INFRASTRUCTURE ONLY (see tops_oracle.h).  Built with strict IEEE
 * double arithmetic (-ffp-contract=off, no -ffast-math) so that index and
 * LUT-bin decisions are reproducible.  OpenMP parallelises over output rows
 * and DEM rows; every reduction is combined in a fixed order, so results do
 * not depend on the thread count.
 */
#include "tops_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.1415926535897931e+0   /* Constants.h:7 */
#define ORC_SOL 299792458.0            /* Constants.h:6 */
#define ORC_INTERVAL 2047              /* Constants.h:8 */
#define ORC_ELL_A 6378137.0            /* cuConstants.cuh:5 */
#define ORC_ELL_B 6356752.3142451794975639665996337   /* cuConstants.cuh:6 */

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

static double sqr(double x) { return x * x; }

/* Constants.h:13 */
static double orc_sinc(double x) { return (x == 0) ? 1 : sin(ORC_PI * x) / (ORC_PI * x); }

/* Constants.h:25-31 */
static double orc_rect(double x) {
  double ans = 0.0;
  if (x < 0.5 && x > -0.5) ans = 1;
  else if (x == 0.5 || x == -0.5) ans = 0.5;
  return ans;
}

/* ------------------------------------------------------------------ LUT */
/* Func.cpp:2105-2158.  The stored value is float; the normalisation divides
 * the stored float by the double row sum and rounds back to float, exactly
 * as the reference's `KernelAz[i*Npoints + p] /= Sum_Az`. */
void orc_lut(int npoints, double prf, double abw, double rsr2x, float *kaz, float *krg) {
  const double chi_az = prf / abw;
  const double chi_rg = (rsr2x / 2.0) / abw;   /* reference quirk: azimuth bandwidth */
  const double dx = 1.0 / ORC_INTERVAL;
  const int npd2 = npoints / 2;
  const int nint = ORC_INTERVAL + 1;
  for (int i = 0; i < nint; i++) {
    double sum_az = 0.0, sum_rg = 0.0;
    for (int j = 0; j < npoints; j++) {
      double x = 1.0 - npd2 + j - dx * i;
      double v_az = 1. - 1. / chi_az;
      double v_rg = 1. - 1. / chi_rg;
      double c_az = orc_sinc(x) * orc_rect(x / (double)npoints) * cos(v_az * ORC_PI * x) /
                    (1.0 - sqr(2.0 * v_az * x));
      sum_az += c_az;
      kaz[i * npoints + j] = (float)c_az;
      double c_rg = orc_sinc(x) * orc_rect(x / (double)npoints) * cos(v_rg * ORC_PI * x) /
                    (1.0 - sqr(2.0 * v_rg * x));
      sum_rg += c_rg;
      krg[i * npoints + j] = (float)c_rg;
    }
    for (int p = 0; p < npoints; p++) {
      kaz[i * npoints + p] = (float)((double)kaz[i * npoints + p] / sum_az);
      krg[i * npoints + p] = (float)((double)krg[i * npoints + p] / sum_rg);
    }
  }
}

/* ------------------------------------------------------- orbit fitting */
/* Func.cpp:940-957 (matTxmat): Res = A^T B with A [alines][rlines]. */
static void mat_t_mat(const double *a, const double *b, double *res, int alines, int rlines,
                      int rpixels) {
  for (int i = 0; i < rlines; i++)
    for (int j = 0; j < rpixels; j++) {
      double sum = 0.0;
      for (int k = 0; k < alines; k++) sum += a[k * rlines + i] * b[k * rpixels + j];
      res[i * rpixels + j] = sum;
    }
}

/* Func.cpp:959-983 (choles): lower factor stored in the lower triangle.
 * Returns 1 if the matrix is not positive definite. */
static int choles(double *a, int n) {
  int bad = 0;
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      double sum = a[i * n + j];
      for (int k = i - 1; k >= 0; --k) sum -= a[i * n + k] * a[j * n + k];
      if (i == j) {
        if (sum <= 0.) bad = 1;
        a[i * n + i] = sqrt(sum);
      } else {
        a[j * n + i] = sum / a[i * n + i];
      }
    }
  return bad;
}

/* Func.cpp:985-1013 (solvechol) for a single right-hand side. */
static void solvechol(const double *a, double *b, int n) {
  for (int i = 0; i < n; ++i) {
    double sum = b[i];
    for (int j = i - 1; j >= 0; --j) sum -= a[i * n + j] * b[j];
    b[i] = sum / a[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double sum = b[i];
    for (int j = i + 1; j < n; ++j) sum -= a[j * n + i] * b[j];
    b[i] = sum / a[i * n + i];
  }
}

/* Func.cpp:1050-1126 */
int orc_polyfit_orbit(int npts, const double *t, const double *x, const double *y,
                      const double *z, double *cx, double *cy, double *cz) {
  double *nt = (double *)malloc(sizeof(double) * npts);
  for (int i = 0; i < npts; i++) nt[i] = (t[i] - t[npts / 2]) / 10.0;
  int degree = (npts > 6) ? 5 : npts - 2;
  int nu = degree + 1;
  double *a = (double *)malloc(sizeof(double) * npts * nu);
  double n[64] = {0}, rx[8] = {0}, ry[8] = {0}, rz[8] = {0};
  for (int i = 0; i < npts; i++)
    for (int j = 0; j < nu; j++) a[i * nu + j] = pow(nt[i], j);
  mat_t_mat(a, a, n, npts, nu, nu);
  mat_t_mat(a, x, rx, npts, nu, 1);
  mat_t_mat(a, y, ry, npts, nu, 1);
  mat_t_mat(a, z, rz, npts, nu, 1);
  choles(n, nu);
  solvechol(n, rx, nu);
  solvechol(n, ry, nu);
  solvechol(n, rz, nu);
  for (int i = 0; i < nu; i++) {
    cx[i] = rx[i];
    cy[i] = ry[i];
    cz[i] = rz[i];
  }
  free(a);
  free(nt);
  return nu;
}

/* Func.cpp:1284-1314 */
void orc_orbit_velocity(double t, const double *cx, const double *cy, const double *cz, int n,
                        double v[3]) {
  v[0] = cx[1];
  v[1] = cy[1];
  v[2] = cz[1];
  for (int i = 2; i < n; ++i) {
    double powt = (double)i * pow(t, i - 1);
    v[0] += cx[i] * powt;
    v[1] += cy[i] * powt;
    v[2] += cz[i] * powt;
  }
  v[0] /= (double)10.0;
  v[1] /= (double)10.0;
  v[2] /= (double)10.0;
}

/* ---------------------------------------------------- deramp parameters */
/* Func.cpp:1828-1865.  The reference reads Input[N] when AzTime is after the
 * last estimate (i1 = N); the restatement clamps to the last entry. */
void orc_compute_dc(double aztime, const orc_poly *in, int n, orc_poly *res) {
  int i0 = 0, i1 = 0;
  if (aztime < in[0].aztime) {
    i0 = 0;
    i1 = 1;
  } else if (aztime > in[n - 1].aztime) {
    i0 = n - 2;
    i1 = n - 1;
  } else {
    for (int i = 0; i < n - 1; i++)
      if (aztime >= in[i].aztime && aztime < in[i + 1].aztime) {
        i0 = i;
        i1 = i + 1;
        break;
      }
  }
  res->aztime = aztime;
  res->t0 = in[i0].t0;
  double mu = (aztime - in[i0].aztime) / (in[i1].aztime - in[i0].aztime);
  res->c0 = (1 - mu) * in[i0].c0 + mu * in[i1].c0;
  res->c1 = (1 - mu) * in[i0].c1 + mu * in[i1].c1;
  res->c2 = (1 - mu) * in[i0].c2 + mu * in[i1].c2;
}

/* Func.cpp:1938-2091 */
void orc_deramp_params(const orc_deramp_in *in, double *dc, double *fmrate, double *reftime,
                       double *kt) {
  const int nb = in->n_bursts, W = in->samples_per_burst;
  orc_poly *dcb = (orc_poly *)malloc(sizeof(orc_poly) * nb);
  if (in->n_dc > nb) {                                   /* Func.cpp:1939-1945 */
    for (int b = 0; b < nb; b++) dcb[b] = in->dc_list[b];
  } else {                                               /* Func.cpp:1946-1955 */
    for (int b = 0; b < nb; b++) {
      double centre = 0.5 * (in->burst_first_line_time[b] + in->burst_last_line_time[b]);
      orc_compute_dc(centre, in->dc_list, in->n_dc, &dcb[b]);
    }
  }
  for (int b = 0; b < nb; b++)                           /* Func.cpp:1960-1970 */
    for (int x = 0; x < W; x++) {
      double slrt = (in->slr_time_first_pixel + x * in->range_pixel_spacing / ORC_SOL) * 2;
      double d = slrt - dcb[b].t0;
      dc[b * W + x] = dcb[b].c0 + dcb[b].c1 * d + dcb[b].c2 * sqr(d);
    }
  for (int b = 0; b < nb; b++)                           /* Func.cpp:2021-2031 */
    for (int x = 0; x < W; x++) {
      double slrt = (in->slr_time_first_pixel + x * in->range_pixel_spacing / ORC_SOL) * 2;
      double d = slrt - in->fm_list[b].t0;
      fmrate[b * W + x] = in->fm_list[b].c0 + in->fm_list[b].c1 * d + in->fm_list[b].c2 * d * d;
    }
  double temp1 = in->lines_per_burst * in->azimuth_time_interval / 2.0;  /* Func.cpp:2037 */
  for (int b = 0; b < nb; b++) {                         /* Func.cpp:2042-2056 */
    double temp2 = temp1 + dc[b * W + in->first_valid_pixel] / fmrate[b * W + in->first_valid_pixel];
    for (int x = 0; x < W; x++) reftime[b * W + x] = temp2 - dc[b * W + x] / fmrate[b * W + x];
  }
  double az = (in->first_line_time + in->last_line_time) / 2.0;   /* Func.cpp:2073-2091 */
  az = (az - in->orb_mid_time) / 10.0;
  for (int b = 0; b < nb; b++) {
    double v[3];
    orc_orbit_velocity(az, in->orb_cx, in->orb_cy, in->orb_cz, in->orb_ncoef, v);
    double speed = sqrt(sqr(v[0]) + sqr(v[1]) + sqr(v[2]));
    double steer = in->steering_rate_deg * ORC_PI / 180.0;
    double krot = 2 * speed * steer / in->wavelength;
    for (int x = 0; x < W; x++) {
      double r = fmrate[b * W + x];
      kt[b * W + x] = r * krot / (r - krot);
    }
  }
  free(dcb);
}

/* Func.cpp:2935-2960 */
void orc_overlap_size(int n_bursts, const double *first_time, const double *last_time, double dt,
                      int *ov, int *total, int *maximum) {
  *total = 0;
  *maximum = -9999;
  for (int i = 0; i < n_bursts - 1; i++) {
    double endtime = last_time[i];
    double starttime = first_time[i + 1];
    int lines = (int)floor((endtime - starttime) / dt);
    ov[i] = lines;
    *total += lines;
    if (lines > *maximum) *maximum = lines;
  }
}

/* Func.cpp:2962-2976 */
double orc_spectral_sep(int n_bursts, int W, int L, double dt, const double *kt) {
  double tcycle = L * dt;
  double sum = 0.0;
  for (int i = 0; i < n_bursts; i++)
    for (int p = 0; p < W; p++) sum += kt[i * W + p] * tcycle;
  return sum / W / n_bursts;
}

/* --------------------------------------------------------------- geocoreg */
/* ----------------------------------------------------------- stitching */
/* getLineIdxInMetaData (Func.cpp:2766-2820), line for line */
static int orc_line_idx(int nb, int L, const double *first, const double *last, double dt,
                        int num_lines, double target, int b0, int bN) {
  int sy0 = -1, sy1 = -1, burst_num0 = -1, burst_num1 = -1, k = 0;
  for (int i = 0; i < nb; i++) {
    if (target >= first[i] && target < last[i]) {
      int sy = i * L + (int)(((target - first[i]) / dt) + 0.5);
      if (k == 0) {
        sy0 = sy;
        burst_num0 = i;
      } else {
        sy1 = sy;
        burst_num1 = i;
        break;
      }
      ++k;
    }
  }
  if (sy0 != -1 && sy1 != -1) {
    if (burst_num1 == b0) return sy1;
    if (burst_num1 == bN + 1) return sy0;
    double mid = (last[burst_num0] + first[burst_num1]) / 2.0;
    if (target > mid) return sy1;
  }
  if (target < last[nb - 1] + dt && target >= last[nb - 1]) sy0 = num_lines - 1;
  return sy0;
}

/* Stitch_OneSubswath (Func.cpp:2822-2933): the output lines and the gapped-
 * image row each one reads */
int orc_stitch_line_map(int n_bursts, int lines_per_burst, const double *first_time,
                        const double *last_time, double dt, double first_line_time,
                        const int *first_valid, const int *last_valid, int burst0, int burstN,
                        int *map, int capacity) {
  double t_first = first_time[burst0] + first_valid[burst0] * dt;   /* Func.cpp:401 */
  double t_last = first_time[burstN] + last_valid[burstN] * dt;      /* Func.cpp:403 */
  int y_min = (int)((t_first - first_line_time) / dt);
  int y_max = (int)((t_last - first_line_time) / dt);
  int height = y_max - y_min + 1;
  if (!map) return height;
  if (height > capacity) return -1;
  for (int y = y_min; y <= y_max; y++) {
    int yy = y - y_min;
    double line_time = t_first + yy * dt;
    int idx = orc_line_idx(n_bursts, lines_per_burst, first_time, last_time, dt,
                           n_bursts * lines_per_burst, line_time, burst0, burstN);
    if (idx == -1) return -1;
    idx -= burst0 * lines_per_burst;
    if (idx < 0 || idx >= (burstN - burst0 + 1) * lines_per_burst) return -1;
    map[yy] = idx;
  }
  return height;
}

/* cuConstants.cuh:53-56 */
double orc_normalize_warp(double v, double lo, double hi) {
  return (v - (0.5 * (lo + hi))) / (0.25 * (hi - lo));
}

/* cuConstants.cuh:58-65 */
double orc_polyval(double x, double y, const double *c) {
  return (c[0] + c[1] * x + c[2] * y + c[3] * x * x + c[4] * x * y + c[5] * y * y);
}

/* Geocoreg_cuda.cu:87-99 */
static void llh2xyz(double phi, double lam, float height, double e2, double res[3]) {
  double sl = sin(lam), cl = cos(lam), sp = sin(phi), cp = cos(phi);
  double nph = ORC_ELL_A / sqrt(1.0 - e2 * sqr(sp)) + height;
  res[0] = nph * cp * cl;
  res[1] = nph * cp * sl;
  res[2] = (nph - e2 * (nph - height)) * sp;
}

/* Geocoreg_cuda.cu:123-144 */
static void get_pos(double t, double *p, const double *cx, const double *cy, const double *cz,
                    int n) {
  p[0] = p[1] = p[2] = 0.0;
  for (int i = n - 1; i >= 0; --i) {
    p[0] *= t;
    p[0] += cx[i];
    p[1] *= t;
    p[1] += cy[i];
    p[2] *= t;
    p[2] += cz[i];
  }
}

/* Geocoreg_cuda.cu:176-205 */
static void get_acc(double t, double *a, const double *cx, const double *cy, const double *cz,
                    int n) {
  a[0] = a[1] = a[2] = 0.0;
  for (int i = 2; i < n; ++i) {
    double powt1 = (double)((i - 1) * i) * pow(t, i - 2);
    a[0] += cx[i] * powt1;
    a[1] += cy[i] * powt1;
    a[2] += cz[i] * powt1;
  }
  a[0] /= 100.0;
  a[1] /= 100.0;
  a[2] /= 100.0;
}

/* Geocoreg_cuda.cu:101-112 */
static double solve_newton(const double tgt[3], double ps[3], const double vs[3],
                           const double as[3]) {
  ps[0] = tgt[0] - ps[0];
  ps[1] = tgt[1] - ps[1];
  ps[2] = tgt[2] - ps[2];
  return (-(vs[0] * ps[0] + vs[1] * ps[1] + vs[2] * ps[2]) /
          ((as[0] * ps[0] + as[1] * ps[1] + as[2] * ps[2]) - vs[0] * vs[0] - vs[1] * vs[1] -
           vs[2] * vs[2]));
}

/* Geocoreg_cuda.cu:250-311 for one image k: returns line and pixel. */
static void ell2lp(const orc_geo_in *in, int k, const double tgt[3], double *line, double *pixel) {
  double az = in->azi_init[k];
  double ps[3], vs[3], as[3];
  for (int i = 0; i <= 10; i++) {
    double t = (az - in->mid_time[k]) / 10.0;
    get_pos(t, ps, in->cx[k], in->cy[k], in->cz[k], in->ncoef[k]);
    orc_orbit_velocity(t, in->cx[k], in->cy[k], in->cz[k], in->ncoef[k], vs);
    get_acc(t, as, in->cx[k], in->cy[k], in->cz[k], in->ncoef[k]);
    double sol = solve_newton(tgt, ps, vs, as);
    az += sol;
    if (fabs(sol) < 1e-010) break;
  }
  double t = (az - in->mid_time[k]) / 10.0;
  get_pos(t, ps, in->cx[k], in->cy[k], in->cz[k], in->ncoef[k]);
  *line = in->line_offset[k] + (az - in->first_line_time[k]) / in->dt[k];
  double r = sqrt(sqr(tgt[0] - ps[0]) + sqr(tgt[1] - ps[1]) + sqr(tgt[2] - ps[2]));
  *pixel = (r - in->slr_time[k] * ORC_SOL) / in->range_spacing[k];
}

/* Geocoreg_cuda.cu:211-323, 548-605, 822-851 */
int orc_geocoreg(const orc_geo_in *in, const float *dem, double *cpm_az, double *cpm_rg,
                 double *pix, long *n_valid) {
  const double e2 = 1.0 - (ORC_ELL_B * ORC_ELL_B / ORC_ELL_A / ORC_ELL_A);   /* :666-668 */
  const int rows = in->dem_lines, cols = in->dem_pixels;
  const long npx = (long)rows * cols;
  /* per-row partial normal equations: 21 (upper N) + 6 + 6, combined in
   * row order after the parallel loop */
  double *part = (double *)calloc((size_t)rows * 36, sizeof(double));
  long *cnt = (long *)calloc((size_t)rows, sizeof(long));
#pragma omp parallel for schedule(dynamic, 4)
  for (int row = 0; row < rows; row++) {
    double *acc = part + (size_t)row * 36;
    for (int col = 0; col < cols; col++) {
      long id = (long)row * cols + col;
      float h = dem[id];
      double ml = -99999999, mp = -99999999, sl = -99999999, sp = -99999999;
      if (h != in->nodata) {
        double tgt[3];
        double lat = (in->lat0 - in->dlat * row) * ORC_PI / 180.0;
        double lon = (in->lon0 + in->dlon * col) * ORC_PI / 180.0;
        llh2xyz(lat, lon, h, e2, tgt);
        ell2lp(in, 0, tgt, &ml, &mp);
        ell2lp(in, 1, tgt, &sl, &sp);
      }
      if (pix) {
        pix[id] = ml;
        pix[npx + id] = mp;
        pix[2 * npx + id] = sl;
        pix[3 * npx + id] = sp;
      }
      /* WeighthSet (:566-570) */
      if (h != in->nodata && ml >= in->ymin && ml <= in->ymax && mp >= in->xmin &&
          mp <= in->xmax) {
        /* AMatrixSet (:591-602) */
        double L = orc_normalize_warp(ml, in->ymin, in->ymax);
        double P = orc_normalize_warp(mp, in->xmin, in->xmax);
        double a[6] = {1, L, P, L * L, L * P, P * P};
        int q = 0;
        for (int i = 0; i < 6; i++)
          for (int j = i; j < 6; j++) acc[q++] += a[i] * a[j];
        for (int i = 0; i < 6; i++) {
          acc[21 + i] += a[i] * sl;
          acc[27 + i] += a[i] * sp;
        }
        cnt[row]++;
      }
    }
  }
  double tot[33] = {0};
  long nv = 0;
  for (int row = 0; row < rows; row++) {
    for (int q = 0; q < 33; q++) tot[q] += part[(size_t)row * 36 + q];
    nv += cnt[row];
  }
  free(part);
  free(cnt);
  if (n_valid) *n_valid = nv;
  double n[36];
  int q = 0;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++) {
      n[i * 6 + j] = tot[q];
      n[j * 6 + i] = tot[q];
      q++;
    }
  if (choles(n, 6)) return 1;
  double raz[6], rrg[6];
  for (int i = 0; i < 6; i++) {
    raz[i] = tot[21 + i];
    rrg[i] = tot[27 + i];
  }
  solvechol(n, raz, 6);
  solvechol(n, rrg, 6);
  for (int i = 0; i < 6; i++) {
    cpm_az[i] = raz[i];
    cpm_rg[i] = rrg[i];
  }
  return 0;
}

/* --------------------------------------------------------------- resample */
/* DerampAndResample.cu:150-158: deramp + demodulation phase of slave sample
 * (y, x) in full-image coordinates. */
static double deramp_phase(const orc_resample_in *in, int y, int x) {
  int first_line = in->s_burst_idx * in->s_lines_per_burst;
  double ta = (y - first_line) * in->dt;
  double kt = in->kt[x];
  double deramp = -ORC_PI * kt * sqr(ta - in->tref[x]);
  double demod = -2.0 * ORC_PI * in->fdc[x] * ta;
  return deramp + demod;
}

/* Interpolation_12p (DerampAndResample.cu:349-520) for master row `row`
 * (0-based inside the master box); writes mPixels complex128 values. */
static void resample_row(const orc_resample_in *in, const double *dr, const double *ph,
                         int s_pix, int row, double *out, long cnt[3]) {
  const int mpix = in->mbox[1] - in->mbox[0] + 1;
  const int n2m1 = in->npoints / 2 - 1;
  const int sx0 = in->sbox[0], sxm = in->sbox[1], sy0 = in->sbox[2], sym = in->sbox[3];
  for (int col = 0; col < mpix; col++) {
    double P = orc_normalize_warp(col, in->mbox[0], in->mbox[1]);
    double L = orc_normalize_warp(row + 0 + in->mbox[2], in->mbox[2], in->mbox[3]);
    double yl = orc_polyval(L, P, in->cpm_az) + in->az_shift;
    double xp = orc_polyval(L, P, in->cpm_rg);
    /* GetIndexes (:108-112) */
    int il0 = (int)trunc(yl);
    int il1 = (int)((yl - il0) * ORC_INTERVAL + 0.5);
    int ip0 = (int)trunc(xp);
    int ip1 = (int)((xp - ip0) * ORC_INTERVAL + 0.5);
    double *o = out + 2 * (size_t)col;
    if (il0 > sym || il0 < sy0 || ip0 > sxm || ip0 < sx0) {
      o[0] = 0.0;
      o[1] = 0.0;
      if (cnt) cnt[0]++;
    } else if (il0 > sym - n2m1 - 2 || il0 < sy0 + n2m1 || ip0 > sxm - n2m1 - 2 ||
               ip0 < sx0 + n2m1) {
      /* nearest sample, reramped with its own phase (:393-399) */
      size_t k = (size_t)(il0 - sy0) * s_pix + (ip0 - sx0);
      double c = cos(ph[k]), s = sin(ph[k]);
      o[0] = dr[2 * k] * c + dr[2 * k + 1] * s;
      o[1] = dr[2 * k + 1] * c - dr[2 * k] * s;
      if (cnt) cnt[1]++;
    } else {
      /* LUT rows are clamped like the reference's clamped texture fetch */
      if (il1 < 0) il1 = 0;
      if (il1 > ORC_LUT_BINS - 1) il1 = ORC_LUT_BINS - 1;
      if (ip1 < 0) ip1 = 0;
      if (ip1 > ORC_LUT_BINS - 1) ip1 = ORC_LUT_BINS - 1;
      const float *kl = in->kaz + (size_t)il1 * in->npoints;
      const float *kp = in->krg + (size_t)ip1 * in->npoints;
      int p0 = ip0 - (sx0 + n2m1);
      int l0 = il0 - (sy0 + n2m1);
      double sre = 0.0, sim = 0.0, sph = 0.0;
      for (int j = 0; j < in->npoints; j++) {
        const double *drow = dr + 2 * ((size_t)(l0 + j) * s_pix + p0);
        const double *prow = ph + (size_t)(l0 + j) * s_pix + p0;
        double tre = 0.0, tim = 0.0, tph = 0.0;
        for (int i = 0; i < in->npoints; i++) {
          tre += drow[2 * i] * (double)kp[i];
          tim += drow[2 * i + 1] * (double)kp[i];
          tph += prow[i] * (double)kp[i];
        }
        sre += tre * (double)kl[j];
        sim += tim * (double)kl[j];
        sph += tph * (double)kl[j];
      }
      double c = cos(sph), s = sin(sph);
      o[0] = sre * c + sim * s;
      o[1] = sim * c - sre * s;
      if (cnt) cnt[2]++;
    }
  }
}

/* DerampDemod_Shared (DerampAndResample.cu:117-183) over the whole slave box. */
static void deramp_box(const orc_resample_in *in, double *dr, double *ph) {
  const int s_pix = in->sbox[1] - in->sbox[0] + 1;
  const int s_lin = in->sbox[3] - in->sbox[2] + 1;
#pragma omp parallel for schedule(static)
  for (int r = 0; r < s_lin; r++)
    for (int c = 0; c < s_pix; c++) {
      size_t k = (size_t)r * s_pix + c;
      double phi = deramp_phase(in, r + in->sbox[2], c + in->sbox[0]);
      const int16_t *s = in->slave + 2 * ((size_t)r * in->slave_stride + c);
      double re = s[0], im = s[1];
      double cs = cos(phi), sn = sin(phi);
      double dre = re * cs - im * sn, dim = re * sn + im * cs;
      if (in->f32_phase) {
        /* reference storage: float phase array and float complex product */
        ph[k] = (double)(float)phi;
        dre = (double)(float)(re * (double)(float)cs - im * (double)(float)sn);
        dim = (double)(float)(re * (double)(float)sn + im * (double)(float)cs);
      } else {
        ph[k] = phi;
      }
      dr[2 * k] = dre;
      dr[2 * k + 1] = dim;
    }
}

void orc_resample_rows(const orc_resample_in *in, int row0, int nrows, double *out) {
  const int s_pix = in->sbox[1] - in->sbox[0] + 1;
  const int s_lin = in->sbox[3] - in->sbox[2] + 1;
  const int mpix = in->mbox[1] - in->mbox[0] + 1;
  double *dr = (double *)malloc(sizeof(double) * 2 * (size_t)s_pix * s_lin);
  double *ph = (double *)malloc(sizeof(double) * (size_t)s_pix * s_lin);
  deramp_box(in, dr, ph);
#pragma omp parallel for schedule(dynamic, 2)
  for (int r = 0; r < nrows; r++)
    resample_row(in, dr, ph, s_pix, row0 + r, out + 2 * (size_t)r * mpix, NULL);
  free(dr);
  free(ph);
}

void orc_resample(const orc_resample_in *in, double *out, long cnt[3]) {
  const int s_pix = in->sbox[1] - in->sbox[0] + 1;
  const int s_lin = in->sbox[3] - in->sbox[2] + 1;
  const int mpix = in->mbox[1] - in->mbox[0] + 1;
  const int mlin = in->mbox[3] - in->mbox[2] + 1;
  double *dr = (double *)malloc(sizeof(double) * 2 * (size_t)s_pix * s_lin);
  double *ph = (double *)malloc(sizeof(double) * (size_t)s_pix * s_lin);
  long *rc = (long *)calloc((size_t)mlin * 3, sizeof(long));
  deramp_box(in, dr, ph);
#pragma omp parallel for schedule(dynamic, 2)
  for (int r = 0; r < mlin; r++)
    resample_row(in, dr, ph, s_pix, r, out + 2 * (size_t)r * mpix, rc + 3 * (size_t)r);
  if (cnt) {
    cnt[0] = cnt[1] = cnt[2] = 0;
    for (int r = 0; r < mlin; r++)
      for (int q = 0; q < 3; q++) cnt[q] += rc[3 * (size_t)r + q];
  }
  free(rc);
  free(dr);
  free(ph);
}

/* -------------------------------------------------------------- coherence */
/* EstCoh.cu:101-139 + 413-456: box [r-dy, r-dy+win_az) x [c-dx, c-dx+win_rg)
 * with dx = (win_rg-1)/2, dy = (win_az-1)/2 (Func.cpp:2643-2644), zero
 * outside the burst, gamma = 0 where |slave| < 0.001. */
void orc_coherence(const int16_t *master, const float *slave, int lines, int pixels, int win_rg,
                   int win_az, double *coh) {
  const int dx = (win_rg - 1) / 2, dy = (win_az - 1) / 2;
#pragma omp parallel for schedule(dynamic, 4)
  for (int r = 0; r < lines; r++)
    for (int c = 0; c < pixels; c++) {
      double sre = 0, sim = 0, ps = 0, pm = 0;
      for (int j = 0; j < win_az; j++) {
        int y = r - dy + j;
        if (y < 0 || y >= lines) continue;
        for (int i = 0; i < win_rg; i++) {
          int x = c - dx + i;
          if (x < 0 || x >= pixels) continue;
          size_t k = (size_t)y * pixels + x;
          double mr = master[2 * k], mi = master[2 * k + 1];
          double sr = slave[2 * k], si = slave[2 * k + 1];
          sre += mr * sr + mi * si;   /* m * conj(s) */
          sim += mi * sr - mr * si;
          ps += sr * sr + si * si;
          pm += mr * mr + mi * mi;
        }
      }
      size_t k = (size_t)r * pixels + c;
      double amp = hypot((double)slave[2 * k], (double)slave[2 * k + 1]);
      double p = ps * pm;
      if (amp < 0.001)
        coh[k] = 0.0;
      else
        coh[k] = (p > 0.0) ? sqrt(sre * sre + sim * sim) / sqrt(p) : 0.0;
    }
}

/* ------------------------------------------------------------------- ESD */
/* One band's coherence (CohMatrixSet + prefix kernels + CpCoh2_ESD,
 * EstESD.cu:94-128, 297-546): zero padded, no amplitude mask. */
static double band_gamma(const int16_t *m, const float *s, int lines, int W, int win_az,
                         int win_rg, int r, int c) {
  const int dw = (win_rg - 1) / 2, dh = (win_az - 1) / 2;
  double sre = 0, sim = 0, ps = 0, pm = 0;
  for (int j = 0; j < win_az; j++) {
    int y = r - dh + j;
    if (y < 0 || y >= lines) continue;
    for (int i = 0; i < win_rg; i++) {
      int x = c - dw + i;
      if (x < 0 || x >= W) continue;
      size_t k = (size_t)y * W + x;
      double mr = m[2 * k], mi = m[2 * k + 1];
      double sr = s[2 * k], si = s[2 * k + 1];
      sre += mr * sr + mi * si;
      sim += mi * sr - mr * si;
      ps += sr * sr + si * si;
      pm += mr * mr + mi * mi;
    }
  }
  double pp = ps * pm;
  return (pp > 0.0) ? sqrt(sre * sre + sim * sim) / sqrt(pp) : 0.0;
}

void orc_esd(const int16_t *mF, const int16_t *mB, const float *sF, const float *sB,
             const int *ov, int n_ov, int W, int win_az, int win_rg, double thr, double spec_sep,
             double dt, double *shift, double *sums, long *n_used) {
  long off = 0;
  for (int o = 0; o < n_ov; o++) {
    const int lines = ov[o];
    const int16_t *mf = mF + 2 * off * W, *mb = mB + 2 * off * W;
    const float *sf = sF + 2 * off * W, *sb = sB + 2 * off * W;
    double *rs = (double *)calloc((size_t)(lines > 0 ? lines : 1) * 2, sizeof(double));
    long *ru = (long *)calloc((size_t)(lines > 0 ? lines : 1), sizeof(long));
#pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < lines; r++) {
      double ar = 0, ai = 0;
      long used = 0;
      for (int c = 0; c < W; c++) {
        double gf = band_gamma(mf, sf, lines, W, win_az, win_rg, r, c);
        double gb = band_gamma(mb, sb, lines, W, win_az, win_rg, r, c);
        double g = (gf + gb) / 2.0;                       /* Divide2 :243-259 */
        size_t k = (size_t)r * W + c;
        /* DoubleDifference4OneD (:62-91): (mF sF*) conj(mB sB*) */
        double fr = mf[2 * k] * (double)sf[2 * k] + mf[2 * k + 1] * (double)sf[2 * k + 1];
        double fi = mf[2 * k + 1] * (double)sf[2 * k] - mf[2 * k] * (double)sf[2 * k + 1];
        double br = mb[2 * k] * (double)sb[2 * k] + mb[2 * k + 1] * (double)sb[2 * k + 1];
        double bi = mb[2 * k + 1] * (double)sb[2 * k] - mb[2 * k] * (double)sb[2 * k + 1];
        double dre = fr * br + fi * bi, dim = fi * br - fr * bi;
        /* MaskOut (:130-161) */
        if (g < thr || g >= 1) continue;
        /* An exactly-zero double difference (slave outside its box) gets
         * the phase atan2 gives its signed zeros (0, -0, pi or -pi), as the
         * reference's MaskOut does; the products above produce the same
         * signs of zero as its FP32 cuCmulf chain. */
        double th = atan2(dim, dre);
        ar += cos(th);
        ai += sin(th);
        used++;
      }
      rs[2 * r] = ar;
      rs[2 * r + 1] = ai;
      ru[r] = used;
    }
    double tr = 0, ti = 0;
    long tu = 0;
    for (int r = 0; r < lines; r++) {
      tr += rs[2 * r];
      ti += rs[2 * r + 1];
      tu += ru[r];
    }
    free(rs);
    free(ru);
    if (sums) {
      sums[2 * o] = tr;
      sums[2 * o + 1] = ti;
    }
    if (n_used) n_used[o] = tu;
    /* EstESD.cu:1213-1217 */
    shift[o] = atan2(ti, tr) / (2 * ORC_PI * spec_sep * dt);
    off += lines;
  }
}

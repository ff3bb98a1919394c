// tops_host.cpp -- host-side TOPS precomputes and the config.txt reader.
//
// These are the host functions the reference's stage drivers feed to the
// GPU wrappers: the interpolation LUT (InKernelInit, Func.cpp:2105-2158),
// the orbit polynomial fit (Polyfit_Orbit, Func.cpp:1050-1126), the TOPS
// deramp parameters (ComputeDerampPara / computeDC, Func.cpp:1828-2099),
// burst overlaps and spectral separation (Func.cpp:2935-2976), and the
// key=value configuration reader (ReadInput, Func.cpp:7-130).  The
// formulas and their evaluation order are kept (the LUT is bit-identical to
// the reference's, which matters for the LUT-bin parity of the resampler).
#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <array>
#include <string>
#include <vector>

#include "tops_b200.h"

namespace {

constexpr double kPi = 3.1415926535897931e+0;
constexpr double kSol = 299792458.0;
constexpr int kInterval = 2047;

double sinc(double x) { return (x == 0) ? 1 : sin(kPi * x) / (kPi * x); }
double rect(double x) {
  if (x < 0.5 && x > -0.5) return 1.0;
  if (x == 0.5 || x == -0.5) return 0.5;
  return 0.0;
}

// Raised-cosine windowed sinc of one LUT entry.
double rc_sinc(double x, double v, int npoints) {
  return sinc(x) * rect(x / (double)npoints) * cos(v * kPi * x) / (1.0 - (2.0 * v * x) * (2.0 * v * x));
}

// Normal-equation least squares with a lower Cholesky factor.
struct Chol {
  int n;
  std::vector<double> a;  // row-major, lower factor in the lower triangle
  bool factor() {
    bool ok = true;
    for (int i = 0; i < n; ++i)
      for (int j = i; j < n; ++j) {
        double s = a[i * n + j];
        for (int k = i - 1; k >= 0; --k) s -= a[i * n + k] * a[j * n + k];
        if (i == j) {
          if (s <= 0.) ok = false;
          a[i * n + i] = sqrt(s);
        } else {
          a[j * n + i] = s / a[i * n + i];
        }
      }
    return ok;
  }
  void solve(double *b) const {
    for (int i = 0; i < n; ++i) {
      double s = b[i];
      for (int j = i - 1; j >= 0; --j) s -= a[i * n + j] * b[j];
      b[i] = s / a[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = b[i];
      for (int j = i + 1; j < n; ++j) s -= a[j * n + i] * b[j];
      b[i] = s / a[i * n + i];
    }
  }
};

tops_poly interpolate_dc(double t, const tops_poly *list, int n) {
  int i0 = 0, i1 = 0;
  if (t < list[0].aztime) {
    i0 = 0;
    i1 = 1;
  } else if (t > list[n - 1].aztime) {
    i0 = n - 2;
    i1 = n - 1;  // the reference reads list[n] here (Func.cpp:1838-1839)
  } else {
    for (int i = 0; i < n - 1; i++)
      if (t >= list[i].aztime && t < list[i + 1].aztime) {
        i0 = i;
        i1 = i + 1;
        break;
      }
  }
  tops_poly r;
  r.aztime = t;
  r.t0 = list[i0].t0;
  double mu = (t - list[i0].aztime) / (list[i1].aztime - list[i0].aztime);
  r.c0 = (1 - mu) * list[i0].c0 + mu * list[i1].c0;
  r.c1 = (1 - mu) * list[i0].c1 + mu * list[i1].c1;
  r.c2 = (1 - mu) * list[i0].c2 + mu * list[i1].c2;
  return r;
}

}  // namespace

extern "C" {

int tops_lut(int npoints, double prf, double abw, double rsr2x, float *kaz, float *krg) {
  if (npoints <= 0 || !kaz || !krg || abw == 0.0 || prf == 0.0) return TOPS_E_INVALID;
  const double dx = 1.0 / kInterval;
  const int half = npoints / 2;
  // v = 1 - 1/CHI; the range kernel uses the azimuth bandwidth too
  // (reference quirk, Func.cpp:2111)
  const double v_az = 1. - 1. / (prf / abw);
  const double v_rg = 1. - 1. / ((rsr2x / 2.0) / abw);
  for (int i = 0; i <= kInterval; i++) {
    float *ra = kaz + (size_t)i * npoints, *rr = krg + (size_t)i * npoints;
    double sa = 0.0, sr = 0.0;
    for (int j = 0; j < npoints; j++) {
      const double x = 1.0 - half + j - dx * i;
      const double ca = rc_sinc(x, v_az, npoints), cr = rc_sinc(x, v_rg, npoints);
      sa += ca;
      sr += cr;
      ra[j] = (float)ca;
      rr[j] = (float)cr;
    }
    for (int j = 0; j < npoints; j++) {
      ra[j] = (float)((double)ra[j] / sa);
      rr[j] = (float)((double)rr[j] / sr);
    }
  }
  return TOPS_OK;
}

int tops_polyfit_orbit(int npts, const double *t, const double *x, const double *y,
                       const double *z, double *cx, double *cy, double *cz, int *ncoef) {
  if (npts < 3 || !t || !x || !y || !z || !cx || !cy || !cz) return TOPS_E_INVALID;
  const int nu = (npts > 6 ? 5 : npts - 2) + 1;
  std::vector<double> tn(npts), A((size_t)npts * nu);
  for (int i = 0; i < npts; i++) tn[i] = (t[i] - t[npts / 2]) / 10.0;
  for (int i = 0; i < npts; i++)
    for (int j = 0; j < nu; j++) A[(size_t)i * nu + j] = pow(tn[i], j);
  Chol C{nu, std::vector<double>((size_t)nu * nu)};
  for (int i = 0; i < nu; i++)
    for (int j = 0; j < nu; j++) {
      double s = 0.0;
      for (int k = 0; k < npts; k++) s += A[(size_t)k * nu + i] * A[(size_t)k * nu + j];
      C.a[i * nu + j] = s;
    }
  const double *src[3] = {x, y, z};
  double *dst[3] = {cx, cy, cz};
  std::vector<double> rhs(nu);
  for (int a = 0; a < 3; a++) {
    for (int i = 0; i < nu; i++) {
      double s = 0.0;
      for (int k = 0; k < npts; k++) s += A[(size_t)k * nu + i] * src[a][k];
      rhs[i] = s;
    }
    if (a == 0 && !C.factor()) return TOPS_E_NOT_PD;
    C.solve(rhs.data());
    for (int i = 0; i < nu; i++) dst[a][i] = rhs[i];
  }
  if (ncoef) *ncoef = nu;
  return TOPS_OK;
}

int tops_deramp_params(const tops_deramp_desc *d, double *dc, double *fmrate, double *reftime,
                       double *kt) {
  if (!d || !dc || !fmrate || !reftime || !kt || d->n_bursts <= 0 || d->samples_per_burst <= 0 ||
      !d->dc_list || !d->fm_list || d->n_dc < 2 || d->n_fm < d->n_bursts || !d->orb_cx ||
      !d->orb_cy || !d->orb_cz || d->orb_ncoef < 2 || !d->burst_first_line_time ||
      !d->burst_last_line_time || d->first_valid_pixel < 0 ||
      d->first_valid_pixel >= d->samples_per_burst)
    return TOPS_E_INVALID;
  const int nb = d->n_bursts, W = d->samples_per_burst;
  // per-burst Doppler centroid polynomial (Func.cpp:1938-1955)
  std::vector<tops_poly> dcb(nb);
  for (int b = 0; b < nb; b++)
    dcb[b] = (d->n_dc > nb)
                 ? d->dc_list[b]
                 : interpolate_dc(0.5 * (d->burst_first_line_time[b] + d->burst_last_line_time[b]),
                                  d->dc_list, d->n_dc);
  for (int b = 0; b < nb; b++) {
    const tops_poly &p = dcb[b], &f = d->fm_list[b];
    for (int x = 0; x < W; x++) {
      const double slrt = (d->slr_time_first_pixel + x * d->range_pixel_spacing / kSol) * 2;
      const double u = slrt - p.t0, v = slrt - f.t0;
      dc[(size_t)b * W + x] = p.c0 + p.c1 * u + p.c2 * (u * u);
      fmrate[(size_t)b * W + x] = f.c0 + f.c1 * v + f.c2 * v * v;
    }
  }
  // reference time (Func.cpp:2035-2056)
  const double half_burst = d->lines_per_burst * d->azimuth_time_interval / 2.0;
  for (int b = 0; b < nb; b++) {
    const size_t o = (size_t)b * W;
    const double t2 = half_burst + dc[o + d->first_valid_pixel] / fmrate[o + d->first_valid_pixel];
    for (int x = 0; x < W; x++) reftime[o + x] = t2 - dc[o + x] / fmrate[o + x];
  }
  // Doppler rate kt from the antenna steering (Func.cpp:2073-2091)
  const double tn = ((d->first_line_time + d->last_line_time) / 2.0 - d->orb_mid_time) / 10.0;
  double v[3] = {d->orb_cx[1], d->orb_cy[1], d->orb_cz[1]};
  for (int i = 2; i < d->orb_ncoef; ++i) {
    const double pw = (double)i * pow(tn, i - 1);
    v[0] += d->orb_cx[i] * pw;
    v[1] += d->orb_cy[i] * pw;
    v[2] += d->orb_cz[i] * pw;
  }
  for (int k = 0; k < 3; k++) v[k] /= (double)10.0;
  const double speed = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  const double krot = 2 * speed * (d->steering_rate_deg * kPi / 180.0) / d->wavelength;
  for (size_t k = 0; k < (size_t)nb * W; k++) kt[k] = fmrate[k] * krot / (fmrate[k] - krot);
  return TOPS_OK;
}

int tops_overlap_size(int n_bursts, const double *first_time, const double *last_time, double dt,
                      int *ov, int *total, int *maximum) {
  if (n_bursts < 1 || !first_time || !last_time || !ov || !total || !maximum || dt == 0.0)
    return TOPS_E_INVALID;
  *total = 0;
  *maximum = -9999;
  for (int i = 0; i + 1 < n_bursts; i++) {
    const int lines = (int)floor((last_time[i] - first_time[i + 1]) / dt);
    ov[i] = lines;
    *total += lines;
    if (lines > *maximum) *maximum = lines;
  }
  return TOPS_OK;
}

double tops_spectral_sep(int n_bursts, int W, int L, double dt, const double *kt) {
  const double tcycle = L * dt;
  double s = 0.0;
  for (int i = 0; i < n_bursts; i++)
    for (int p = 0; p < W; p++) s += kt[(size_t)i * W + p] * tcycle;
  return s / W / n_bursts;
}

// ------------------------------------------------------------ config.txt
int tops_config_defaults(tops_config *c) {
  if (!c) return TOPS_E_INVALID;
  memset(c, 0, sizeof(*c));
  strcpy(c->process_dir, ".");
  strcpy(c->polarisation, "vv");
  c->firstsubswath = 1;
  c->lastsubswath = 1;
  c->multi_az = 1;
  c->multi_rg = 1;
  c->burst0 = 1;
  c->burstN = 2;
  c->seed = 1;
  c->n_bursts = 2;
  c->lines_per_burst = 1500;
  c->samples_per_burst = 4096;
  c->overlap_lines = 100;
  c->dem_lines = 512;
  c->dem_pixels = 512;
  c->sigma_dn = 1000.0;
  c->az_shift_true = 0.0;
  c->coh_win_rg = 10;
  c->coh_win_az = 3;
  c->npoints = 12;
  c->esd_coh_threshold = 0.3;
  c->hbm_budget_gb = 150.0;
  c->arrival_rate = 40.0;
  c->n_jobs = 64;
  return TOPS_OK;
}

static bool parse_long(const char *s, long *out) {
  errno = 0;
  char *end;
  long v = strtol(s, &end, 10);
  if (end == s || errno) return false;
  while (*end == ' ' || *end == '\t' || *end == '\r') end++;
  if (*end) return false;
  *out = v;
  return true;
}

static bool parse_double(const char *s, double *out) {
  errno = 0;
  char *end;
  double v = strtod(s, &end);
  if (end == s || errno) return false;
  while (*end == ' ' || *end == '\t' || *end == '\r') end++;
  if (*end) return false;
  *out = v;
  return true;
}

// Tokenizer of the reference (Func.cpp:20-43): skip ' ', '\t', '='; a word
// runs until '\t', '=' or end of line.  Blank lines are skipped.
int tops_config_read(const char *path, tops_config *cfg, int *err_line) {
  if (!path || !cfg) return TOPS_E_INVALID;
  if (err_line) *err_line = 0;
  FILE *f = fopen(path, "r");
  if (!f) return TOPS_E_CONFIG;
  char line[2048];
  int lineno = 0, status = TOPS_OK;
  while (fgets(line, sizeof(line), f)) {
    lineno++;
    size_t n = strlen(line);
    while (n && (line[n - 1] == '\n' || line[n - 1] == '\r')) line[--n] = 0;
    const char *words[2] = {"", ""};
    char *c = line;
    for (int i = 0; i < 2; i++) {
      while (*c == ' ' || *c == '\t' || *c == '=') c++;
      words[i] = c;
      while (*c != '\t' && *c != '\0' && *c != '=') c++;
      if (*c != '\0') *c++ = '\0';
    }
    std::string key = words[0], val = words[1];
    while (!key.empty() && key.back() == ' ') key.pop_back();
    while (!val.empty() && (val.back() == ' ' || val.back() == '\t')) val.pop_back();
    if (key.empty() || key[0] == '#') continue;
    auto set_str = [&](char *dst, size_t cap) {
      snprintf(dst, cap, "%s", val.c_str());
    };
    auto set_int = [&](int *dst) {
      long v;
      if (!parse_long(val.c_str(), &v)) return false;
      *dst = (int)v;
      return true;
    };
    auto set_dbl = [&](double *dst) { return parse_double(val.c_str(), dst); };
    bool ok = true;
    if (key == "masterpath") set_str(cfg->masterpath, sizeof cfg->masterpath);
    else if (key == "slavepath") set_str(cfg->slavepath, sizeof cfg->slavepath);
    else if (key == "process_dir") set_str(cfg->process_dir, sizeof cfg->process_dir);
    else if (key == "polarisation") set_str(cfg->polarisation, sizeof cfg->polarisation);
    else if (key == "preciseOrbitMaster") set_str(cfg->preciseOrbitMaster, sizeof cfg->preciseOrbitMaster);
    else if (key == "preciseOrbitSlave") set_str(cfg->preciseOrbitSlave, sizeof cfg->preciseOrbitSlave);
    else if (key == "SpecificDemPath") set_str(cfg->SpecificDemPath, sizeof cfg->SpecificDemPath);
    else if (key == "firstsubswath") ok = set_int(&cfg->firstsubswath);
    else if (key == "lastsubswath") ok = set_int(&cfg->lastsubswath);
    else if (key == "multi_az") ok = set_int(&cfg->multi_az);
    else if (key == "multi_rg") ok = set_int(&cfg->multi_rg);
    else if (key == "burst0") ok = set_int(&cfg->burst0);
    else if (key == "burstN") ok = set_int(&cfg->burstN);
    else if (key == "seed") {
      long v;
      ok = parse_long(val.c_str(), &v);
      if (ok) cfg->seed = v;
    }
    else if (key == "n_bursts") ok = set_int(&cfg->n_bursts);
    else if (key == "lines_per_burst") ok = set_int(&cfg->lines_per_burst);
    else if (key == "samples_per_burst") ok = set_int(&cfg->samples_per_burst);
    else if (key == "overlap_lines") ok = set_int(&cfg->overlap_lines);
    else if (key == "dem_lines") ok = set_int(&cfg->dem_lines);
    else if (key == "dem_pixels") ok = set_int(&cfg->dem_pixels);
    else if (key == "sigma_dn") ok = set_dbl(&cfg->sigma_dn);
    else if (key == "az_shift_true") ok = set_dbl(&cfg->az_shift_true);
    else if (key == "coh_win_rg") ok = set_int(&cfg->coh_win_rg);
    else if (key == "coh_win_az") ok = set_int(&cfg->coh_win_az);
    else if (key == "npoints") ok = set_int(&cfg->npoints);
    else if (key == "esd_coh_threshold") ok = set_dbl(&cfg->esd_coh_threshold);
    else if (key == "hbm_budget_gb") ok = set_dbl(&cfg->hbm_budget_gb);
    else if (key == "arrival_rate") ok = set_dbl(&cfg->arrival_rate);
    else if (key == "n_jobs") ok = set_int(&cfg->n_jobs);
    else if (key == "stitch") ok = set_int(&cfg->stitch);
    // unknown keys are ignored, as in the reference
    if (!ok) {
      status = TOPS_E_CONFIG;
      break;
    }
  }
  fclose(f);
  if (status != TOPS_OK && err_line) *err_line = lineno;
  if (status == TOPS_OK) {
    if (cfg->burstN < cfg->burst0 || cfg->lastsubswath < cfg->firstsubswath ||
        cfg->lines_per_burst <= 0 || cfg->samples_per_burst <= 0 || cfg->n_bursts <= 0 ||
        cfg->coh_win_rg <= 0 || cfg->coh_win_az <= 0 || cfg->npoints != 12)
      status = TOPS_E_CONFIG;
  }
  return status;
}

}  // extern "C"

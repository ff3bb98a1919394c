// synth.cpp -- seeded synthetic Sentinel-1 TOPS burst pairs (see tops_synth.h).
//
// Geometry is FP64 throughout.  The slave image is built from the master's
// reflectivity by geocoding slave pixels through the DEM (coarse grid,
// bilinear in between), so the offsets the geometric coregistration must
// recover are implied by the two orbits and the terrain, as for real data.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "tops_synth.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kC = 299792458.0;
constexpr double kA = 6378137.0;
constexpr double kB = 6356752.3142451794975639665996337;
constexpr double kE2 = 1.0 - (kB * kB) / (kA * kA);
constexpr double kGM = 3.986004418e14;
constexpr double kWe = 7.2921159e-5;
constexpr double kTCenter = 50000.0;  // scene centre time, seconds of day
constexpr int kPad = 24;              // reflectivity grid margin

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------------ RNG
uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

struct Rng {  // xoshiro256**
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    for (int i = 0; i < 4; i++) s[i] = splitmix64(seed);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  void gauss2(double &a, double &b) {  // Box-Muller
    double u = uniform(), v = uniform();
    double r = sqrt(-2.0 * log(u));
    a = r * cos(2 * kPi * v);
    b = r * sin(2 * kPi * v);
  }
};

uint64_t stream_seed(long seed, uint64_t tag, uint64_t idx) {
  uint64_t x = (uint64_t)seed * 0x9e3779b97f4a7c15ULL ^ (tag << 48) ^ idx;
  splitmix64(x);
  return splitmix64(x);
}

// ------------------------------------------------------------ geometry
void llh2xyz(double lat, double lon, double h, double X[3]) {
  const double s = sin(lat), c = cos(lat);
  const double N = kA / sqrt(1.0 - kE2 * s * s);
  X[0] = (N + h) * c * cos(lon);
  X[1] = (N + h) * c * sin(lon);
  X[2] = (N * (1.0 - kE2) + h) * s;
}

void xyz2llh(const double X[3], double &lat, double &lon, double &h) {
  lon = atan2(X[1], X[0]);
  const double p = sqrt(X[0] * X[0] + X[1] * X[1]);
  lat = atan2(X[2], p * (1.0 - kE2));
  for (int i = 0; i < 6; i++) {
    const double s = sin(lat);
    const double N = kA / sqrt(1.0 - kE2 * s * s);
    h = p / cos(lat) - N;
    lat = atan2(X[2], p * (1.0 - kE2 * N / (N + h)));
  }
  const double s = sin(lat);
  h = p / cos(lat) - kA / sqrt(1.0 - kE2 * s * s);
}

double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double norm3(const double a[3]) { return sqrt(dot3(a, a)); }
void cross3(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Circular inertial orbit, expressed in the Earth-fixed frame.
struct Orbit {
  double Rs = 0, n = 0, incl = 0, Omega = 0, u0 = 0;
  double shift = 0;        // time shift, s
  double b_out = 0, b_rad = 0;   // baseline along the orbit normal / radial, m
  void eci(double t, double r[3]) const {
    const double u = u0 + n * (t - kTCenter + shift);
    const double e1[3] = {cos(Omega), sin(Omega), 0.0};
    const double e2[3] = {-sin(Omega) * cos(incl), cos(Omega) * cos(incl), sin(incl)};
    double nrm[3];
    cross3(e1, e2, nrm);
    const double cu = cos(u), su = sin(u);
    for (int k = 0; k < 3; k++) {
      const double rh = cu * e1[k] + su * e2[k];
      r[k] = (Rs + b_rad) * rh + b_out * nrm[k];
    }
  }
  void pos(double t, double r[3]) const {
    double q[3];
    eci(t, q);
    const double th = kWe * (t - kTCenter);
    const double c = cos(th), s = sin(th);
    r[0] = c * q[0] + s * q[1];
    r[1] = -s * q[0] + c * q[1];
    r[2] = q[2];
  }
  void pva(double t, double r[3], double v[3], double a[3]) const {
    const double h = 0.01;
    double rp[3], rm[3];
    pos(t, r);
    pos(t + h, rp);
    pos(t - h, rm);
    for (int k = 0; k < 3; k++) {
      v[k] = (rp[k] - rm[k]) / (2 * h);
      a[k] = (rp[k] - 2 * r[k] + rm[k]) / (h * h);
    }
  }
  // zero-Doppler time and range of ground point X, starting at t0
  void zero_doppler(const double X[3], double t0, double &t, double &R) const {
    t = t0;
    double r[3], v[3], a[3], d[3];
    for (int it = 0; it < 12; it++) {
      pva(t, r, v, a);
      for (int k = 0; k < 3; k++) d[k] = X[k] - r[k];
      const double f = dot3(v, d), fp = dot3(a, d) - dot3(v, v);
      const double step = -f / fp;
      t += step;
      if (fabs(step) < 1e-12) break;
    }
    pos(t, r);
    for (int k = 0; k < 3; k++) d[k] = X[k] - r[k];
    R = norm3(d);
  }
};

struct Dem {
  int lines = 0, pixels = 0;
  double lat0 = 0, lon0 = 0, dlat = 0, dlon = 0;  // degrees
  std::vector<float> h;
  double height(double lat_deg, double lon_deg) const {
    double fr = (lat0 - lat_deg) / dlat, fc = (lon_deg - lon0) / dlon;
    fr = std::min(std::max(fr, 0.0), (double)lines - 1.001);
    fc = std::min(std::max(fc, 0.0), (double)pixels - 1.001);
    const int r = (int)fr, c = (int)fc;
    const double a = fr - r, b = fc - c;
    const float *p = h.data() + (size_t)r * pixels + c;
    return (1 - a) * ((1 - b) * p[0] + b * p[1]) + a * ((1 - b) * p[pixels] + b * p[pixels + 1]);
  }
};

// Ground point seen at azimuth time t and slant range R (right looking),
// with terrain height from the DEM (dem may be null: constant height h0).
// Points X(a) = r + R (cos a e1 + sin a e2) on the zero-Doppler range circle
// satisfy the range and Doppler equations exactly; the look angle a is found
// by bisection on (ellipsoidal height - terrain height), which decreases
// monotonically with a away from layover.
bool geocode(const Orbit &O, double t, double R, const Dem *dem, double h0, double X[3]) {
  double r[3], v[3], a[3];
  O.pva(t, r, v, a);
  const double vn = norm3(v), rs = norm3(r);
  double vh[3] = {v[0] / vn, v[1] / vn, v[2] / vn};
  // e1: nadir direction projected orthogonal to v; e2 = v x e1 points right
  double e1[3] = {-r[0] / rs, -r[1] / rs, -r[2] / rs};
  const double pr = dot3(e1, vh);
  for (int k = 0; k < 3; k++) e1[k] -= pr * vh[k];
  const double n1 = norm3(e1);
  for (int k = 0; k < 3; k++) e1[k] /= n1;
  double e2[3];
  cross3(vh, e1, e2);
  // orientation check: right of the velocity is v x r / |v x r|
  double right[3];
  cross3(v, r, right);
  if (dot3(right, e2) < 0)
    for (int k = 0; k < 3; k++) e2[k] = -e2[k];
  auto point = [&](double al, double P[3]) {
    const double c = cos(al), s = sin(al);
    for (int k = 0; k < 3; k++) P[k] = r[k] + R * (c * e1[k] + s * e2[k]);
  };
  auto f = [&](double al) {
    double P[3], la, lo, hh;
    point(al, P);
    xyz2llh(P, la, lo, hh);
    const double terrain = dem ? dem->height(la * 180.0 / kPi, lo * 180.0 / kPi) : h0;
    return hh - terrain;
  };
  // flat-earth look angle for the initial bracket
  const double Re = 6371000.0;
  double ca = (rs * rs + R * R - Re * Re) / (2 * rs * R);
  ca = std::min(std::max(ca, -1.0), 1.0);
  const double a0 = acos(ca);
  double lo_a = a0 - 0.05, hi_a = a0 + 0.05;
  double flo = f(lo_a), fhi = f(hi_a);
  if (!(flo > 0 && fhi < 0)) {
    point(a0, X);
    return false;
  }
  for (int it = 0; it < 60 && hi_a - lo_a > 1e-12; it++) {
    const double mid = 0.5 * (lo_a + hi_a);
    const double fm = f(mid);
    if (fm > 0)
      lo_a = mid;
    else
      hi_a = mid;
  }
  point(0.5 * (lo_a + hi_a), X);
  return true;
}

// ---------------------------------------------------------------- DEM
void make_fbm(int lines, int pixels, double hurst, double hmin, double hmax, long seed,
              std::vector<float> &out) {
  int n = 1;
  while (n + 1 < std::max(lines, pixels)) n <<= 1;
  const int N = n + 1;
  std::vector<double> g((size_t)N * N, 0.0);
  Rng rng(stream_seed(seed, 7, 0));
  auto at = [&](int r, int c) -> double & { return g[(size_t)r * N + c]; };
  double a, b;
  rng.gauss2(a, b);
  at(0, 0) = a;
  at(0, n) = b;
  rng.gauss2(a, b);
  at(n, 0) = a;
  at(n, n) = b;
  double amp = 1.0;
  for (int step = n; step > 1; step >>= 1) {
    const int hs = step / 2;
    amp *= pow(0.5, hurst);
    for (int r = hs; r < N; r += step)
      for (int c = hs; c < N; c += step) {
        rng.gauss2(a, b);
        at(r, c) = 0.25 * (at(r - hs, c - hs) + at(r - hs, c + hs) + at(r + hs, c - hs) +
                           at(r + hs, c + hs)) + amp * a;
      }
    for (int r = 0; r < N; r += hs)
      for (int c = ((r / hs) % 2 == 0) ? hs : 0; c < N; c += step) {
        double s = 0;
        int k = 0;
        if (r >= hs) { s += at(r - hs, c); k++; }
        if (r + hs < N) { s += at(r + hs, c); k++; }
        if (c >= hs) { s += at(r, c - hs); k++; }
        if (c + hs < N) { s += at(r, c + hs); k++; }
        rng.gauss2(a, b);
        at(r, c) = s / k + amp * a;
      }
  }
  double lo = 1e300, hi = -1e300;
  for (int r = 0; r < lines; r++)
    for (int c = 0; c < pixels; c++) {
      lo = std::min(lo, at(r, c));
      hi = std::max(hi, at(r, c));
    }
  out.resize((size_t)lines * pixels);
  const double sc = (hi > lo) ? (hmax - hmin) / (hi - lo) : 0.0;
  for (int r = 0; r < lines; r++)
    for (int c = 0; c < pixels; c++)
      out[(size_t)r * pixels + c] = (float)(hmin + (at(r, c) - lo) * sc);
}

// Kaiser-windowed low-pass FIR (cutoff in cycles/sample), unit DC gain.
std::vector<float> lowpass(double fc, int taps) {
  std::vector<float> h(taps);
  const double beta = 5.0, m = (taps - 1) / 2.0;
  auto i0 = [](double x) {
    double s = 1, t = 1;
    for (int k = 1; k < 30; k++) {
      t *= (x / (2 * k)) * (x / (2 * k));
      s += t;
    }
    return s;
  };
  double sum = 0;
  for (int k = 0; k < taps; k++) {
    const double x = k - m, u = x / m;
    const double s = (x == 0) ? 2 * fc : sin(2 * kPi * fc * x) / (kPi * x);
    const double w = i0(beta * sqrt(std::max(0.0, 1 - u * u))) / i0(beta);
    h[k] = (float)(s * w);
    sum += s * w;
  }
  for (auto &v : h) v = (float)(v / sum);
  return h;
}

// Windowed-sinc interpolation weights at fractional offset f for `taps`
// samples starting at floor(x) - taps/2 + 1.
inline void interp_weights(double f, int taps, double *w) {
  const int half = taps / 2;
  double sum = 0;
  const double sp = sin(kPi * f);
  for (int k = 0; k < taps; k++) {
    const double x = f + (half - 1) - k;  // distance from sample k
    double s;
    if (fabs(x) < 1e-12)
      s = 1.0;
    else
      s = (((half - 1 - k) & 1) ? -sp : sp) / (kPi * x);
    const double u = x / (half + 0.5);
    const double win = (fabs(u) < 1) ? 0.5 * (1 + cos(kPi * u)) : 0.0;
    w[k] = s * win;
    sum += w[k];
  }
  for (int k = 0; k < taps; k++) w[k] /= sum;
}

int16_t sat16(double v) {
  v = nearbyint(v);
  if (v > 32767) v = 32767;
  if (v < -32768) v = -32768;
  return (int16_t)v;
}

}  // namespace

struct tops_scene {
  tops_synth_cfg cfg;
  tops_swath_info sw[2];
  Orbit orb[2];
  Dem dem;
  std::vector<int16_t> slc[2];
  std::vector<double> truth[TOPS_SYNTH_MAX_BURSTS];
  std::vector<double> kt[2], tref[2], fdc[2];
  double timing[5] = {0, 0, 0, 0, 0};
};

extern "C" {

int tops_synth_defaults(tops_synth_cfg *c) {
  if (!c) return TOPS_E_INVALID;
  memset(c, 0, sizeof(*c));
  c->seed = 1;
  c->n_bursts = 2;
  c->lines_per_burst = 1500;
  c->samples_per_burst = 4096;
  c->overlap_lines = 100;
  c->sigma_dn = 1000.0;
  c->wavelength = 0.05547;
  c->dt = 2.055e-3;
  c->rsr = 64.345e6;
  c->steering_rate_deg = 1.59;
  c->az_bandwidth = 327.0;
  c->rg_bandwidth = 56.5e6;
  c->altitude = 693000.0;
  c->inc_mid_deg = 35.0;
  c->lat_center_deg = 38.0;
  c->dem_lines = 512;
  c->dem_pixels = 512;
  c->hurst = 0.8;
  c->h_min = 0.0;
  c->h_max = 1500.0;
  c->dem_spacing_arcsec = 1.0;
  c->bperp = 40.0;
  c->bpar = -4.0;
  c->along_track_s = -0.3 * 2.055e-3;
  c->az_shift_true = 0.0;
  c->topo_phase = 1;
  c->interp_taps = 16;
  c->threads = 0;
  return TOPS_OK;
}

void tops_synth_destroy(tops_scene *s) { delete s; }

int tops_synth_create(const tops_synth_cfg *cfg, tops_scene **out) {
  if (!cfg || !out) return TOPS_E_INVALID;
  const int nb = cfg->n_bursts, L = cfg->lines_per_burst, W = cfg->samples_per_burst,
            ov = cfg->overlap_lines;
  if (nb < 1 || nb > TOPS_SYNTH_MAX_BURSTS || L < 64 || W < 64 || ov < 1 || ov >= L / 2 ||
      cfg->dem_lines < 64 || cfg->dem_pixels < 64 || cfg->interp_taps < 4 ||
      cfg->interp_taps > 32 || (cfg->interp_taps & 1))
    return TOPS_E_INVALID;
#ifdef _OPENMP
  if (cfg->threads > 0) omp_set_num_threads(cfg->threads);
#endif
  tops_scene *S = new tops_scene();
  S->cfg = *cfg;
  double t0 = now_s();

  // ---- orbits
  const double Rs = kA + cfg->altitude;
  Orbit &M = S->orb[0];
  M.Rs = Rs;
  M.n = sqrt(kGM / (Rs * Rs * Rs));
  M.incl = 98.18 * kPi / 180.0;
  M.Omega = 0.3;
  M.u0 = asin(sin(cfg->lat_center_deg * kPi / 180.0) / sin(M.incl));
  // look angle at mid swath, baseline components in the orbit frame
  const double Re = 6371000.0, inc = cfg->inc_mid_deg * kPi / 180.0;
  const double look = asin(Re / Rs * sin(inc));
  const double R_mid = Rs * cos(look) - sqrt(Re * Re - Rs * Rs * sin(look) * sin(look));
  Orbit &Sl = S->orb[1];
  Sl = M;
  Sl.shift = cfg->along_track_s;
  // right-looking: the look vector points along -normal (v x r) and -radial
  Sl.b_out = -(cfg->bpar * sin(look) + cfg->bperp * cos(look));
  Sl.b_rad = -cfg->bpar * cos(look) + cfg->bperp * sin(look);

  // ---- swath timing and sampling
  const double dt = cfg->dt, dr = kC / (2.0 * cfg->rsr);
  const double tcyc = (L - ov - 1) * dt - 1e-6 * dt;
  const double span = (nb - 1) * tcyc + (L - 1) * dt;
  const double t_start = kTCenter - span / 2;
  for (int w = 0; w < 2; w++) {
    tops_swath_info &I = S->sw[w];
    memset(&I, 0, sizeof(I));
    I.n_bursts = nb;
    I.lines_per_burst = L;
    I.samples_per_burst = W;
    I.first_valid_pixel = 0;
    I.dt = dt;
    I.prf = 1.0 / dt;
    I.range_spacing = dr;
    I.slr_time = (R_mid - 0.5 * W * dr) / kC;
    I.wavelength = cfg->wavelength;
    I.rsr = cfg->rsr;
    I.az_bandwidth = cfg->az_bandwidth;
    I.steering_rate_deg = cfg->steering_rate_deg;
    for (int b = 0; b < nb; b++) {
      I.burst_first_line_time[b] = t_start + b * tcyc;
      I.burst_last_line_time[b] = I.burst_first_line_time[b] + (L - 1) * dt;
    }
    I.first_line_time = I.burst_first_line_time[0];
    I.last_line_time = I.burst_last_line_time[nb - 1];
    const double t0w = 2 * (I.slr_time + 0.5 * W * dr / kC);
    I.n_dc = nb + 2;
    I.n_fm = nb + 2;
    for (int k = 0; k < nb + 2; k++) {
      const double tc = t_start + (k - 1) * tcyc + 0.5 * (L - 1) * dt;
      const double kk = k - 1 + 0.37 * w;
      I.dc_list[k] = tops_poly{tc, t0w, 25.0 + 3.0 * sin(0.7 * kk), 3.0e4, 0.0};
      I.fm_list[k] = tops_poly{tc, t0w, -2300.0 + 1.5 * kk, 4.3e5, -7.6e7};
    }
    I.n_sv = 17;
    for (int k = 0; k < 17; k++) {
      const double t = kTCenter + (k - 8) * 10.0;
      double r[3];
      S->orb[w].pos(t, r);
      I.sv_t[k] = t;
      I.sv_x[k] = r[0];
      I.sv_y[k] = r[1];
      I.sv_z[k] = r[2];
    }
    // deramp parameters with the product's host code (needed for the ramps)
    double cx[8], cy[8], cz[8];
    int nc = 0;
    tops_polyfit_orbit(17, I.sv_t, I.sv_x, I.sv_y, I.sv_z, cx, cy, cz, &nc);
    tops_deramp_desc d;
    memset(&d, 0, sizeof(d));
    d.n_bursts = nb;
    d.samples_per_burst = W;
    d.lines_per_burst = L;
    d.first_valid_pixel = 0;
    d.slr_time_first_pixel = I.slr_time;
    d.range_pixel_spacing = dr;
    d.azimuth_time_interval = dt;
    d.first_line_time = I.first_line_time;
    d.last_line_time = I.last_line_time;
    d.steering_rate_deg = I.steering_rate_deg;
    d.wavelength = I.wavelength;
    d.burst_first_line_time = I.burst_first_line_time;
    d.burst_last_line_time = I.burst_last_line_time;
    d.dc_list = I.dc_list;
    d.n_dc = I.n_dc;
    d.fm_list = I.fm_list;
    d.n_fm = I.n_fm;
    d.orb_cx = cx;
    d.orb_cy = cy;
    d.orb_cz = cz;
    d.orb_ncoef = nc;
    d.orb_mid_time = I.sv_t[8];
    std::vector<double> dc((size_t)nb * W), fm((size_t)nb * W);
    S->kt[w].resize((size_t)nb * W);
    S->tref[w].resize((size_t)nb * W);
    tops_deramp_params(&d, dc.data(), fm.data(), S->tref[w].data(), S->kt[w].data());
    S->fdc[w] = dc;
  }

  // ---- DEM covering the swath footprint
  {
    const tops_swath_info &I = S->sw[0];
    double lamin = 1e9, lamax = -1e9, lomin = 1e9, lomax = -1e9;
    for (int b = 0; b < nb; b++)
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 3; c++)
          for (double hh : {cfg->h_min, cfg->h_max}) {
            const double t = I.burst_first_line_time[b] + 0.5 * a * (L - 1) * dt;
            const double R = I.slr_time * kC + 0.5 * c * (W - 1) * dr;
            double X[3], la, lo, he;
            geocode(M, t, R, nullptr, hh, X);
            xyz2llh(X, la, lo, he);
            la *= 180.0 / kPi;
            lo *= 180.0 / kPi;
            lamin = std::min(lamin, la);
            lamax = std::max(lamax, la);
            lomin = std::min(lomin, lo);
            lomax = std::max(lomax, lo);
          }
    const int margin = 40;
    Dem &D = S->dem;
    D.lines = cfg->dem_lines;
    D.pixels = cfg->dem_pixels;
    const double req = cfg->dem_spacing_arcsec / 3600.0;
    D.dlat = std::max(req, (lamax - lamin) / (D.lines - 2 * margin));
    D.dlon = std::max(req, (lomax - lomin) / (D.pixels - 2 * margin));
    D.lat0 = 0.5 * (lamax + lamin) + 0.5 * (D.lines - 1) * D.dlat;
    D.lon0 = 0.5 * (lomax + lomin) - 0.5 * (D.pixels - 1) * D.dlon;
    make_fbm(D.lines, D.pixels, cfg->hurst, cfg->h_min, cfg->h_max, cfg->seed, D.h);
  }
  double t1 = now_s();
  S->timing[0] = t1 - t0;

  // ---- band-limited reflectivity on the ground grid (float complex)
  const int GL = (nb - 1) * (L - ov - 1) + L + 2 * kPad, GW = W + 2 * kPad;
  std::vector<float> Z((size_t)GL * GW * 2);
  {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < GL; r++) {
      Rng rng(stream_seed(cfg->seed, 1, (uint64_t)r));
      float *row = Z.data() + (size_t)r * GW * 2;
      for (int c = 0; c < GW; c++) {
        double a, b;
        rng.gauss2(a, b);
        row[2 * c] = (float)a;
        row[2 * c + 1] = (float)b;
      }
    }
    const std::vector<float> haz = lowpass(0.5 * cfg->az_bandwidth * dt, 31);
    const std::vector<float> hrg = lowpass(0.5 * cfg->rg_bandwidth / cfg->rsr, 31);
    double eaz = 0, erg = 0;
    for (float v : haz) eaz += (double)v * v;
    for (float v : hrg) erg += (double)v * v;
    const float scale = (float)(cfg->sigma_dn / sqrt(2.0) / sqrt(eaz * erg));
    // range pass (per row)
#pragma omp parallel
    {
      std::vector<float> tmp((size_t)GW * 2);
#pragma omp for schedule(static)
      for (int r = 0; r < GL; r++) {
        float *row = Z.data() + (size_t)r * GW * 2;
        memcpy(tmp.data(), row, sizeof(float) * 2 * GW);
        for (int c = 0; c < GW; c++) {
          float re = 0, im = 0;
          for (int k = 0; k < 31; k++) {
            int cc = c + k - 15;
            if (cc < 0 || cc >= GW) continue;
            re += hrg[k] * tmp[2 * cc];
            im += hrg[k] * tmp[2 * cc + 1];
          }
          row[2 * c] = re;
          row[2 * c + 1] = im;
        }
      }
    }
    // azimuth pass (blocks of columns)
    const int CB = 64;
#pragma omp parallel
    {
      std::vector<float> tmp((size_t)GL * CB * 2);
#pragma omp for schedule(static)
      for (int c0 = 0; c0 < GW; c0 += CB) {
        const int cn = std::min(CB, GW - c0);
        for (int r = 0; r < GL; r++)
          memcpy(&tmp[(size_t)r * CB * 2], Z.data() + ((size_t)r * GW + c0) * 2,
                 sizeof(float) * 2 * cn);
        for (int r = 0; r < GL; r++)
          for (int c = 0; c < cn; c++) {
            float re = 0, im = 0;
            for (int k = 0; k < 31; k++) {
              int rr = r + k - 15;
              if (rr < 0 || rr >= GL) continue;
              re += haz[k] * tmp[((size_t)rr * CB + c) * 2];
              im += haz[k] * tmp[((size_t)rr * CB + c) * 2 + 1];
            }
            Z[((size_t)r * GW + c0 + c) * 2] = re * scale;
            Z[((size_t)r * GW + c0 + c) * 2 + 1] = im * scale;
          }
      }
    }
  }
  double t2 = now_s();
  S->timing[1] = t2 - t1;

  // ---- master: reflectivity with the master TOPS ramp
  auto ramp = [&](int w, int b, double l, int x) {
    const size_t k = (size_t)b * W + x;
    const double ta = l * dt, e = ta - S->tref[w][k];
    return -kPi * S->kt[w][k] * e * e - 2.0 * kPi * S->fdc[w][k] * ta;
  };
  S->slc[0].resize((size_t)nb * L * W * 2);
  S->slc[1].resize((size_t)nb * L * W * 2);
#pragma omp parallel for collapse(2) schedule(static)
  for (int b = 0; b < nb; b++)
    for (int l = 0; l < L; l++) {
      const float *zr = Z.data() + ((size_t)(kPad + b * (L - ov - 1) + l) * GW + kPad) * 2;
      int16_t *o = S->slc[0].data() + ((size_t)(b * L + l) * W) * 2;
      for (int x = 0; x < W; x++) {
        const double ph = -ramp(0, b, l, x);
        const double c = cos(ph), s = sin(ph);
        o[2 * x] = sat16(zr[2 * x] * c - zr[2 * x + 1] * s);
        o[2 * x + 1] = sat16(zr[2 * x] * s + zr[2 * x + 1] * c);
      }
    }
  double t3 = now_s();
  S->timing[2] = t3 - t2;

  // ---- slave geometry on a coarse grid: slave pixel -> master pixel, phase
  const int GS_L = 8, GS_W = 32;
  const int nl = (L - 1) / GS_L + 2, nw = (W - 1) / GS_W + 2;
  std::vector<double> node((size_t)nb * nl * nw * 3);
  for (int b = 0; b < nb; b++) S->truth[b].assign((size_t)nl * nw * 4, 0.0);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int b = 0; b < nb; b++)
    for (int i = 0; i < nl; i++) {
      const tops_swath_info &I = S->sw[1];
      const double ls = std::min(i * GS_L, L - 1) + (i == nl - 1 ? 0.0 : 0.0);
      const double tsl = I.burst_first_line_time[b] + ls * dt;
      for (int j = 0; j < nw; j++) {
        const double xs = std::min(j * GS_W, W - 1);
        const double Rs_ = I.slr_time * kC + xs * dr;
        double X[3];
        geocode(S->orb[1], tsl, Rs_, &S->dem, 0.5 * (cfg->h_min + cfg->h_max), X);
        double tm, Rm;
        M.zero_doppler(X, tsl, tm, Rm);
        const double lm = (tm - S->sw[0].burst_first_line_time[b]) / dt;
        const double xm = (Rm - S->sw[0].slr_time * kC) / dr;
        const double th = cfg->topo_phase ? -4.0 * kPi / cfg->wavelength * (Rs_ - Rm) : 0.0;
        double *nd = node.data() + (((size_t)b * nl + i) * nw + j) * 3;
        nd[0] = lm;
        nd[1] = xm;
        nd[2] = th;
        double *tr = S->truth[b].data() + ((size_t)i * nw + j) * 4;
        tr[0] = b * L + lm;
        tr[1] = xm;
        tr[2] = b * L + ls;
        tr[3] = xs;
      }
    }
  double t4 = now_s();
  S->timing[3] = t4 - t3;

  // ---- slave: resample the reflectivity at the geocoded positions
  const int taps = cfg->interp_taps, half = taps / 2;
  const double dshift = cfg->az_shift_true;
#pragma omp parallel for collapse(2) schedule(static)
  for (int b = 0; b < nb; b++)
    for (int l = 0; l < L; l++) {
      const int i = std::min(l / GS_L, nl - 2);
      const double l_lo = std::min(i * GS_L, L - 1), l_hi = std::min((i + 1) * GS_L, L - 1);
      const double fa = (l_hi > l_lo) ? (l - l_lo) / (l_hi - l_lo) : 0.0;
      int16_t *o = S->slc[1].data() + ((size_t)(b * L + l) * W) * 2;
      double wa[32], wr[32];
      for (int x = 0; x < W; x++) {
        const int j = std::min(x / GS_W, nw - 2);
        const double x_lo = std::min(j * GS_W, W - 1), x_hi = std::min((j + 1) * GS_W, W - 1);
        const double fb = (x_hi > x_lo) ? (x - x_lo) / (x_hi - x_lo) : 0.0;
        const double *n00 = node.data() + (((size_t)b * nl + i) * nw + j) * 3;
        const double *n01 = n00 + 3, *n10 = n00 + (size_t)nw * 3, *n11 = n10 + 3;
        double v[3];
        for (int k = 0; k < 3; k++)
          v[k] = (1 - fa) * ((1 - fb) * n00[k] + fb * n01[k]) + fa * ((1 - fb) * n10[k] + fb * n11[k]);
        const double g = kPad + b * (L - ov - 1) + v[0] + dshift, c = kPad + v[1];
        const int gi = (int)floor(g), ci = (int)floor(c);
        interp_weights(g - gi, taps, wa);
        interp_weights(c - ci, taps, wr);
        double re = 0, im = 0;
        for (int a = 0; a < taps; a++) {
          const int rr = std::min(std::max(gi - half + 1 + a, 0), GL - 1);
          const float *zr = Z.data() + (size_t)rr * GW * 2;
          double tre = 0, tim = 0;
          for (int q = 0; q < taps; q++) {
            const int cc = std::min(std::max(ci - half + 1 + q, 0), GW - 1);
            tre += wr[q] * zr[2 * cc];
            tim += wr[q] * zr[2 * cc + 1];
          }
          re += wa[a] * tre;
          im += wa[a] * tim;
        }
        // A ground point keeps the Doppler history it has in the master burst
        // (same burst synchronisation): the slave sample carries the master
        // ramp at the point's master position, shifted by the injected
        // misregistration, plus the topographic phase.
        const double xm = std::min(std::max(v[1], 0.0), (double)W - 1.0);
        const int x0 = std::min((int)xm, W - 2);
        const double fx = xm - x0;
        const double ph0 = ramp(0, b, v[0] + dshift, x0), ph1 = ramp(0, b, v[0] + dshift, x0 + 1);
        const double ph = -((1 - fx) * ph0 + fx * ph1) + v[2];
        const double cs = cos(ph), sn = sin(ph);
        o[2 * x] = sat16(re * cs - im * sn);
        o[2 * x + 1] = sat16(re * sn + im * cs);
      }
    }
  S->timing[4] = now_s() - t4;
  *out = S;
  return TOPS_OK;
}

int tops_synth_swath(const tops_scene *s, int which, tops_swath_info *info) {
  if (!s || !info || which < 0 || which > 1) return TOPS_E_INVALID;
  *info = s->sw[which];
  return TOPS_OK;
}

const int16_t *tops_synth_slc(const tops_scene *s, int which) {
  if (!s || which < 0 || which > 1) return nullptr;
  return s->slc[which].data();
}

const float *tops_synth_dem(const tops_scene *s, tops_dem_info *info) {
  if (!s) return nullptr;
  if (info) {
    info->lines = s->dem.lines;
    info->pixels = s->dem.pixels;
    info->lat0 = s->dem.lat0;
    info->lon0 = s->dem.lon0;
    info->dlat = s->dem.dlat;
    info->dlon = s->dem.dlon;
  }
  return s->dem.h.data();
}

int tops_synth_burst_dem_window(const tops_scene *s, int burst, int margin, int *row0, int *col0,
                                int *rows, int *cols) {
  if (!s || burst < 0 || burst >= s->cfg.n_bursts || !row0 || !col0 || !rows || !cols)
    return TOPS_E_INVALID;
  const tops_swath_info &I = s->sw[0];
  const int L = I.lines_per_burst, W = I.samples_per_burst;
  double lamin = 1e9, lamax = -1e9, lomin = 1e9, lomax = -1e9;
  for (int a = 0; a < 3; a++)
    for (int c = 0; c < 3; c++)
      for (double hh : {s->cfg.h_min, s->cfg.h_max}) {
        const double t = I.burst_first_line_time[burst] + 0.5 * a * (L - 1) * I.dt;
        const double R = I.slr_time * kC + 0.5 * c * (W - 1) * I.range_spacing;
        double X[3], la, lo, he;
        geocode(s->orb[0], t, R, nullptr, hh, X);
        xyz2llh(X, la, lo, he);
        la *= 180.0 / kPi;
        lo *= 180.0 / kPi;
        lamin = std::min(lamin, la);
        lamax = std::max(lamax, la);
        lomin = std::min(lomin, lo);
        lomax = std::max(lomax, lo);
      }
  const Dem &D = s->dem;
  // RefDem::getData: extend by margin pixels, floor the upper-left and ceil
  // the lower-right DEM indexes (DataTypes.cpp:278-293)
  lamin -= margin * D.dlat;
  lamax += margin * D.dlat;
  lomin -= margin * D.dlon;
  lomax += margin * D.dlon;
  int r0 = (int)floor((D.lat0 - lamax) / D.dlat), c0 = (int)floor((lomin - D.lon0) / D.dlon);
  int r1 = (int)ceil((D.lat0 - lamin) / D.dlat), c1 = (int)ceil((lomax - D.lon0) / D.dlon);
  r0 = std::max(r0, 0);
  c0 = std::max(c0, 0);
  r1 = std::min(r1, D.lines - 1);
  c1 = std::min(c1, D.pixels - 1);
  if (r1 < r0 || c1 < c0) return TOPS_E_INVALID;
  *row0 = r0;
  *col0 = c0;
  *rows = r1 - r0 + 1;
  *cols = c1 - c0 + 1;
  return TOPS_OK;
}

int tops_synth_truth(const tops_scene *s, int burst, long *n, const double **nodes) {
  if (!s || burst < 0 || burst >= s->cfg.n_bursts || !n || !nodes) return TOPS_E_INVALID;
  *n = (long)(s->truth[burst].size() / 4);
  *nodes = s->truth[burst].data();
  return TOPS_OK;
}

int tops_synth_timing(const tops_scene *s, double t[5]) {
  if (!s || !t) return TOPS_E_INVALID;
  for (int i = 0; i < 5; i++) t[i] = s->timing[i];
  return TOPS_OK;
}

}  // extern "C"

// pipeline.cpp -- burst-pair processing of one sub-swath (tops_pipeline.h).
//
// tops_pair_*: device-resident plan.  Stage order and per-burst semantics
// follow the reference drivers (Func.cpp:2215-2297, 2326-2406, 2496-2763);
// every stage is one batched launch over the bursts and the offset
// polynomials / ESD shifts stay on the device between stages.
//
// tops_plain_pair: the same drivers, per burst, through the reference-
// compatible entry points with host buffers.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "launch.h"
#include "pair_impl.h"

namespace {

int fit_orbit(const tops_swath_info &s, OrbitFit &f) {
  return tops_polyfit_orbit(s.n_sv, s.sv_t, s.sv_x, s.sv_y, s.sv_z, f.cx, f.cy, f.cz, &f.n);
}

int deramp_of(const tops_swath_info &s, const OrbitFit &f, Deramp &d) {
  const size_t n = (size_t)s.n_bursts * s.samples_per_burst;
  d.dc.resize(n);
  d.fm.resize(n);
  d.tref.resize(n);
  d.kt.resize(n);
  tops_deramp_desc x;
  memset(&x, 0, sizeof(x));
  x.n_bursts = s.n_bursts;
  x.samples_per_burst = s.samples_per_burst;
  x.lines_per_burst = s.lines_per_burst;
  x.first_valid_pixel = s.first_valid_pixel;
  x.slr_time_first_pixel = s.slr_time;
  x.range_pixel_spacing = s.range_spacing;
  x.azimuth_time_interval = s.dt;
  x.first_line_time = s.first_line_time;
  x.last_line_time = s.last_line_time;
  x.steering_rate_deg = s.steering_rate_deg;
  x.wavelength = s.wavelength;
  x.burst_first_line_time = s.burst_first_line_time;
  x.burst_last_line_time = s.burst_last_line_time;
  x.dc_list = s.dc_list;
  x.n_dc = s.n_dc;
  x.fm_list = s.fm_list;
  x.n_fm = s.n_fm;
  x.orb_cx = f.cx;
  x.orb_cy = f.cy;
  x.orb_cz = f.cz;
  x.orb_ncoef = f.n;
  x.orb_mid_time = s.sv_t[s.n_sv / 2];
  return tops_deramp_params(&x, d.dc.data(), d.fm.data(), d.tref.data(), d.kt.data());
}

#define P_TRY(expr)               \
  do {                            \
    int _s = (expr);              \
    if (_s != TOPS_OK) return _s; \
  } while (0)

#define P_CUDA(expr)                                                              \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      (void)cudaGetLastError();                                                   \
      return _e == cudaErrorMemoryAllocation ? TOPS_E_NOMEM : TOPS_E_CUDA;        \
    }                                                                             \
  } while (0)

}  // namespace

extern "C" {

int tops_pair_opts_default(tops_pair_opts *o) {
  if (!o) return TOPS_E_INVALID;
  o->win_rg = 10;
  o->win_az = 3;
  o->esd_threshold = 0.3f;
  o->reslave_full = 1;
  o->burst0_deramp_rows = 1;
  o->precision = TOPS_PREC_SPLIT;
  o->compensated = 0;
  o->coh_overlap = 0;
  return TOPS_OK;
}

static void pitches(int W, int dem_pixels, size_t &slc, size_t &cplx, size_t &coh, size_t &dem) {
  slc = align_up((size_t)W * 4, 512);
  cplx = align_up((size_t)W * 8, 512);
  coh = align_up((size_t)W * 4, 512);
  dem = align_up((size_t)dem_pixels * 4, 512);
}

size_t tops_pair_footprint(const tops_swath_info *m, const tops_pair_opts *o, int dem_lines,
                           int dem_pixels) {
  if (!m || !o) return 0;
  const int nb = m->n_bursts, L = m->lines_per_burst, W = m->samples_per_burst;
  size_t slc, cplx, coh, dem;
  pitches(W, dem_pixels, slc, cplx, coh, dem);
  const size_t lines = (size_t)nb * L;
  size_t b = 2 * lines * slc + lines * cplx + lines * coh + (size_t)dem_lines * dem;
  int ov[TOPS_MAX_BURSTS] = {}, tot = 0, mx = 0;
  tops_overlap_size(nb, m->burst_first_line_time, m->burst_last_line_time, m->dt, ov, &tot,
                    &mx);
  if (o->reslave_full)
    b += lines * cplx;
  else
    b += 2 * (size_t)(tot > 0 ? tot : 0) * cplx;
  b += 3 * sizeof(double) * (size_t)nb * W;           // deramp rows
  b += (size_t)nb * 4096 * 33 * sizeof(double);       // geocoreg partials (upper bound)
  // ESD partials: one 16-byte sum per (224-column strip, 32-line segment)
  // of every overlap, as the ESD kernel tiles it
  size_t esd_items = 0;
  for (int i = 0; i + 1 < nb; i++) {
    const int lines_i = ov[i] > 0 ? ov[i] : 0;
    esd_items += (size_t)((W + 223) / 224) * (size_t)(lines_i > 0 ? (lines_i + 31) / 32 : 1);
  }
  b += esd_items * 16;
  b += 2 * sizeof(float) * 2048 * 12 + 2048 * 4 + 4096;
  b += 32 * Arena::kAlign;                             // per-buffer alignment
  return b;
}

int tops_pair_create(const tops_swath_info *m, const tops_swath_info *s, const tops_pair_opts *o,
                     int dem_lines, int dem_pixels, tops_pair **out) {
  if (dem_lines <= 0 || dem_pixels <= 0) return TOPS_E_INVALID;
  return pair_create(m, s, o, dem_lines, dem_pixels, nullptr, nullptr, nullptr, false, out);
}

}  // extern "C"

int pair_create(const tops_swath_info *m, const tops_swath_info *s, const tops_pair_opts *o,
                int dem_lines, int dem_pixels, Arena *arena, tops_lut_dev *shared_lut,
                cudaStream_t stream, bool async_copy, tops_pair **out) {
  if (!m || !s || !o || !out) return TOPS_E_INVALID;
  const int nb = m->n_bursts, L = m->lines_per_burst, W = m->samples_per_burst;
  if (nb < 1 || nb > TOPS_MAX_BURSTS || L < 16 || W < 16 || s->n_bursts != nb ||
      s->lines_per_burst != L || s->samples_per_burst != W || dem_lines < 0 || dem_pixels < 0 ||
      m->n_sv < 3 || s->n_sv < 3 ||
      (o->precision != TOPS_PREC_SPLIT && o->precision != TOPS_PREC_FP64))
    return TOPS_E_INVALID;
  tops_pair *P = new tops_pair();
  P->arena = arena;
  P->m = *m;
  P->s = *s;
  P->o = *o;
  P->nb = nb;
  P->L = L;
  P->W = W;
  P->dem_lines = dem_lines;
  P->dem_pixels = dem_pixels;
  int st = TOPS_OK;
  auto fail = [&](int e) {
    delete P;
    return e;
  };
  // host precomputes (reference Main.cpp:57-76, Func.cpp:2510-2555)
  if ((st = fit_orbit(*m, P->fm)) || (st = fit_orbit(*s, P->fs))) return fail(st);
  if ((st = deramp_of(*m, P->fm, P->dm)) || (st = deramp_of(*s, P->fs, P->ds))) return fail(st);
  if (!shared_lut) {
    P->kaz.resize(2048 * 12);
    P->krg.resize(2048 * 12);
    if ((st = tops_lut(12, m->prf, m->az_bandwidth, 2 * m->rsr, P->kaz.data(), P->krg.data())))
      return fail(st);
  }
  if (nb > 1) {
    P->ov.resize(nb - 1);
    int tot = 0, mx = 0;
    if ((st = tops_overlap_size(nb, m->burst_first_line_time, m->burst_last_line_time, m->dt,
                                P->ov.data(), &tot, &mx)))
      return fail(st);
    for (int v : P->ov)
      if (v < 1 || v >= L) return fail(TOPS_E_INVALID);
    P->ov_off.resize(nb - 1);
    int off = 0;
    for (int i = 0; i < nb - 1; i++) {
      P->ov_off[i] = off;
      off += P->ov[i];
    }
    P->ov_total = off;
  }
  P->spec_sep = tops_spectral_sep(nb, W, L, m->dt, P->dm.kt.data());
  // device buffers
  pitches(W, dem_pixels, P->slc_pitch, P->cplx_pitch, P->coh_pitch, P->dem_pitch);
  const size_t lines = (size_t)nb * L;
  void *v;
#define P_ALLOC(dst, bytes)                     \
  do {                                          \
    if ((st = P->alloc(&v, (bytes)))) return fail(st); \
    dst = reinterpret_cast<decltype(dst)>(v);   \
  } while (0)
  P_ALLOC(P->d_master, lines * P->slc_pitch);
  P_ALLOC(P->d_slave, lines * P->slc_pitch);
  if (o->reslave_full) {
    P_ALLOC(P->d_reslave, lines * P->cplx_pitch);
  } else if (nb > 1) {
    P_ALLOC(P->d_fwd, (size_t)P->ov_total * P->cplx_pitch);
    P_ALLOC(P->d_back, (size_t)P->ov_total * P->cplx_pitch);
  }
  P_ALLOC(P->d_res_esd, lines * P->cplx_pitch);
  P_ALLOC(P->d_coh, lines * P->coh_pitch);
  if (dem_lines > 0) P_ALLOC(P->d_dem, (size_t)dem_lines * P->dem_pitch);
  P_ALLOC(P->d_kt, sizeof(double) * lines / L * W);
  P_ALLOC(P->d_tref, sizeof(double) * lines / L * W);
  P_ALLOC(P->d_fdc, sizeof(double) * lines / L * W);
  P_ALLOC(P->d_cpm, sizeof(double) * 12 * nb);
  P_ALLOC(P->d_status, sizeof(int) * nb);
  P_ALLOC(P->d_shift, sizeof(double) * (nb > 1 ? nb - 1 : 1));
  P_ALLOC(P->d_sums, sizeof(double) * 2 * (nb > 1 ? nb - 1 : 1));
  P->geo_scratch = (size_t)nb * 4096 * 33 * sizeof(double);
  P_ALLOC(P->d_geo_scratch, P->geo_scratch);
#undef P_ALLOC
  // slave deramp rows (Func.cpp:2383 passes burst 0's rows for every burst);
  // the host vectors live in the plan, so an asynchronous copy may be pending
  const size_t rb = sizeof(double) * nb * W;
  if (async_copy) {
    if (cudaMemcpyAsync(P->d_kt, P->ds.kt.data(), rb, cudaMemcpyHostToDevice, stream) ||
        cudaMemcpyAsync(P->d_tref, P->ds.tref.data(), rb, cudaMemcpyHostToDevice, stream) ||
        cudaMemcpyAsync(P->d_fdc, P->ds.dc.data(), rb, cudaMemcpyHostToDevice, stream))
      return fail(TOPS_E_CUDA);
  } else if (cudaMemcpy(P->d_kt, P->ds.kt.data(), rb, cudaMemcpyHostToDevice) ||
             cudaMemcpy(P->d_tref, P->ds.tref.data(), rb, cudaMemcpyHostToDevice) ||
             cudaMemcpy(P->d_fdc, P->ds.dc.data(), rb, cudaMemcpyHostToDevice)) {
    return fail(TOPS_E_CUDA);
  }
  if (shared_lut) {
    P->lut = shared_lut;
    P->lut_owned = false;
  } else if ((st = tops_lut_create(P->kaz.data(), P->krg.data(), &P->lut))) {
    return fail(st);
  }
  // ESD scratch
  if (nb > 1) {
    std::vector<tops_esd_overlap> ovs(nb - 1);
    for (int i = 0; i < nb - 1; i++) {
      tops_esd_overlap &e = ovs[i];
      e.mF = e.mB = P->d_master;
      e.sF = e.sB = P->d_res_esd;
      e.m_pitch = P->slc_pitch;
      e.s_pitch = P->cplx_pitch;
      e.lines = P->ov[i];
      e.pixels = W;
      e.spec_sep = P->spec_sep;
      e.dt = m->dt;
    }
    P->esd_scratch = tops_esd_scratch_bytes(ovs.data(), nb - 1);
    void *sp;
    if ((st = P->alloc(&sp, P->esd_scratch))) return fail(st);
    P->d_esd_scratch = sp;
  }
  *out = P;
  return TOPS_OK;
}

extern "C" {

int tops_pair_destroy(tops_pair *p) {
  delete p;
  return TOPS_OK;
}

int tops_pair_set_dem(tops_pair *P, const float *dem, double lat0, double lon0, double dlat,
                      double dlon, const tops_dem_window *win, void *stream) {
  if (!P || !dem || !win || !P->d_dem) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  P_CUDA(cudaMemcpy2DAsync(P->d_dem, P->dem_pitch, dem, (size_t)P->dem_pixels * 4,
                           (size_t)P->dem_pixels * 4, P->dem_lines, cudaMemcpyHostToDevice, st));
  return pair_bind_dem(P, P->d_dem, P->dem_pitch, P->dem_lines, P->dem_pixels, lat0, lon0, dlat,
                       dlon, win);
}

}  // extern "C"

int pair_bind_dem(tops_pair *P, const float *d_dem, size_t dem_pitch, int dem_lines,
                  int dem_pixels, double lat0, double lon0, double dlat, double dlon,
                  const tops_dem_window *win) {
  if (!P || !d_dem || !win) return TOPS_E_INVALID;
  const int nb = P->nb, L = P->L, W = P->W;
  P->geo.assign(nb, tops_geo_job());
  for (int b = 0; b < nb; b++) {
    const tops_dem_window &w = win[b];
    if (w.row0 < 0 || w.col0 < 0 || w.rows < 1 || w.cols < 1 || w.row0 + w.rows > dem_lines ||
        w.col0 + w.cols > dem_pixels)
      return TOPS_E_INVALID;
    tops_geo_job &g = P->geo[b];
    memset(&g, 0, sizeof(g));
    g.dem = reinterpret_cast<const float *>(reinterpret_cast<const char *>(d_dem) +
                                            (size_t)w.row0 * dem_pitch) + w.col0;
    g.dem_pitch = dem_pitch;
    g.dem_lines = w.rows;
    g.dem_pixels = w.cols;
    g.lat0 = lat0 - w.row0 * dlat;
    g.lon0 = lon0 + w.col0 * dlon;
    g.dlat = dlat;
    g.dlon = dlon;
    g.nodata = -32768.0;
    // master burst box (Func.cpp:2228-2231)
    g.xmin = 0;
    g.xmax = W - 1;
    g.ymin = b * L;
    g.ymax = (b + 1) * L - 1;
    const tops_swath_info *sw[2] = {&P->m, &P->s};
    const OrbitFit *of[2] = {&P->fm, &P->fs};
    for (int k = 0; k < 2; k++) {
      g.dt[k] = sw[k]->dt;
      g.first_line_time[k] = sw[k]->burst_first_line_time[b];
      g.slr_time[k] = sw[k]->slr_time;
      g.range_spacing[k] = sw[k]->range_spacing;
      g.mid_time[k] = sw[k]->sv_t[sw[k]->n_sv / 2];
      // initial azimuth time: burst centre (Func.cpp:2234-2235)
      g.azi_init[k] = 0.5 * (sw[k]->burst_first_line_time[b] + sw[k]->burst_last_line_time[b]);
      g.line_offset[k] = b * L;
      g.ncoef[k] = of[k]->n;
      for (int i = 0; i < of[k]->n; i++) {
        g.coef[k][0][i] = of[k]->cx[i];
        g.coef[k][1][i] = of[k]->cy[i];
        g.coef[k][2][i] = of[k]->cz[i];
      }
    }
    g.cpm_dev = P->d_cpm + 12 * b;
    g.status_dev = P->d_status + b;
  }
  if (tops_geocoreg_scratch_bytes(P->geo.data(), nb) > P->geo_scratch) return TOPS_E_INVALID;
  P->dem_set = true;
  return TOPS_OK;
}

extern "C" {

int tops_pair_upload(tops_pair *P, const void *master, const void *slave, void *stream) {
  if (!P || !master || !slave) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t row = (size_t)P->W * 4, lines = (size_t)P->nb * P->L;
  P_CUDA(cudaMemcpy2DAsync(P->d_master, P->slc_pitch, master, row, row, lines,
                           cudaMemcpyHostToDevice, st));
  P_CUDA(cudaMemcpy2DAsync(P->d_slave, P->slc_pitch, slave, row, row, lines,
                           cudaMemcpyHostToDevice, st));
  return TOPS_OK;
}

static tops_resample_job base_job(const tops_pair *P, int b) {
  tops_resample_job j;
  memset(&j, 0, sizeof(j));
  const int L = P->L, W = P->W;
  j.slave = P->d_slave + (size_t)b * L * P->slc_pitch;
  j.slave_pitch = P->slc_pitch;
  const int row = P->o.burst0_deramp_rows ? 0 : b;
  j.kt = P->d_kt + (size_t)row * W;
  j.tref = P->d_tref + (size_t)row * W;
  j.fdc = P->d_fdc + (size_t)row * W;
  j.mbox[0] = 0;
  j.mbox[1] = W - 1;
  j.mbox[2] = b * L;
  j.mbox[3] = (b + 1) * L - 1;
  j.sbox[0] = 0;
  j.sbox[1] = W - 1;
  j.sbox[2] = b * L;
  j.sbox[3] = (b + 1) * L - 1;
  j.cpm_dev = P->d_cpm + 12 * b;
  j.s_first_line = b * L;
  j.dt = P->s.dt;
  j.out_pitch = P->cplx_pitch;
  return j;
}

}  // extern "C"

// ---- stage job lists of one pair (shared by the single-pair and batched runs)
void pair_rs1_jobs(const tops_pair *P, std::vector<tops_resample_job> &jobs) {
  const int nb = P->nb, L = P->L;
  if (P->o.reslave_full) {
    for (int b = 0; b < nb; b++) {
      tops_resample_job j = base_job(P, b);
      j.out = P->d_reslave + (size_t)b * L * P->cplx_pitch;
      j.out_rows = -1;
      jobs.push_back(j);
    }
  } else {
    for (int i = 0; i < nb - 1; i++) {
      tops_resample_job f = base_job(P, i);   // forward band: end of burst i
      f.out = P->d_fwd + (size_t)P->ov_off[i] * P->cplx_pitch;
      f.out_row0 = L - P->ov[i];
      f.out_rows = P->ov[i];
      jobs.push_back(f);
      tops_resample_job k = base_job(P, i + 1);   // backward band: start of burst i+1
      k.out = P->d_back + (size_t)P->ov_off[i] * P->cplx_pitch;
      k.out_row0 = 0;
      k.out_rows = P->ov[i];
      jobs.push_back(k);
    }
  }
}

void pair_esd_overlaps(const tops_pair *P, std::vector<tops_esd_overlap> &ovs) {
  const int nb = P->nb, L = P->L, W = P->W;
  for (int i = 0; i < nb - 1; i++) {
    tops_esd_overlap e;
    memset(&e, 0, sizeof(e));
    const size_t fl = (size_t)(i + 1) * L - P->ov[i], bl = (size_t)(i + 1) * L;
    e.mF = P->d_master + fl * P->slc_pitch;
    e.mB = P->d_master + bl * P->slc_pitch;
    e.m_pitch = P->slc_pitch;
    if (P->o.reslave_full) {
      e.sF = P->d_reslave + fl * P->cplx_pitch;
      e.sB = P->d_reslave + bl * P->cplx_pitch;
    } else {
      e.sF = P->d_fwd + (size_t)P->ov_off[i] * P->cplx_pitch;
      e.sB = P->d_back + (size_t)P->ov_off[i] * P->cplx_pitch;
    }
    e.s_pitch = P->cplx_pitch;
    e.lines = P->ov[i];
    e.pixels = W;
    e.spec_sep = P->spec_sep;
    e.dt = P->m.dt;
    ovs.push_back(e);
  }
}

// shifts: the device ESD shifts of this pair's overlaps.  One job per burst.
// The first burst's ReSlaveESD is its ReSlave (the reference copies it,
// ResampleFirstBurst, Func.cpp:2653-2674): its job is the ReSlave job (slave
// interval, no shift), so its output equals that burst's ReSlave bit for
// bit; pair_first_burst_copy replaces it by a copy when the full ReSlave is
// computed.  Later bursts: the ESD shift of the overlap before them and the
// master's interval, as DerampDemodResample_ESD gets it (Func.cpp:2704).
void pair_rs2_jobs(const tops_pair *P, const double *shifts,
                   std::vector<tops_resample_job> &jobs) {
  const int nb = P->nb, L = P->L;
  for (int b = 0; b < nb; b++) {
    tops_resample_job j = base_job(P, b);
    j.out = P->d_res_esd + (size_t)b * L * P->cplx_pitch;
    j.out_rows = -1;
    if (b > 0) {
      j.az_shift_dev = shifts + (b - 1);
      j.dt = P->m.dt;
    }
    jobs.push_back(j);
  }
}

int pair_first_burst_copy(const tops_pair *P, tops::RowCopy *c) {
  if (!P->o.reslave_full) return 0;
  *c = {P->d_reslave, P->cplx_pitch, P->d_res_esd, P->cplx_pitch, (size_t)P->W * 8, P->L};
  return 1;
}

void pair_coh_jobs(const tops_pair *P, std::vector<tops_coh_job> &cj) {
  const int nb = P->nb, L = P->L, W = P->W;
  for (int b = 0; b < nb; b++) {
    tops_coh_job c;
    memset(&c, 0, sizeof(c));
    c.master = P->d_master + (size_t)b * L * P->slc_pitch;
    c.master_pitch = P->slc_pitch;
    c.slave = P->d_res_esd + (size_t)b * L * P->cplx_pitch;
    c.slave_pitch = P->cplx_pitch;
    c.coh = reinterpret_cast<float *>(reinterpret_cast<char *>(P->d_coh) +
                                      (size_t)b * L * P->coh_pitch);
    c.coh_pitch = P->coh_pitch;
    c.lines = L;
    c.pixels = W;
    cj.push_back(c);
  }
}

// The ReSlaveESD resample in up to three chunks of bursts on `st`, and each
// chunk's coherence on a second stream as soon as the chunk is resampled, so
// the coherence of one chunk (L1- and HBM-bound) overlaps the resample of the
// next (issue-bound).  Chunks rather than single bursts keep each launch
// several waves long.  The kernels and their inputs are those of the
// one-launch form, so the outputs are the same bit for bit.  The coherence
// stream has the highest priority: its CTAs are dispatched ahead of the
// resample's pending ones.
static int pair_tail_overlapped(tops_pair *P, const std::vector<tops_resample_job> &rs2,
                                const std::vector<tops_coh_job> &cj, int skip,
                                const tops::RowCopy &first, cudaStream_t st, int &launches) {
  const int nb = P->nb;
  if (!P->s_coh) {
    int lo = 0, hi = 0;
    P_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    P_CUDA(cudaStreamCreateWithPriority(&P->s_coh, cudaStreamNonBlocking, hi));
  }
  while ((int)P->cev.size() < nb + 1) {
    cudaEvent_t e;
    P_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    P->cev.push_back(e);
  }
  cudaStream_t cs = P->s_coh;
  const int per = (nb + 2) / 3;   // bursts per chunk
  int e = 0;
  for (int b0 = 0; b0 < nb; b0 += per) {
    const int b1 = std::min(nb, b0 + per);
    int r0 = b0;
    if (b0 == 0 && skip) {
      tops::RowCopy c = first;
      P_TRY(tops::row_copy(&c, 1, st, &launches));
      r0 = 1;
    }
    if (b1 > r0) {
      P_TRY(tops_resample_ex(P->lut, &rs2[r0], b1 - r0, P->o.precision, st));
      launches += 1;
    }
    P_CUDA(cudaEventRecord(P->cev[e], st));
    P_CUDA(cudaStreamWaitEvent(cs, P->cev[e], 0));
    e++;
    P_TRY(tops::coherence_launch(&cj[b0], b1 - b0, P->o.win_rg, P->o.win_az, coh_cfg(P->o), cs));
    launches += 1;
  }
  // `st` completes when the last coherence has
  P_CUDA(cudaEventRecord(P->cev[e], cs));
  P_CUDA(cudaStreamWaitEvent(st, P->cev[e], 0));
  return TOPS_OK;
}

extern "C" {

int tops_pair_run(tops_pair *P, void *stream) {
  if (!P || !P->dem_set) return TOPS_E_INVALID;
  const int nb = P->nb;
  int launches = 0;
  // 1. geometric coregistration of every burst (2 kernels)
  P_TRY(tops_geocoreg(P->geo.data(), nb, P->d_geo_scratch, P->geo_scratch, stream));
  launches += 2;
  // 2. resample without shift: full ReSlave, or only the overlap bands
  std::vector<tops_resample_job> jobs;
  pair_rs1_jobs(P, jobs);
  if (!jobs.empty()) {
    P_TRY(tops_resample_ex(P->lut, jobs.data(), (int)jobs.size(), P->o.precision, stream));
    launches += 1;
  }
  // 3. ESD over the overlaps (shifts stay on the device)
  if (nb > 1) {
    std::vector<tops_esd_overlap> ovs;
    pair_esd_overlaps(P, ovs);
    P_TRY(tops::esd_launch(ovs.data(), nb - 1, P->o.win_az, P->o.win_rg, P->o.esd_threshold, P->d_shift,
                   P->d_sums, P->d_esd_scratch, P->esd_scratch, P->o.compensated, static_cast<cudaStream_t>(stream)));
    launches += 2;
  }
  // 4. resample with the ESD shift of the preceding overlap (first burst
  //    uncorrected, Func.cpp:2653-2702)
  jobs.clear();
  pair_rs2_jobs(P, P->d_shift, jobs);
  if (P->o.coh_overlap && nb > 1) {
    // 4 + 5 overlapped: each burst's coherence as soon as it is resampled
    tops::RowCopy c;
    const int skip = pair_first_burst_copy(P, &c);
    std::vector<tops_coh_job> cj;
    pair_coh_jobs(P, cj);
    P_TRY(pair_tail_overlapped(P, jobs, cj, skip, c, static_cast<cudaStream_t>(stream),
                               launches));
    P->n_launches = launches;
    return TOPS_OK;
  }
  {
    tops::RowCopy c;
    const int skip = pair_first_burst_copy(P, &c);
    if (skip) P_TRY(tops::row_copy(&c, 1, static_cast<cudaStream_t>(stream), &launches));
    if (nb - skip > 0) {
      P_TRY(tops_resample_ex(P->lut, jobs.data() + skip, nb - skip, P->o.precision, stream));
      launches += 1;
    }
  }
  // 5. coherence of master vs ReSlaveESD
  std::vector<tops_coh_job> cj;
  pair_coh_jobs(P, cj);
  P_TRY(tops::coherence_launch(cj.data(), nb, P->o.win_rg, P->o.win_az, coh_cfg(P->o), static_cast<cudaStream_t>(stream)));
  launches += 1;
  P->n_launches = launches;
  return TOPS_OK;
}

// Stage timing: the launches of tops_pair_run with CUDA events between the
// stages, then a synchronisation; ms[5] = geocoreg, ReSlave resample, ESD,
// ReSlaveESD resample, coherence.
int tops_pair_stage_times(tops_pair *P, void *stream, float *ms) {
  if (!P || !P->dem_set || !ms) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = P->nb;
  cudaEvent_t ev[6];
  for (int i = 0; i < 6; i++) P_CUDA(cudaEventCreate(&ev[i]));
  int r = TOPS_OK;
  std::vector<tops_resample_job> jobs;
  std::vector<tops_esd_overlap> ovs;
  std::vector<tops_coh_job> cj;
  do {
    if (cudaEventRecord(ev[0], st) != cudaSuccess) { r = TOPS_E_CUDA; break; }
    if ((r = tops_geocoreg(P->geo.data(), nb, P->d_geo_scratch, P->geo_scratch, stream)) != TOPS_OK)
      break;
    cudaEventRecord(ev[1], st);
    pair_rs1_jobs(P, jobs);
    if (!jobs.empty() &&
        (r = tops_resample_ex(P->lut, jobs.data(), (int)jobs.size(), P->o.precision, stream)) !=
            TOPS_OK)
      break;
    cudaEventRecord(ev[2], st);
    if (nb > 1) {
      pair_esd_overlaps(P, ovs);
      if ((r = tops::esd_launch(ovs.data(), nb - 1, P->o.win_az, P->o.win_rg, P->o.esd_threshold,
                        P->d_shift, P->d_sums, P->d_esd_scratch, P->esd_scratch, P->o.compensated, static_cast<cudaStream_t>(stream))) !=
          TOPS_OK)
        break;
    }
    cudaEventRecord(ev[3], st);
    jobs.clear();
    pair_rs2_jobs(P, P->d_shift, jobs);
    tops::RowCopy c;
    const int skip = pair_first_burst_copy(P, &c);
    if (skip && (r = tops::row_copy(&c, 1, st, nullptr)) != TOPS_OK) break;
    if (nb - skip > 0 &&
        (r = tops_resample_ex(P->lut, jobs.data() + skip, nb - skip, P->o.precision, stream)) !=
            TOPS_OK)
      break;
    cudaEventRecord(ev[4], st);
    pair_coh_jobs(P, cj);
    if ((r = tops::coherence_launch(cj.data(), nb, P->o.win_rg, P->o.win_az, coh_cfg(P->o), static_cast<cudaStream_t>(stream))) != TOPS_OK) break;
    if (cudaEventRecord(ev[5], st) != cudaSuccess || cudaEventSynchronize(ev[5]) != cudaSuccess) {
      r = TOPS_E_CUDA;
      break;
    }
    for (int i = 0; i < 5; i++)
      if (cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]) != cudaSuccess) r = TOPS_E_CUDA;
  } while (0);
  if (r != TOPS_OK) cudaStreamSynchronize(st);
  for (int i = 0; i < 6; i++) cudaEventDestroy(ev[i]);
  return r;
}

// The per-burst launch loop: every stage launched once per burst (or
// overlap), as the reference's drivers call their stages; the comparison form
// for the batched plans.
int tops_pair_run_per_burst(tops_pair *P, void *stream) {
  if (!P || !P->dem_set) return TOPS_E_INVALID;
  const int nb = P->nb;
  int launches = 0;
  for (int b = 0; b < nb; b++) {
    P_TRY(tops_geocoreg(&P->geo[b], 1, P->d_geo_scratch, P->geo_scratch, stream));
    launches += 2;
  }
  std::vector<tops_resample_job> jobs;
  pair_rs1_jobs(P, jobs);
  for (const tops_resample_job &j : jobs) {
    P_TRY(tops_resample_ex(P->lut, &j, 1, P->o.precision, stream));
    launches += 1;
  }
  if (nb > 1) {
    std::vector<tops_esd_overlap> ovs;
    pair_esd_overlaps(P, ovs);
    for (int i = 0; i < nb - 1; i++) {
      P_TRY(tops::esd_launch(&ovs[i], 1, P->o.win_az, P->o.win_rg, P->o.esd_threshold, P->d_shift + i,
                     P->d_sums + 2 * i, P->d_esd_scratch, P->esd_scratch, P->o.compensated, static_cast<cudaStream_t>(stream)));
      launches += 2;
    }
  }
  jobs.clear();
  pair_rs2_jobs(P, P->d_shift, jobs);
  for (const tops_resample_job &j : jobs) {
    P_TRY(tops_resample_ex(P->lut, &j, 1, P->o.precision, stream));
    launches += 1;
  }
  std::vector<tops_coh_job> cj;
  pair_coh_jobs(P, cj);
  for (const tops_coh_job &c : cj) {
    P_TRY(tops::coherence_launch(&c, 1, P->o.win_rg, P->o.win_az, coh_cfg(P->o), static_cast<cudaStream_t>(stream)));
    launches += 1;
  }
  P->n_launches = launches;
  return TOPS_OK;
}

int tops_pair_run_graph(tops_pair *P, void *stream) {
  if (!P) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!P->graph_exec) {
    // one eager run first: it sets per-kernel attributes outside the capture
    P_TRY(tops_pair_run(P, stream));
    if (!P->capture_stream)
      P_CUDA(cudaStreamCreateWithFlags(&P->capture_stream, cudaStreamNonBlocking));
    cudaStream_t cs = P->capture_stream;
    P_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int s = tops_pair_run(P, cs);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    if (s != TOPS_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    P_CUDA(e);
    P->graph = g;
    P_CUDA(cudaGraphInstantiate(&P->graph_exec, g, 0));
  }
  P_CUDA(cudaGraphLaunch(P->graph_exec, st));
  return TOPS_OK;
}

int tops_pair_download(tops_pair *P, void *reslave, void *reslave_esd, float *coh, double *cpm,
                       double *shifts, void *stream) {
  if (!P) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t lines = (size_t)P->nb * P->L, W = P->W;
  if (reslave) {
    if (!P->o.reslave_full) return TOPS_E_INVALID;
    P_CUDA(cudaMemcpy2DAsync(reslave, W * 8, P->d_reslave, P->cplx_pitch, W * 8, lines,
                             cudaMemcpyDeviceToHost, st));
  }
  if (reslave_esd)
    P_CUDA(cudaMemcpy2DAsync(reslave_esd, W * 8, P->d_res_esd, P->cplx_pitch, W * 8, lines,
                             cudaMemcpyDeviceToHost, st));
  if (coh)
    P_CUDA(cudaMemcpy2DAsync(coh, W * 4, P->d_coh, P->coh_pitch, W * 4, lines,
                             cudaMemcpyDeviceToHost, st));
  if (cpm)
    P_CUDA(cudaMemcpyAsync(cpm, P->d_cpm, sizeof(double) * 12 * P->nb, cudaMemcpyDeviceToHost, st));
  if (shifts && P->nb > 1)
    P_CUDA(cudaMemcpyAsync(shifts, P->d_shift, sizeof(double) * (P->nb - 1),
                           cudaMemcpyDeviceToHost, st));
  return TOPS_OK;
}

// Host to host, pipelined per burst.  Three streams: `up` copies the SLCs of
// burst b, `stream` runs burst b's kernels as soon as its SLCs are on the
// device, `down` copies burst b's outputs as soon as its coherence is done.
// The copies of one burst then overlap the kernels of its neighbours and the
// two PCIe directions run at once; the dependencies between bursts are those
// of the stages (ESD of overlap b-1 needs the ReSlave of bursts b-1 and b).
int tops_pair_process(tops_pair *P, const void *master, const void *slave, void *reslave,
                      void *reslave_esd, float *coh, double *cpm, double *shifts, void *stream) {
  if (!P || !P->dem_set || !master || !slave) return TOPS_E_INVALID;
  if (reslave && !P->o.reslave_full) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = P->nb, L = P->L, W = P->W;
  const int n_ev = 3 * nb + 2;
  if (!P->s_up) {
    P_CUDA(cudaStreamCreateWithFlags(&P->s_up, cudaStreamNonBlocking));
    P_CUDA(cudaStreamCreateWithFlags(&P->s_down, cudaStreamNonBlocking));
  }
  while ((int)P->pev.size() < n_ev) {
    cudaEvent_t e;
    P_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    P->pev.push_back(e);
  }
  cudaEvent_t ev_start = P->pev[0], ev_end = P->pev[1];
  cudaEvent_t *ev_up = &P->pev[2], *ev_rs1 = &P->pev[2 + nb], *ev_done = &P->pev[2 + 2 * nb];
  // earlier work on `stream` may still read the buffers the uploads overwrite
  P_CUDA(cudaEventRecord(ev_start, st));
  P_CUDA(cudaStreamWaitEvent(P->s_up, ev_start, 0));
  P_CUDA(cudaStreamWaitEvent(P->s_down, ev_start, 0));
  const size_t row = (size_t)W * 4;
  for (int b = 0; b < nb; b++) {
    const size_t off = (size_t)b * L;
    P_CUDA(cudaMemcpy2DAsync(P->d_master + off * P->slc_pitch, P->slc_pitch,
                             static_cast<const char *>(master) + off * row, row, row, L,
                             cudaMemcpyHostToDevice, P->s_up));
    P_CUDA(cudaMemcpy2DAsync(P->d_slave + off * P->slc_pitch, P->slc_pitch,
                             static_cast<const char *>(slave) + off * row, row, row, L,
                             cudaMemcpyHostToDevice, P->s_up));
    P_CUDA(cudaEventRecord(ev_up[b], P->s_up));
  }
  int launches = 0;
  P_TRY(tops_geocoreg(P->geo.data(), nb, P->d_geo_scratch, P->geo_scratch, stream));
  launches += 2;
  std::vector<tops_resample_job> rs1, rs2;
  pair_rs1_jobs(P, rs1);
  pair_rs2_jobs(P, P->d_shift, rs2);
  std::vector<tops_esd_overlap> ovs;
  pair_esd_overlaps(P, ovs);
  std::vector<tops_coh_job> cj;
  pair_coh_jobs(P, cj);
  const size_t crow = (size_t)W * 8, frow = (size_t)W * 4;
  for (int b = 0; b < nb; b++) {
    const size_t off = (size_t)b * L;
    P_CUDA(cudaStreamWaitEvent(st, ev_up[b], 0));
    // ReSlave jobs reading slave burst b (the whole burst, or its overlap bands)
    std::vector<tops_resample_job> mine;
    for (const tops_resample_job &j : rs1)
      if (j.s_first_line == b * L) mine.push_back(j);
    if (!mine.empty()) {
      P_TRY(tops_resample_ex(P->lut, mine.data(), (int)mine.size(), P->o.precision, stream));
      launches += 1;
    }
    if (reslave) {
      P_CUDA(cudaEventRecord(ev_rs1[b], st));
      P_CUDA(cudaStreamWaitEvent(P->s_down, ev_rs1[b], 0));
      P_CUDA(cudaMemcpy2DAsync(static_cast<char *>(reslave) + off * crow, crow,
                               P->d_reslave + off * P->cplx_pitch, P->cplx_pitch, crow, L,
                               cudaMemcpyDeviceToHost, P->s_down));
    }
    if (b > 0) {
      P_TRY(tops::esd_launch(&ovs[b - 1], 1, P->o.win_az, P->o.win_rg, P->o.esd_threshold,
                     P->d_shift + (b - 1), P->d_sums + 2 * (b - 1), P->d_esd_scratch,
                     P->esd_scratch, P->o.compensated, static_cast<cudaStream_t>(stream)));
      launches += 2;
    }
    P_TRY(tops_resample_ex(P->lut, &rs2[b], 1, P->o.precision, stream));
    P_TRY(tops::coherence_launch(&cj[b], 1, P->o.win_rg, P->o.win_az, coh_cfg(P->o), static_cast<cudaStream_t>(stream)));
    launches += 2;
    P_CUDA(cudaEventRecord(ev_done[b], st));
    P_CUDA(cudaStreamWaitEvent(P->s_down, ev_done[b], 0));
    if (reslave_esd)
      P_CUDA(cudaMemcpy2DAsync(static_cast<char *>(reslave_esd) + off * crow, crow,
                               P->d_res_esd + off * P->cplx_pitch, P->cplx_pitch, crow, L,
                               cudaMemcpyDeviceToHost, P->s_down));
    if (coh)
      P_CUDA(cudaMemcpy2DAsync(reinterpret_cast<char *>(coh) + off * frow, frow,
                               reinterpret_cast<char *>(P->d_coh) + off * P->coh_pitch,
                               P->coh_pitch, frow, L, cudaMemcpyDeviceToHost, P->s_down));
  }
  if (cpm)
    P_CUDA(cudaMemcpyAsync(cpm, P->d_cpm, sizeof(double) * 12 * nb, cudaMemcpyDeviceToHost,
                           P->s_down));
  if (shifts && nb > 1)
    P_CUDA(cudaMemcpyAsync(shifts, P->d_shift, sizeof(double) * (nb - 1),
                           cudaMemcpyDeviceToHost, P->s_down));
  // `stream` completes when the last copy has landed
  P_CUDA(cudaEventRecord(ev_end, P->s_down));
  P_CUDA(cudaStreamWaitEvent(st, ev_end, 0));
  P->n_launches = launches;
  return TOPS_OK;
}

int tops_pair_buffers_get(const tops_pair *P, tops_pair_buffers *b) {
  if (!P || !b) return TOPS_E_INVALID;
  b->master = P->d_master;
  b->slave = P->d_slave;
  b->reslave = P->d_reslave;
  b->reslave_esd = P->d_res_esd;
  b->coh = P->d_coh;
  b->cpm = P->d_cpm;
  b->shifts = P->d_shift;
  b->geo_status = P->d_status;
  b->slc_pitch = P->slc_pitch;
  b->cplx_pitch = P->cplx_pitch;
  b->coh_pitch = P->coh_pitch;
  b->n_bursts = P->nb;
  b->lines = P->L;
  b->samples = P->W;
  b->n_launches = P->n_launches;
  return TOPS_OK;
}

// ------------------------------------------------------------ plain form
int tops_plain_pair(const tops_swath_info *m, const tops_swath_info *s, const tops_pair_opts *o,
                    const int *dem_int, int dem_lines, int dem_pixels, double lat0, double lon0,
                    double dlat, double dlon, const tops_dem_window *win, const void *master_slc,
                    const void *slave_slc, void *reslave, void *reslave_esd, float *coh,
                    double *cpm, double *shifts) {
  if (!m || !s || !o || !dem_int || !win || !master_slc || !slave_slc || !reslave ||
      !reslave_esd || !coh)
    return TOPS_E_INVALID;
  const int nb = m->n_bursts, L = m->lines_per_burst, W = m->samples_per_burst;
  OrbitFit fm, fs;
  Deramp dm, ds;
  P_TRY(fit_orbit(*m, fm));
  P_TRY(fit_orbit(*s, fs));
  P_TRY(deramp_of(*m, fm, dm));
  P_TRY(deramp_of(*s, fs, ds));
  std::vector<float> kaz(2048 * 12), krg(2048 * 12);
  P_TRY(tops_lut(12, m->prf, m->az_bandwidth, 2 * m->rsr, kaz.data(), krg.data()));
  std::vector<double> az(6 * nb), rg(6 * nb);
  std::vector<double> mt(m->sv_t, m->sv_t + m->n_sv), st_(s->sv_t, s->sv_t + s->n_sv);
  std::vector<int> demw;
  // GeometricCoreg (Func.cpp:2225-2291)
  for (int b = 0; b < nb; b++) {
    const tops_dem_window &w = win[b];
    demw.resize((size_t)w.rows * w.cols);
    for (int r = 0; r < w.rows; r++)
      memcpy(&demw[(size_t)r * w.cols], dem_int + (size_t)(w.row0 + r) * dem_pixels + w.col0,
             sizeof(int) * w.cols);
    P_TRY(GeoCoreg_warp_cuda(
        b, b, 0, W - 1, b * L, (b + 1) * L - 1, dlat, dlon, w.rows, w.cols, &az[6 * b],
        &rg[6 * b], lat0 - w.row0 * dlat, lon0 + w.col0 * dlon, -32768, m->dt, s->dt,
        m->wavelength, L, L, m->burst_first_line_time[b], s->burst_first_line_time[b], W, W,
        mt.data(), st_.data(), m->n_sv, fm.n, s->n_sv, fs.n, m->slr_time, s->slr_time,
        m->range_spacing, s->range_spacing, false, false, demw.data(), fm.cx, fm.cy, fm.cz, fs.cx,
        fs.cy, fs.cz, 0.5 * (m->burst_first_line_time[b] + m->burst_last_line_time[b]),
        0.5 * (s->burst_first_line_time[b] + s->burst_last_line_time[b])));
  }
  if (cpm)
    for (int b = 0; b < nb; b++)
      for (int i = 0; i < 6; i++) {
        cpm[12 * b + i] = az[6 * b + i];
        cpm[12 * b + 6 + i] = rg[6 * b + i];
      }
  // DerampAndResample (Func.cpp:2351-2393)
  const size_t bl = (size_t)L * W;
  auto slave_b = [&](int b) {
    return const_cast<int16_t *>(static_cast<const int16_t *>(slave_slc) + 2 * b * bl);
  };
  auto master_b = [&](int b) {
    return const_cast<int16_t *>(static_cast<const int16_t *>(master_slc) + 2 * b * bl);
  };
  float *rs = static_cast<float *>(reslave), *re = static_cast<float *>(reslave_esd);
  for (int b = 0; b < nb; b++) {
    int MB[4] = {0, W - 1, b * L, (b + 1) * L - 1}, SB[4] = {0, W - 1, b * L, (b + 1) * L - 1};
    const int row = o->burst0_deramp_rows ? 0 : b;
    P_TRY(DerampDemodResample(slave_b(b), &az[6 * b], &rg[6 * b], 0.0, rs + 2 * b * bl,
                              kaz.data(), krg.data(), b, W, L, MB, SB, L, W, s->dt,
                              ds.kt.data() + (size_t)row * W, ds.tref.data() + (size_t)row * W,
                              ds.dc.data() + (size_t)row * W, 12));
  }
  // ESDAndCoh (Func.cpp:2510-2727)
  std::vector<double> sh(nb > 1 ? nb - 1 : 1, 0.0);
  if (nb > 1) {
    std::vector<int> ov(nb - 1);
    int tot = 0, mx = 0;
    P_TRY(tops_overlap_size(nb, m->burst_first_line_time, m->burst_last_line_time, m->dt,
                            ov.data(), &tot, &mx));
    const double ss = tops_spectral_sep(nb, W, L, m->dt, dm.kt.data());
    std::vector<int16_t> mF((size_t)tot * W * 2), mB((size_t)tot * W * 2);
    std::vector<float> sF((size_t)tot * W * 2), sB((size_t)tot * W * 2);
    size_t off = 0;
    for (int i = 0; i < nb - 1; i++) {
      const size_t f = (size_t)(i + 1) * L - ov[i], k = (size_t)(i + 1) * L, n = (size_t)ov[i] * W;
      memcpy(&mF[2 * off * W], static_cast<const int16_t *>(master_slc) + 2 * f * W, 4 * n);
      memcpy(&mB[2 * off * W], static_cast<const int16_t *>(master_slc) + 2 * k * W, 4 * n);
      memcpy(&sF[2 * off * W], rs + 2 * f * W, 8 * n);
      memcpy(&sB[2 * off * W], rs + 2 * k * W, 8 * n);
      off += ov[i];
    }
    P_TRY(EstESDShifts(mF.data(), mB.data(), sF.data(), sB.data(), ov.data(), sh.data(), nb - 1,
                       tot, W, o->win_az, o->win_rg, mx, o->esd_threshold, ss, m->dt));
    for (auto &v : sh)
      if (fabs(v) > 100) v = 0;   // Func.cpp:2612-2621
    if (shifts) memcpy(shifts, sh.data(), sizeof(double) * (nb - 1));
  }
  const int dx = (o->win_rg - 1) / 2, dy = (o->win_az - 1) / 2;
  for (int b = 0; b < nb; b++) {
    void *d = nullptr;
    if (b == 0) {
      memcpy(re, rs, 8 * bl);
      d = ResampleFirstBurst(re, W, L);
      if (!d) return TOPS_E_CUDA;
      P_TRY(CoherenceEst_ESD(0, 0, W, L, dx, dy, o->win_rg, o->win_az, master_b(0), d, coh));
    } else {
      int MB[4] = {0, W - 1, b * L, (b + 1) * L - 1}, SB[4] = {0, W - 1, b * L, (b + 1) * L - 1};
      const int row = o->burst0_deramp_rows ? 0 : b;
      d = DerampDemodResample_ESD(slave_b(b), &az[6 * b], &rg[6 * b], sh[b - 1], re + 2 * b * bl,
                                  kaz.data(), krg.data(), b, W, L, MB, SB, L, W, m->dt,
                                  ds.kt.data() + (size_t)row * W, ds.tref.data() + (size_t)row * W,
                                  ds.dc.data() + (size_t)row * W, 12);
      if (!d) return TOPS_E_CUDA;
      P_TRY(CoherenceEst(0, b * L, W, L, dx, dy, o->win_rg, o->win_az, master_b(b), d,
                         coh + b * bl));
    }
  }
  return TOPS_OK;
}

}  // extern "C"

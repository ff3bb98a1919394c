// capi.cu -- reference-compatible C entry points over the device API.
//
// Each entry point keeps the reference wrapper's name, argument order, units
// and host memory layout, and its call sequence (upload, kernels, download)
// but: returns a status instead of exit(0), never calls cudaDeviceReset,
// runs on the per-thread default stream of the current device, and reuses a
// per-thread grow-only device workspace instead of allocating every call.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <complex>
#include <vector>

#include "common.cuh"
#include "device_slots.h"
#include "launch.h"

namespace tops {

static thread_local int g_last_cuda_error = 0;
void set_cuda_error(cudaError_t e) { g_last_cuda_error = (int)e; }

// Defined in the kernel translation units.
int fill_resample_job(const tops_resample_job &u, ResampleJob &J);
int fill_coh_job(const tops_coh_job &u, CohJob &J);
int fill_esd_overlap(const tops_esd_overlap &u, EsdOverlap &O);
int fill_geo_job(const tops_geo_job &u, GeoJob &J);
int launch_coherence(const CohJob *jobs, int njobs, int win_rg, int win_az, const TileCfg &cfg,
                     cudaStream_t st);
int launch_esd(const EsdOverlap *ovs, int n_ov, int win_az, int win_rg, float thr,
               double *shifts, double *sums, void *scratch, size_t scratch_bytes,
               cudaStream_t st, int compensated);
size_t esd_scratch_bytes(const EsdOverlap *ov, int n);
int launch_geocoreg(const GeoJob *jobs, int njobs, bool dem_is_int, void *scratch,
                    size_t scratch_bytes, cudaStream_t st);
size_t geocoreg_scratch(const GeoJob *J, int n);

// Grow-only device workspace with named slots, one per (host thread,
// device): the entry points run on the calling thread's current device, so
// buffers of another device are never handed to them.
struct Workspace {
  enum { kSlots = 12 };
  int dev = -1;
  void *ptr[kSlots] = {};
  size_t cap[kSlots] = {};
  ~Workspace() {
    if (dev < 0) return;
    int cur = -1;
    const bool have_cur = cudaGetDevice(&cur) == cudaSuccess;
    if (cudaSetDevice(dev) == cudaSuccess)
      for (int i = 0; i < kSlots; i++)
        if (ptr[i]) cudaFree(ptr[i]);
    if (have_cur) cudaSetDevice(cur);
  }
  int get(int slot, size_t bytes, void **out) {
    if (bytes == 0) bytes = 16;
    if (cap[slot] < bytes) {
      if (ptr[slot]) cudaFree(ptr[slot]);
      ptr[slot] = nullptr;
      cap[slot] = 0;
      cudaError_t e = cudaMalloc(&ptr[slot], bytes);
      if (e != cudaSuccess) {
        set_cuda_error(e);
        return TOPS_E_NOMEM;
      }
      cap[slot] = bytes;
    }
    *out = ptr[slot];
    return TOPS_OK;
  }
};
static thread_local DeviceSlots<Workspace, kMaxDevices> g_ws;

// The workspace of the calling thread on its current device.
static int workspace(Workspace **out) {
  int dev = -1;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  Workspace *w = g_ws.at(dev);
  if (!w) return TOPS_E_INVALID;
  *out = w;
  return TOPS_OK;
}

static inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

#define TOPS_TRY(expr)            \
  do {                            \
    int _s = (expr);              \
    if (_s != TOPS_OK) return _s; \
  } while (0)

struct LutScratch {
  int dev = -1;
  tops_lut_dev *lut = nullptr;
  std::vector<float> kaz, krg;
  ~LutScratch() {
    if (!lut) return;
    int cur = -1;
    const bool have_cur = cudaGetDevice(&cur) == cudaSuccess;
    if (cudaSetDevice(dev) == cudaSuccess) tops_lut_destroy(lut);
    if (have_cur) cudaSetDevice(cur);
  }
};
static thread_local DeviceSlots<LutScratch, kMaxDevices> g_lut;

// The reference passes its host LUT on every call; keep one device copy per
// (thread, device) and refresh it when the caller's table changes.
static int lut_for(const float *kaz, const float *krg, int npoints, tops_lut_dev **out) {
  if (npoints != kTaps) return TOPS_E_INVALID;
  int dev = -1;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  LutScratch *gp = g_lut.at(dev);
  if (!gp) return TOPS_E_INVALID;
  LutScratch &g = *gp;
  const size_t n = (size_t)kLutBins * kTaps;
  if (!g.lut || memcmp(g.kaz.data(), kaz, n * sizeof(float)) ||
      memcmp(g.krg.data(), krg, n * sizeof(float))) {
    if (g.lut) tops_lut_destroy(g.lut);
    g.lut = nullptr;
    TOPS_TRY(tops_lut_create(kaz, krg, &g.lut));
    g.kaz.assign(kaz, kaz + n);
    g.krg.assign(krg, krg + n);
  }
  *out = g.lut;
  return TOPS_OK;
}

// Shared body of DerampDemodResample and DerampDemodResample_ESD.  When
// d_keep is non-null a fresh contiguous device copy of the output is
// returned through it (ownership to the caller).
static int resample_host(void *SlaveArray, const double *CpmAz, const double *CpmRg,
                         double AzimuthShift, void *output, const float *KernelAz,
                         const float *KernelRg, int sBurstIdx, const int MasterBox[4],
                         const int SlaveBox[4], int linesPerBurst, int SamplesPerBurst,
                         double dt, const double *kt, const double *tref, const double *fdc,
                         int Npoints, void **d_keep) {
  if (!SlaveArray || !CpmAz || !CpmRg || !output || !KernelAz || !KernelRg || !MasterBox ||
      !SlaveBox || !kt || !tref || !fdc)
    return TOPS_E_INVALID;
  const int sLines = SlaveBox[3] - SlaveBox[2] + 1, sPixels = SlaveBox[1] - SlaveBox[0] + 1;
  const int mLines = MasterBox[3] - MasterBox[2] + 1, mPixels = MasterBox[1] - MasterBox[0] + 1;
  if (sLines <= 0 || sPixels <= 0 || mLines <= 0 || mPixels <= 0) return TOPS_E_INVALID;
  if (SlaveBox[0] < 0 || SlaveBox[1] >= SamplesPerBurst) return TOPS_E_INVALID;
  tops_lut_dev *lut;
  TOPS_TRY(lut_for(KernelAz, KernelRg, Npoints, &lut));
  Workspace *ws;
  TOPS_TRY(workspace(&ws));
  cudaStream_t st = cudaStreamPerThread;
  const size_t spitch = align_up((size_t)sPixels * 4, 256);
  const size_t opitch = align_up((size_t)mPixels * 8, 256);
  void *d_slave, *d_out, *d_par;
  TOPS_TRY(ws->get(0, spitch * sLines, &d_slave));
  TOPS_TRY(ws->get(1, opitch * mLines, &d_out));
  TOPS_TRY(ws->get(2, 3 * sizeof(double) * (size_t)SamplesPerBurst, &d_par));
  double *d_kt = static_cast<double *>(d_par), *d_tref = d_kt + SamplesPerBurst,
         *d_fdc = d_tref + SamplesPerBurst;
  TOPS_CUDA_TRY(cudaMemcpy2DAsync(d_slave, spitch, SlaveArray, (size_t)sPixels * 4,
                                  (size_t)sPixels * 4, sLines, cudaMemcpyHostToDevice, st));
  TOPS_CUDA_TRY(cudaMemcpyAsync(d_kt, kt, sizeof(double) * SamplesPerBurst,
                                cudaMemcpyHostToDevice, st));
  TOPS_CUDA_TRY(cudaMemcpyAsync(d_tref, tref, sizeof(double) * SamplesPerBurst,
                                cudaMemcpyHostToDevice, st));
  TOPS_CUDA_TRY(cudaMemcpyAsync(d_fdc, fdc, sizeof(double) * SamplesPerBurst,
                                cudaMemcpyHostToDevice, st));
  tops_resample_job job;
  memset(&job, 0, sizeof(job));
  job.slave = d_slave;
  job.slave_pitch = spitch;
  job.out = d_out;
  job.out_pitch = opitch;
  job.kt = d_kt;
  job.tref = d_tref;
  job.fdc = d_fdc;
  for (int i = 0; i < 4; i++) {
    job.mbox[i] = MasterBox[i];
    job.sbox[i] = SlaveBox[i];
  }
  for (int i = 0; i < 6; i++) {
    job.cpm_az[i] = CpmAz[i];
    job.cpm_rg[i] = CpmRg[i];
  }
  job.az_shift = AzimuthShift;
  job.s_first_line = sBurstIdx * linesPerBurst;
  job.dt = dt;
  job.out_rows = -1;
  TOPS_TRY(tops_resample(lut, &job, 1, st));
  TOPS_CUDA_TRY(cudaMemcpy2DAsync(output, (size_t)mPixels * 8, d_out, opitch, (size_t)mPixels * 8,
                                  mLines, cudaMemcpyDeviceToHost, st));
  if (d_keep) {
    void *keep = nullptr;
    cudaError_t e = cudaMalloc(&keep, (size_t)mPixels * 8 * mLines);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      return TOPS_E_NOMEM;
    }
    TOPS_CUDA_TRY(cudaMemcpy2DAsync(keep, (size_t)mPixels * 8, d_out, opitch,
                                    (size_t)mPixels * 8, mLines, cudaMemcpyDeviceToDevice, st));
    *d_keep = keep;
  }
  TOPS_CUDA_TRY(cudaStreamSynchronize(st));
  return TOPS_OK;
}

static int coherence_host(int Dw, int Dh, int dx, int dy, int winRg, int winAz,
                          void *masterArray, void *d_slave, float *cohdata) {
  if (!masterArray || !d_slave || !cohdata || Dw <= 0 || Dh <= 0) return TOPS_E_INVALID;
  // the box offsets are fixed by the window in this path (Func.cpp:2643-2644)
  if (dx != (winRg - 1) / 2 || dy != (winAz - 1) / 2) return TOPS_E_INVALID;
  cudaStream_t st = cudaStreamPerThread;
  const size_t mpitch = align_up((size_t)Dw * 4, 256), cpitch = align_up((size_t)Dw * 4, 256);
  void *d_m, *d_c;
  Workspace *ws;
  TOPS_TRY(workspace(&ws));
  TOPS_TRY(ws->get(3, mpitch * Dh, &d_m));
  TOPS_TRY(ws->get(4, cpitch * Dh, &d_c));
  TOPS_CUDA_TRY(cudaMemcpy2DAsync(d_m, mpitch, masterArray, (size_t)Dw * 4, (size_t)Dw * 4, Dh,
                                  cudaMemcpyHostToDevice, st));
  tops_coh_job j{d_m, mpitch, d_slave, (size_t)Dw * 8, static_cast<float *>(d_c), cpitch, Dh, Dw};
  CohJob J;
  TOPS_TRY(fill_coh_job(j, J));
  TOPS_TRY(launch_coherence(&J, 1, winRg, winAz, TileCfg(), st));
  TOPS_CUDA_TRY(cudaMemcpy2DAsync(cohdata, (size_t)Dw * 4, d_c, cpitch, (size_t)Dw * 4, Dh,
                                  cudaMemcpyDeviceToHost, st));
  TOPS_CUDA_TRY(cudaStreamSynchronize(st));
  TOPS_CUDA_TRY(cudaFree(d_slave));
  return TOPS_OK;
}

}  // namespace tops

using namespace tops;

extern "C" {

const char *tops_status_string(int s) {
  switch (s) {
    case TOPS_OK: return "ok";
    case TOPS_E_INVALID: return "invalid argument";
    case TOPS_E_CUDA: return "CUDA error";
    case TOPS_E_NOMEM: return "out of memory";
    case TOPS_E_NOT_PD: return "normal matrix not positive definite";
    case TOPS_E_TIMEOUT: return "device wait timed out";
    case TOPS_E_BUDGET: return "footprint above the HBM budget";
    case TOPS_E_CONFIG: return "malformed config";
    case TOPS_E_NODEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

int tops_last_cuda_error(void) { return g_last_cuda_error; }

const char *tops_version(void) { return "tops_b200 0.1.0 (sm_100a)"; }

int tops_stream_synchronize(void *stream) {
  TOPS_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return TOPS_OK;
}

int GeoCoreg_warp_cuda(int m_burstIdx, int s_burstIdx, int xmin, int xmax, int ymin, int ymax,
                       double dem_DeltaLat, double dem_DeltaLon, int DemLines, int DemPixels,
                       double *AzCpm, double *RgCpm, double lat0, double lon0, int demnodata,
                       double m_azimuthTimeInterval, double s_azimuthTimeInterval,
                       double wavelength, double m_linesPerBurst, double s_linesPerBurst,
                       double m_burstFirstLineTime, double s_burstFirstLineTime,
                       int m_numOfSamples, int s_numOfSamples, double *m_orbitAzTime,
                       double *s_orbitAzTime, int orb_m_numberofpoints, int orb_m_numbercoefs,
                       int orb_s_numberofpoints, int orb_s_numbercoefs,
                       double m_slrTimeToFirstPixel, double s_slrTimeToFirstPixel,
                       double m_rangeSpacing, double s_rangeSpacing, bool m_nearRangeOnLeft,
                       bool s_nearRangeOnLeft, int *inputDEM, double *m_x_coef, double *m_y_coef,
                       double *m_z_coef, double *s_x_coef, double *s_y_coef, double *s_z_coef,
                       double m_aziInitial, double s_aziInitial) {
  (void)wavelength;
  (void)m_numOfSamples;
  (void)s_numOfSamples;
  (void)m_nearRangeOnLeft;
  (void)s_nearRangeOnLeft;
  if (!AzCpm || !RgCpm || !inputDEM || !m_orbitAzTime || !s_orbitAzTime || !m_x_coef ||
      !m_y_coef || !m_z_coef || !s_x_coef || !s_y_coef || !s_z_coef || DemLines <= 0 ||
      DemPixels <= 0 || orb_m_numberofpoints <= 0 || orb_s_numberofpoints <= 0)
    return TOPS_E_INVALID;
  cudaStream_t st = cudaStreamPerThread;
  const size_t dpitch = align_up((size_t)DemPixels * 4, 256);
  void *d_dem, *d_out;
  Workspace *ws;
  TOPS_TRY(workspace(&ws));
  TOPS_TRY(ws->get(5, dpitch * DemLines, &d_dem));
  TOPS_TRY(ws->get(6, 256, &d_out));
  TOPS_CUDA_TRY(cudaMemcpy2DAsync(d_dem, dpitch, inputDEM, (size_t)DemPixels * 4,
                                  (size_t)DemPixels * 4, DemLines, cudaMemcpyHostToDevice, st));
  tops_geo_job g;
  memset(&g, 0, sizeof(g));
  g.dem = static_cast<const float *>(d_dem);
  g.dem_pitch = dpitch;
  g.dem_lines = DemLines;
  g.dem_pixels = DemPixels;
  g.lat0 = lat0;
  g.lon0 = lon0;
  g.dlat = dem_DeltaLat;
  g.dlon = dem_DeltaLon;
  g.nodata = demnodata;
  g.xmin = xmin;
  g.xmax = xmax;
  g.ymin = ymin;
  g.ymax = ymax;
  const double *cf[2][3] = {{m_x_coef, m_y_coef, m_z_coef}, {s_x_coef, s_y_coef, s_z_coef}};
  const int nc[2] = {orb_m_numbercoefs, orb_s_numbercoefs};
  g.dt[0] = m_azimuthTimeInterval;
  g.dt[1] = s_azimuthTimeInterval;
  g.first_line_time[0] = m_burstFirstLineTime;
  g.first_line_time[1] = s_burstFirstLineTime;
  g.slr_time[0] = m_slrTimeToFirstPixel;
  g.slr_time[1] = s_slrTimeToFirstPixel;
  g.range_spacing[0] = m_rangeSpacing;
  g.range_spacing[1] = s_rangeSpacing;
  g.mid_time[0] = m_orbitAzTime[orb_m_numberofpoints / 2];
  g.mid_time[1] = s_orbitAzTime[orb_s_numberofpoints / 2];
  g.azi_init[0] = m_aziInitial;
  g.azi_init[1] = s_aziInitial;
  g.line_offset[0] = (int)(m_burstIdx * m_linesPerBurst);
  g.line_offset[1] = (int)(s_burstIdx * s_linesPerBurst);
  for (int k = 0; k < 2; k++) {
    if (nc[k] < 2 || nc[k] > 8) return TOPS_E_INVALID;
    g.ncoef[k] = nc[k];
    for (int a = 0; a < 3; a++)
      for (int i = 0; i < nc[k]; i++) g.coef[k][a][i] = cf[k][a][i];
  }
  double *d_cpm = static_cast<double *>(d_out);
  int *d_status = reinterpret_cast<int *>(d_cpm + 12);
  g.cpm_dev = d_cpm;
  g.status_dev = d_status;
  GeoJob J;
  TOPS_TRY(fill_geo_job(g, J));
  void *d_scr;
  size_t scr = geocoreg_scratch(&J, 1);
  TOPS_TRY(ws->get(7, scr, &d_scr));
  TOPS_TRY(launch_geocoreg(&J, 1, true, d_scr, scr, st));
  double h[13];
  TOPS_CUDA_TRY(cudaMemcpyAsync(h, d_cpm, 13 * sizeof(double), cudaMemcpyDeviceToHost, st));
  TOPS_CUDA_TRY(cudaStreamSynchronize(st));
  int status;
  memcpy(&status, &h[12], sizeof(int));
  if (status != TOPS_OK) {
    fprintf(stderr, "Error: Cholesky factorization failed\n");
    return TOPS_E_NOT_PD;  // AzCpm/RgCpm left unchanged, as the reference
  }
  for (int i = 0; i < 6; i++) {
    AzCpm[i] = h[i];
    RgCpm[i] = h[6 + i];
  }
  return TOPS_OK;
}

int DerampDemodResample(void *SlaveArray, double *CpmAz, double *CpmRg, double AzimuthShift,
                        void *output, float *KernelAz, float *KernelRg, int sBurstIdx,
                        int slave_pixels, int slave_lines, int MasterBox[4], int SlaveBox[4],
                        int S_linesPerBurst, int S_SamplesPerBurst, double azimuthTimeInterval,
                        double *dopplerRate, double *referenceTime, double *dopplerCentroid,
                        int Npoints) {
  (void)slave_pixels;
  (void)slave_lines;
  return resample_host(SlaveArray, CpmAz, CpmRg, AzimuthShift, output, KernelAz, KernelRg,
                       sBurstIdx, MasterBox, SlaveBox, S_linesPerBurst, S_SamplesPerBurst,
                       azimuthTimeInterval, dopplerRate, referenceTime, dopplerCentroid, Npoints,
                       nullptr);
}

void *DerampDemodResample_ESD(void *SlaveArray, double *CpmAz, double *CpmRg,
                              double AzimuthShift, void *output, float *KernelAz,
                              float *KernelRg, int sBurstIdx, int slave_pixels, int slave_lines,
                              int MasterBox[4], int SlaveBox[4], int linesPerBurst,
                              int SamplesPerBurst, double azimuthTimeInterval,
                              double *dopplerRate, double *referenceTime,
                              double *dopplerCentroid, int Npoints) {
  (void)slave_pixels;
  (void)slave_lines;
  void *keep = nullptr;
  int s = resample_host(SlaveArray, CpmAz, CpmRg, AzimuthShift, output, KernelAz, KernelRg,
                        sBurstIdx, MasterBox, SlaveBox, linesPerBurst, SamplesPerBurst,
                        azimuthTimeInterval, dopplerRate, referenceTime, dopplerCentroid,
                        Npoints, &keep);
  if (s != TOPS_OK) {
    if (keep) cudaFree(keep);
    return nullptr;
  }
  return keep;
}

void *ResampleFirstBurst(void *SlaveArray, int ww, int hh) {
  if (!SlaveArray || ww <= 0 || hh <= 0) return nullptr;
  cudaStream_t st = cudaStreamPerThread;
  void *d = nullptr;
  cudaError_t e = cudaMalloc(&d, (size_t)ww * hh * 8);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d, SlaveArray, (size_t)ww * hh * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    if (d) cudaFree(d);
    return nullptr;
  }
  return d;
}

int tops_free_device(void *d_ptr) {
  if (!d_ptr) return TOPS_OK;
  TOPS_CUDA_TRY(cudaStreamSynchronize(cudaStreamPerThread));
  TOPS_CUDA_TRY(cudaFree(d_ptr));
  return TOPS_OK;
}

int EstESDShifts(void *MasterFor, void *MasterBack, void *SlaveFor, void *SlaveBack,
                 int *OverlapSizeArray, double *ShiftArray, int numOverlap, int ArrayLines,
                 int ArrayPixels, int CohWinAz, int CohWinRg, int OverlapMaxLines,
                 float CohThresHold, double spectralSeparation, double azimuthTimeInterval) {
  (void)OverlapMaxLines;
  if (!MasterFor || !MasterBack || !SlaveFor || !SlaveBack || !OverlapSizeArray || !ShiftArray ||
      numOverlap <= 0 || ArrayPixels <= 0)
    return TOPS_E_INVALID;
  long tot = 0;
  for (int i = 0; i < numOverlap; i++) {
    if (OverlapSizeArray[i] < 0) return TOPS_E_INVALID;
    tot += OverlapSizeArray[i];
  }
  if (tot > ArrayLines) return TOPS_E_INVALID;
  cudaStream_t st = cudaStreamPerThread;
  const size_t mbytes = (size_t)tot * ArrayPixels * 4, sbytes = (size_t)tot * ArrayPixels * 8;
  void *d_m, *d_s, *d_o;
  Workspace *ws;
  TOPS_TRY(workspace(&ws));
  TOPS_TRY(ws->get(8, 2 * mbytes, &d_m));
  TOPS_TRY(ws->get(9, 2 * sbytes, &d_s));
  TOPS_TRY(ws->get(10, sizeof(double) * 3 * (size_t)numOverlap, &d_o));
  char *mF = static_cast<char *>(d_m), *mB = mF + mbytes;
  char *sF = static_cast<char *>(d_s), *sB = sF + sbytes;
  TOPS_CUDA_TRY(cudaMemcpyAsync(mF, MasterFor, mbytes, cudaMemcpyHostToDevice, st));
  TOPS_CUDA_TRY(cudaMemcpyAsync(mB, MasterBack, mbytes, cudaMemcpyHostToDevice, st));
  TOPS_CUDA_TRY(cudaMemcpyAsync(sF, SlaveFor, sbytes, cudaMemcpyHostToDevice, st));
  TOPS_CUDA_TRY(cudaMemcpyAsync(sB, SlaveBack, sbytes, cudaMemcpyHostToDevice, st));
  std::vector<EsdOverlap> O(numOverlap);
  long off = 0;
  for (int i = 0; i < numOverlap; i++) {
    tops_esd_overlap u;
    u.mF = mF + off * ArrayPixels * 4;
    u.mB = mB + off * ArrayPixels * 4;
    u.sF = sF + off * ArrayPixels * 8;
    u.sB = sB + off * ArrayPixels * 8;
    u.m_pitch = (size_t)ArrayPixels * 4;
    u.s_pitch = (size_t)ArrayPixels * 8;
    u.lines = OverlapSizeArray[i];
    u.pixels = ArrayPixels;
    u.spec_sep = spectralSeparation;
    u.dt = azimuthTimeInterval;
    TOPS_TRY(fill_esd_overlap(u, O[i]));
    off += OverlapSizeArray[i];
  }
  size_t scr = esd_scratch_bytes(O.data(), numOverlap);
  void *d_scr;
  TOPS_TRY(ws->get(11, scr, &d_scr));
  double *d_shift = static_cast<double *>(d_o);
  TOPS_TRY(launch_esd(O.data(), numOverlap, CohWinAz, CohWinRg, CohThresHold, d_shift, nullptr,
                      d_scr, scr, st, 0));
  TOPS_CUDA_TRY(cudaMemcpyAsync(ShiftArray, d_shift, sizeof(double) * numOverlap,
                                cudaMemcpyDeviceToHost, st));
  TOPS_CUDA_TRY(cudaStreamSynchronize(st));
  return TOPS_OK;
}

int CoherenceEst(int Dx0, int Dy0, int Dw, int Dh, int dx, int dy, int cohWinRg, int cohWinAz,
                 void *masterArray, void *d_slaveArray, float *cohdata) {
  (void)Dx0;
  (void)Dy0;
  return coherence_host(Dw, Dh, dx, dy, cohWinRg, cohWinAz, masterArray, d_slaveArray, cohdata);
}

int CoherenceEst_ESD(int Dx0, int Dy0, int Dw, int Dh, int dx, int dy, int cohWinRg,
                     int cohWinAz, void *masterArray, void *d_slaveArray, float *cohdata) {
  (void)Dx0;
  (void)Dy0;
  return coherence_host(Dw, Dh, dx, dy, cohWinRg, cohWinAz, masterArray, d_slaveArray, cohdata);
}

}  // extern "C"

// common.cuh -- shared device helpers and internal job layouts for the
// B200 TOPS burst-pair kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>

#include "tops_b200.h"

namespace tops {

// ------------------------------------------------------------ status
// Thread-local record of the last CUDA error (tops_last_cuda_error()).
void set_cuda_error(cudaError_t e);

// On failure: record the error, clear the thread's last-error state (so a
// later, unrelated launch check does not report it again) and return.
#define TOPS_CUDA_TRY(expr)                      \
  do {                                           \
    cudaError_t _e = (expr);                     \
    if (_e != cudaSuccess) {                     \
      ::tops::set_cuda_error(_e);                \
      (void)cudaGetLastError();                  \
      return (_e == cudaErrorMemoryAllocation) ? TOPS_E_NOMEM : TOPS_E_CUDA; \
    }                                            \
  } while (0)

// --------------------------------------------------------- constants
constexpr double kPi = 3.1415926535897931e+0;       // reference Constants.h:7
constexpr double kSol = 299792458.0;                // reference Constants.h:6
constexpr int kInterval = 2047;                     // reference Constants.h:8
constexpr int kLutBins = 2048;
constexpr int kTaps = 12;
constexpr int kMaxDevices = 64;
constexpr double kTwoPiHi = 6.283185307179586232e+00;
constexpr double kTwoPiLo = 2.449293598294706414e-16;
constexpr double kInvTwoPi = 0.15915494309189533577;

// ------------------------------------------- per-device one-time set-up
// Function attributes and occupancy queries are per device.  The first host
// thread that launches on a device runs init(value) under the lock and
// publishes the positive value it produced; later callers read it without
// locking.  A failed init is not published, so the next call retries it.
struct PerDeviceOnce {
  std::mutex mu;
  std::atomic<int> value[kMaxDevices]{};
};

template <class F>
int once_per_device(PerDeviceOnce &o, int dev, F init, int *out) {
  if (dev < 0 || dev >= kMaxDevices) return TOPS_E_INVALID;
  int v = o.value[dev].load(std::memory_order_acquire);
  if (v == 0) {
    std::lock_guard<std::mutex> lock(o.mu);
    v = o.value[dev].load(std::memory_order_relaxed);
    if (v == 0) {
      int r = 1;
      const int s = init(r);
      if (s != TOPS_OK) return s;
      v = r > 0 ? r : 1;
      o.value[dev].store(v, std::memory_order_release);
    }
  }
  if (out) *out = v;
  return TOPS_OK;
}

// Cody-Waite reduction of a double phase to [-pi, pi] with a two-term 2*pi,
// returned as float.  Exact to ~1e-15 rad for |phi| < 1e9.
__device__ __forceinline__ float reduce_2pi(double phi) {
  double n = rint(phi * kInvTwoPi);
  double r = fma(-n, kTwoPiHi, phi);
  r = fma(-n, kTwoPiLo, r);
  return (float)r;
}

// Shared-memory index padding: one slot every 8 elements, so threads that
// each own 8 consecutive elements (lanes 8 apart) hit distinct banks.
__host__ __device__ constexpr int pad8(int x) { return x + (x >> 3); }

// Float reduction for small arguments (|x| < ~1e3) before __sincosf.
__device__ __forceinline__ float reduce_2pi_f(float x) {
  float n = rintf(x * 0.15915494309189535f);
  x = fmaf(-n, 6.28318548202514648f, x);
  x = fmaf(-n, -1.7484556e-07f, x);
  return x;
}

// ------------------------------------------------- internal job layouts
// Device copies of the interpolation kernels (tops_lut_dev).
struct LutPtrs {
  const float *kaz, *krg;  // [2048][12]
  const float4 *krg2;      // [2048][6]: range taps duplicated (w0,w0,w1,w1), ...
  const float *sp1;        // [2048]: sum(krg row) - 1
};

// Device-side view of one resample job (built from tops_resample_job).
struct ResampleJob {
  LutPtrs lut;            // interpolation kernels of the job's sub-swath
  const short2 *slave;
  long slave_pitch;       // short2 elements per row
  float2 *out;
  long out_pitch;         // float2 elements per row
  int slave_al8;          // slave base and pitch 8-byte aligned (pair loads)
  int out_al16;           // output base and pitch 16-byte aligned (pair stores)
  const double *kt, *tref, *fdc;
  int mx0, mx1, my0, my1;
  int sx0, sx1, sy0, sy1;
  double caz[6], crg[6];
  double az_shift;
  const double *az_shift_dev;
  const double *cpm_dev;  // if set: 6 azimuth then 6 range coefficients
  int s_first_line;
  double dt;
  int row0, nrows;        // master rows [row0, row0+nrows) (0-based in box)
  // normalizeWarp constants: (v - mid) * inv
  double midP, invP, midL, invL;
  // work decomposition
  int strips, segs, seg_rows;
  int item_begin;         // first global work item of this job
};

struct CohJob {
  const short2 *master;
  long master_pitch;      // elements
  const float2 *slave;
  long slave_pitch;
  float *coh;
  long coh_pitch;
  int lines, pixels;
  int strips, segs, seg_rows;
  int item_begin;
};

struct EsdOverlap {
  const short2 *mF, *mB;
  long m_pitch;
  const float2 *sF, *sB;
  long s_pitch;
  int lines, pixels;
  double spec_sep, dt;
  int strips, segs, seg_rows;
  int item_begin;
};

struct GeoJob {
  const float *dem;
  long dem_pitch;         // floats per row
  int lines, pixels;
  double lat0, lon0, dlat, dlon, nodata;
  int xmin, xmax, ymin, ymax;
  double dt[2], first_line_time[2], slr_time[2], range_spacing[2];
  double inv_dt[2], inv_range_spacing[2];   // reciprocals (host FP64)
  double inv_yq, inv_xq;                     // 1 / (span / 4) of the master box
  double mid_time[2], azi_init[2];
  int line_offset[2];
  double coef[2][3][8];
  int ncoef[2];
  double *cpm;
  int *status;
  int blocks;             // blocks assigned to this job
  int block_begin;
};

}  // namespace tops

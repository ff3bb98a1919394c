// geocoreg.cu -- DEM-assisted geometric coregistration (sm_100a, FP64).
//
// Reference (GeoCoreg_warp_cuda, Geocoreg_cuda.cu:610-913): per DEM pixel
//   llh2xyz (:87-99) -> ECEF target; for master and slave a zero-Doppler
//   Newton solve (ell2lpGeo :211-323 with getPos/getVelo/getAcc :123-205
//   and SolveNewtonEq :101-112, <= 11 iterations, |step| < 1e-10 s) giving
//   (line, pixel); weight 1 if the DEM is valid and the master position is
//   inside the burst box (WeighthSet :548-574); A row [1, L, P, L^2, LP, P^2]
//   of the normalised master position (AMatrixSet :576-605); then
//   N = (WA)^T A, rhs = (WA)^T {slave line, slave pixel} by cuBLAS and a
//   Cholesky solve by cuSOLVER (:822-851).
//
// B200 design: one fused kernel.  A block walks tiles of GC_TR DEM rows x
// GC_NT columns; the sine, cosine and prime-vertical radius of each tile row
// and the sine and cosine of each column are computed once per tile (the
// reference computes them per pixel; the values are the same), then each
// thread geocodes its column's pixels (master and slave share the target
// position) and accumulates the 21 distinct
// entries of N and the two right-hand sides (33 FP64 sums) in registers;
// the block reduces them with warp shuffles in a fixed order and writes one
// partial per block.  A one-block kernel per burst sums the partials in a
// fixed order and solves the 6x6 system with the reference's own Cholesky
// scheme (Func.cpp:959-1013).  No per-pixel buffers touch HBM; results are
// bit-for-bit reproducible run to run.  Orbit polynomials and their first
// two derivatives are evaluated with Horner's rule instead of pow(), and
// the Newton step folds the reference's velocity / 10 and acceleration / 100
// scalings into one division; the root and the stopping rule are the
// reference's, the rounding of the iterates differs in the last bits.  Down
// a column, each solve starts from the previous solutions extrapolated
// linearly, and its first Newton step takes the orbit state there from a
// Taylor shift of the previous solve's position, velocity and acceleration
// (kept in shared memory), so most solves need one polynomial evaluation.
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace tops {

constexpr int GC_NT = 256;
constexpr int GC_TR = 32;   // DEM rows per tile (each starts its columns' Newton chains afresh)
constexpr int GC_MAXJOBS = 16;
constexpr int GC_NSUM = 33;
constexpr double kEllA = 6378137.0;                              // cuConstants.cuh:5
constexpr double kEllB = 6356752.3142451794975639665996337;      // cuConstants.cuh:6

struct GcBatch {
  int njobs, total_blocks;
  int dem_is_int;
  GeoJob jobs[GC_MAXJOBS];
};

// Position and the first two derivatives with respect to the normalised time
// t of an orbit polynomial (getPos/getVelo/getAcc, Geocoreg_cuda.cu:123-205,
// return the derivatives divided by 10 and 100).
// The same with the coefficient count N known at compile time (fully
// unrolled; the orbit fit returns 6 coefficients for more than 6 state
// vectors, Func.cpp:1050-1126).
template <int N>
__device__ __forceinline__ void orbit_eval_n(const double (*c)[8], double t, double p[3],
                                             double v[3], double a[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double pp = c[k][N - 1], vv = 0.0, aa = 0.0;
#pragma unroll
    for (int i = N - 2; i >= 0; --i) {
      aa = fma(aa, t, 2.0 * vv);
      vv = fma(vv, t, pp);
      pp = fma(pp, t, c[k][i]);
    }
    p[k] = pp;
    v[k] = vv;
    a[k] = aa;
  }
}

__device__ __forceinline__ void orbit_eval(const double (*c)[8], int n, double t, double p[3],
                                           double v[3], double a[3]) {
  if (n == 6) {
    orbit_eval_n<6>(c, t, p, v, a);
    return;
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double pp = c[k][n - 1], vv = 0.0, aa = 0.0;
    for (int i = n - 2; i >= 0; --i) {
      aa = fma(aa, t, 2.0 * vv);
      vv = fma(vv, t, pp);
      pp = fma(pp, t, c[k][i]);
    }
    p[k] = pp;
    v[k] = vv;
    a[k] = aa;
  }
}

__device__ __forceinline__ void orbit_pos(const double (*c)[8], int n, double t, double p[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    double pp = c[k][n - 1];
    for (int i = n - 2; i >= 0; --i) pp = fma(pp, t, c[k][i]);
    p[k] = pp;
  }
}

// Zero-Doppler (line, pixel) of target T for image k of job J.
// 1/x: the hardware's approximate FP64 reciprocal refined by two
// Newton-Raphson steps r <- r + r (1 - x r) (each doubles the correct bits;
// a Newton step of the zero-Doppler solve needs no correctly rounded
// quotient, only its root does not move)
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}

// az: the Newton start on entry (the reference starts every pixel at the
// burst-centre time; here a thread starts from the solutions of the pixels
// above in its column, extrapolated linearly, which converges to the same
// root in fewer steps), the zero-Doppler azimuth time on return.  st: the
// orbit position, velocity and acceleration at the last solution of this
// column (9 doubles at a stride of GC_NT in shared memory), valid when have
// is set, and delta = start - that solution.  The first Newton step then
// takes the orbit state at the start from a Taylor shift of st (a few FMAs)
// instead of a polynomial evaluation; on return st holds this solve's state.
__device__ void ell2lp(const GeoJob &J, int k, const double T[3], double &az, double delta,
                       double &line, double &pixel, double *st, bool &have) {
  const double (*c)[8] = J.coef[k];
  const int n = J.ncoef[k];
  double P[3], V[3], A[3];
  double sol = 0.0;
  int it0 = 0;
  if (have) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      // shift by dt = delta / 10 in normalised time (third-order term: below
      // 1e-9 m for the millisecond steps between DEM rows)
      const double dt = 0.1 * delta;
      const double a = st[(6 + q) * GC_NT], v = st[(3 + q) * GC_NT];
      P[q] = fma(dt, fma(0.5 * dt, a, v), st[q * GC_NT]);
      V[q] = fma(dt, a, v);
      A[q] = a;
    }
    const double dx = T[0] - P[0], dy = T[1] - P[1], dz = T[2] - P[2];
    sol = -10.0 * (V[0] * dx + V[1] * dy + V[2] * dz) *
          rcp_nr((A[0] * dx + A[1] * dy + A[2] * dz) - V[0] * V[0] - V[1] * V[1] - V[2] * V[2]);
    az += sol;
    it0 = 1;   // that step is the solve's first iteration
  }
  // at least one step from an exact orbit evaluation, also when the shifted
  // step is already below the bound: the zero-Doppler root is sensitive to
  // the velocity's direction, which the shift only approximates
  for (int it = it0; it <= 10 && !(it > it0 && fabs(sol) < 1e-010); it++) {
    const double t = (az - J.mid_time[k]) * 0.1;
    orbit_eval(c, n, t, P, V, A);
    const double dx = T[0] - P[0], dy = T[1] - P[1], dz = T[2] - P[2];
    // -(V/10 . d) / ((A/100 . d) - |V/10|^2) (SolveNewtonEq, :101-112)
    sol = -10.0 * (V[0] * dx + V[1] * dy + V[2] * dz) *
          rcp_nr((A[0] * dx + A[1] * dy + A[2] * dz) - V[0] * V[0] - V[1] * V[1] - V[2] * V[2]);
    az += sol;
    if (fabs(sol) < 1e-010) break;
  }
  // position at the final az: from the last evaluation and one Taylor term
  // when the last step was below the stopping bound (dP/daz = V / 10; the
  // next term is below 1e-19 m), else evaluated afresh
  if (fabs(sol) < 1e-010) {
#pragma unroll
    for (int q = 0; q < 3; q++) P[q] = fma(0.1 * sol, V[q], P[q]);
  } else {
    orbit_pos(c, n, (az - J.mid_time[k]) * 0.1, P);
  }
  line = J.line_offset[k] + (az - J.first_line_time[k]) * J.inv_dt[k];
  const double r = sqrt((T[0] - P[0]) * (T[0] - P[0]) + (T[1] - P[1]) * (T[1] - P[1]) +
                        (T[2] - P[2]) * (T[2] - P[2]));
  pixel = (r - J.slr_time[k] * kSol) * J.inv_range_spacing[k];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    st[q * GC_NT] = P[q];
    st[(3 + q) * GC_NT] = V[q];
    st[(6 + q) * GC_NT] = A[q];
  }
  have = true;
}

__global__ void __launch_bounds__(GC_NT, 2) geocoreg_kernel(const __grid_constant__ GcBatch B,
                                                         double *partials) {
  __shared__ double red[GC_NT / 32][GC_NSUM];
  __shared__ double row_s[GC_TR], row_c[GC_TR], row_n[GC_TR];
  __shared__ double ostate[2][9][GC_NT];   // last solve's orbit state per thread and image
  const int blk = blockIdx.x;
  if (blk >= B.total_blocks) return;
  int jb = 0;
  while (jb + 1 < B.njobs && B.jobs[jb + 1].block_begin <= blk) jb++;
  const GeoJob &J = B.jobs[jb];
  const int lblk = blk - J.block_begin;
  const double e2 = 1.0 - (kEllB * kEllB / kEllA / kEllA);
  const double d2r = kPi / 180.0;
  const int tiles_x = (J.pixels + GC_NT - 1) / GC_NT;
  const int tiles = tiles_x * ((J.lines + GC_TR - 1) / GC_TR);
  const double ymid = 0.5 * ((double)J.ymin + (double)J.ymax);
  const double xmid = 0.5 * ((double)J.xmin + (double)J.xmax);
  // sums of the monomials L^i P^j (i + j <= 4) of the design row a = (1, L,
  // P, L^2, LP, P^2) -- its 21 distinct products a_i a_j are 15 monomials --
  // and of a_i times the slave line and pixel: 27 accumulators, expanded to
  // the 33 normal-equation sums after the loop
  constexpr int GC_NMOM = 27;
  double acc[GC_NMOM];
#pragma unroll
  for (int q = 0; q < GC_NMOM; q++) acc[q] = 0.0;

  for (int tile = lblk; tile < tiles; tile += J.blocks) {
    const int row0 = (tile / tiles_x) * GC_TR;
    const int col = (tile % tiles_x) * GC_NT + threadIdx.x;
    // llh2xyz (Geocoreg_cuda.cu:87-99): the latitude terms per tile row, the
    // longitude terms per column
    __syncthreads();   // the previous tile's row terms are no longer read
    if (threadIdx.x < GC_TR && row0 + threadIdx.x < J.lines) {
      double sphi, cphi;
      sincos((J.lat0 - J.dlat * (row0 + threadIdx.x)) * d2r, &sphi, &cphi);
      row_s[threadIdx.x] = sphi;
      row_c[threadIdx.x] = cphi;
      row_n[threadIdx.x] = kEllA / sqrt(1.0 - e2 * sphi * sphi);
    }
    __syncthreads();
    if (col >= J.pixels) continue;
    double slam, clam;
    sincos((J.lon0 + J.dlon * col) * d2r, &slam, &clam);
    const int nr = min(GC_TR, J.lines - row0);
    double azm = J.azi_init[0], azs = J.azi_init[1];   // Newton starts down the column
    bool hm = false, hs = false;   // orbit state of a solve above held (master / slave)
    // per-row change of each solution between the last two solved rows (0
    // unless they are adjacent): the next row's start is extrapolated by it
    double dm = 0.0, ds = 0.0;
    int lm = -2, ls = -2;   // last row solved for master / slave
    for (int rr = 0; rr < nr; rr++) {
      const long off = (long)(row0 + rr) * J.dem_pitch + col;
      float h;
      if (B.dem_is_int)
        h = (float)reinterpret_cast<const int *>(J.dem)[off];
      else
        h = J.dem[off];
      if (h == (float)J.nodata) continue;
      const double sphi = row_s[rr], cphi = row_c[rr];
      const double nph = row_n[rr] + h;
      const double T[3] = {nph * cphi * clam, nph * cphi * slam, (nph - e2 * (nph - h)) * sphi};
      double ml, mp, sl, sp;
      {
        const double d = lm == rr - 1 ? dm : 0.0;
        double a = azm + d;
        ell2lp(J, 0, T, a, d, ml, mp, &ostate[0][0][threadIdx.x], hm);
        dm = (lm == rr - 1) ? a - azm : 0.0;
        azm = a;
        lm = rr;
      }
      if (!(ml >= J.ymin && ml <= J.ymax && mp >= J.xmin && mp <= J.xmax)) continue;
      {
        const double d = ls == rr - 1 ? ds : 0.0;
        double a = azs + d;
        ell2lp(J, 1, T, a, d, sl, sp, &ostate[1][0][threadIdx.x], hs);
        ds = (ls == rr - 1) ? a - azs : 0.0;
        azs = a;
        ls = rr;
      }
      const double L = (ml - ymid) * J.inv_yq;
      const double P = (mp - xmid) * J.inv_xq;
      const double L2 = L * L, LP = L * P, P2 = P * P;
      const double a[6] = {1.0, L, P, L2, LP, P2};
      // monomials in the order M00 M10 M01 M20 M11 M02 M30 M21 M12 M03 M40
      // M31 M22 M13 M04
      const double m[15] = {1.0, L, P, L2, LP, P2, L2 * L, L2 * P, L * P2, P2 * P,
                            L2 * L2, L2 * LP, L2 * P2, LP * P2, P2 * P2};
#pragma unroll
      for (int q = 0; q < 15; q++) acc[q] += m[q];
#pragma unroll
      for (int i = 0; i < 6; i++) {
        acc[15 + i] = fma(a[i], sl, acc[15 + i]);
        acc[21 + i] = fma(a[i], sp, acc[21 + i]);
      }
    }
  }
  // the 33 sums: a_i a_j (i <= j, row-major) from the monomials, then the
  // slave-line and slave-pixel sums
  constexpr int kMono[21] = {0, 1, 2, 3, 4, 5,     // 1 x (1 L P L2 LP P2)
                             3, 4, 6, 7, 8,        // L x (L P L2 LP P2)
                             5, 7, 8, 9,           // P x (P L2 LP P2)
                             10, 11, 12,           // L2 x (L2 LP P2)
                             12, 13,               // LP x (LP P2)
                             14};                  // P2 x P2
  // fixed-order block reduction
#pragma unroll
  for (int q = 0; q < GC_NSUM; q++) {
    double v = q < 21 ? acc[kMono[q]] : acc[q - 6];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < GC_NSUM) {
    double v = 0.0;
    for (int w = 0; w < GC_NT / 32; w++) v += red[w][threadIdx.x];
    partials[(long)blk * GC_NSUM + threadIdx.x] = v;
  }
}

// Cholesky solve of the 6x6 normal equations (choles/solvechol semantics,
// Func.cpp:959-1013); one block per job.
__global__ void geocoreg_solve_kernel(const __grid_constant__ GcBatch B, const double *partials) {
  __shared__ double tot[GC_NSUM];
  const GeoJob &J = B.jobs[blockIdx.x];
  if (threadIdx.x < GC_NSUM) {
    double v = 0.0;
    for (int b = 0; b < J.blocks; b++) v += partials[(long)(J.block_begin + b) * GC_NSUM + threadIdx.x];
    tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double n[36];
  int q = 0;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++) {
      n[i * 6 + j] = tot[q];
      n[j * 6 + i] = tot[q];
      q++;
    }
  int bad = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) {
      double sum = n[i * 6 + j];
      for (int k = i - 1; k >= 0; --k) sum -= n[i * 6 + k] * n[j * 6 + k];
      if (i == j) {
        if (!(sum > 0.0)) bad = 1;
        n[i * 6 + i] = sqrt(sum);
      } else {
        n[j * 6 + i] = sum / n[i * 6 + i];
      }
    }
  if (bad) {
    *J.status = TOPS_E_NOT_PD;
    return;
  }
  for (int r = 0; r < 2; r++) {
    double b[6];
    for (int i = 0; i < 6; i++) b[i] = tot[21 + 6 * r + i];
    for (int i = 0; i < 6; ++i) {
      double sum = b[i];
      for (int j = i - 1; j >= 0; --j) sum -= n[i * 6 + j] * b[j];
      b[i] = sum / n[i * 6 + i];
    }
    for (int i = 5; i >= 0; --i) {
      double sum = b[i];
      for (int j = i + 1; j < 6; ++j) sum -= n[j * 6 + i] * b[j];
      b[i] = sum / n[i * 6 + i];
    }
    for (int i = 0; i < 6; i++) J.cpm[6 * r + i] = b[i];
  }
  *J.status = TOPS_OK;
}

static int gc_blocks_for(int lines, int pixels) {
  // one block per tile up to 4096 blocks (a tile is GC_TR rows x GC_NT columns)
  long t = (long)((pixels + GC_NT - 1) / GC_NT) * ((lines + GC_TR - 1) / GC_TR);
  if (t < 1) t = 1;
  if (t > 4096) t = 4096;
  return (int)t;
}

int fill_geo_job(const tops_geo_job &u, GeoJob &J) {
  if (!u.dem || !u.cpm_dev || !u.status_dev || u.dem_lines <= 0 || u.dem_pixels <= 0)
    return TOPS_E_INVALID;
  if (u.dem_pitch % sizeof(float)) return TOPS_E_INVALID;
  if (u.xmax <= u.xmin || u.ymax <= u.ymin) return TOPS_E_INVALID;
  for (int k = 0; k < 2; k++)
    if (u.ncoef[k] < 2 || u.ncoef[k] > 8 || u.dt[k] == 0.0 || u.range_spacing[k] == 0.0)
      return TOPS_E_INVALID;
  J.dem = u.dem;
  J.dem_pitch = (long)(u.dem_pitch / sizeof(float));
  if (J.dem_pitch < u.dem_pixels) return TOPS_E_INVALID;
  J.lines = u.dem_lines;
  J.pixels = u.dem_pixels;
  J.lat0 = u.lat0;
  J.lon0 = u.lon0;
  J.dlat = u.dlat;
  J.dlon = u.dlon;
  J.nodata = u.nodata;
  J.xmin = u.xmin;
  J.xmax = u.xmax;
  J.ymin = u.ymin;
  J.ymax = u.ymax;
  J.inv_yq = 1.0 / (0.25 * ((double)u.ymax - (double)u.ymin));
  J.inv_xq = 1.0 / (0.25 * ((double)u.xmax - (double)u.xmin));
  for (int k = 0; k < 2; k++) {
    J.dt[k] = u.dt[k];
    J.inv_dt[k] = 1.0 / u.dt[k];
    J.inv_range_spacing[k] = 1.0 / u.range_spacing[k];
    J.first_line_time[k] = u.first_line_time[k];
    J.slr_time[k] = u.slr_time[k];
    J.range_spacing[k] = u.range_spacing[k];
    J.mid_time[k] = u.mid_time[k];
    J.azi_init[k] = u.azi_init[k];
    J.line_offset[k] = u.line_offset[k];
    J.ncoef[k] = u.ncoef[k];
    for (int a = 0; a < 3; a++)
      for (int i = 0; i < 8; i++) J.coef[k][a][i] = u.coef[k][a][i];
  }
  J.cpm = u.cpm_dev;
  J.status = u.status_dev;
  J.blocks = gc_blocks_for(u.dem_lines, u.dem_pixels);
  return TOPS_OK;
}

size_t geocoreg_scratch(const GeoJob *J, int n) {
  size_t blocks = 0;
  for (int i = 0; i < n; i++) blocks += J[i].blocks;
  return blocks * GC_NSUM * sizeof(double);
}

int launch_geocoreg(const GeoJob *jobs, int njobs, bool dem_is_int, void *scratch,
                    size_t scratch_bytes, cudaStream_t st) {
  if (geocoreg_scratch(jobs, njobs) > scratch_bytes || (!scratch && njobs > 0))
    return TOPS_E_INVALID;
  double *part = static_cast<double *>(scratch);
  for (int j0 = 0; j0 < njobs; j0 += GC_MAXJOBS) {
    GcBatch B;
    B.njobs = 0;
    B.dem_is_int = dem_is_int ? 1 : 0;
    int blocks = 0;
    for (int j = j0; j < njobs && j < j0 + GC_MAXJOBS; j++) {
      B.jobs[B.njobs] = jobs[j];
      B.jobs[B.njobs].block_begin = blocks;
      blocks += jobs[j].blocks;
      B.njobs++;
    }
    B.total_blocks = blocks;
    geocoreg_kernel<<<blocks, GC_NT, 0, st>>>(B, part);
    TOPS_CUDA_TRY(cudaGetLastError());
    geocoreg_solve_kernel<<<B.njobs, 64, 0, st>>>(B, part);
    TOPS_CUDA_TRY(cudaGetLastError());
    part += (size_t)blocks * GC_NSUM;
  }
  return TOPS_OK;
}

}  // namespace tops

using namespace tops;

extern "C" size_t tops_geocoreg_scratch_bytes(const tops_geo_job *jobs, int njobs) {
  std::vector<GeoJob> J(njobs > 0 ? njobs : 0);
  for (int i = 0; i < njobs; i++)
    if (fill_geo_job(jobs[i], J[i]) != TOPS_OK) return 0;
  return geocoreg_scratch(J.data(), njobs);
}

extern "C" int tops_geocoreg(const tops_geo_job *jobs, int njobs, void *scratch_dev,
                             size_t scratch_bytes, void *stream) {
  if ((!jobs && njobs > 0) || njobs < 0) return TOPS_E_INVALID;
  std::vector<GeoJob> J(njobs);
  for (int i = 0; i < njobs; i++) {
    int s = fill_geo_job(jobs[i], J[i]);
    if (s != TOPS_OK) return s;
  }
  return launch_geocoreg(J.data(), njobs, false, scratch_dev, scratch_bytes,
                         static_cast<cudaStream_t>(stream));
}

// resample.cu -- TOPS deramp + demodulation + 12-point LUT sinc resampling
// + reramp of slave bursts onto the master grid (sm_100a).
//
// Computes the reference algorithm of DerampDemod_Shared
// (DerampAndResample.cu:117-183) followed by Interpolation_12p
// (DerampAndResample.cu:349-520), GetIndexes (:108-112) and my_polyval /
// normalizeWarp (cuConstants.cuh:53-65):
//   position  y = polyAz(L^, P^) + shift,  x = polyRg(L^, P^)
//   index     L0 = trunc(y), bin = int(frac * 2047 + 0.5)  (same for x)
//   regions   outside the slave box -> 0; within 5/7 samples of its edge ->
//             the nearest sample; interior -> separable 12x12 LUT sinc of the
//             deramped slave d = s exp(i phi), reramped with the LUT-weighted
//             sum of the deramp phase phi.
//
// B200 design (no textures, no phase array in HBM).  A CTA owns a strip of
// RS_TW output columns and sweeps a segment of output rows in groups of RS_GR
// rows; per group:
//   [A] Row statistics from the offset polynomials, not per pixel: along the
//       strip y and x are quadratics in the column, so their range follows
//       from the two ends and the vertex.  A row whose whole strip maps to one
//       (azimuth line, LUT bin) key -- in a TOPS pair nearly every row -- gets
//       one shared azimuth pass.  The same bounds give the slave lines the
//       group needs.  Warp 7, idle in the range pass [D], prepares the next
//       group's keys, ring-row table and azimuth taps during [D], into the
//       second of two per-row tables; the other warps never wait for it.
//   [B] New slave rows are deramped once into a ring of RS_FR rows x RS_FW
//       columns in shared memory: d (complex) and the FP32 residual
//       G = phi - phi_ref of the deramp phase against a reference column.
//   [C] Azimuth pass v(x) = sum_j kAz[j] d(L0-5+j, x) for every ring column,
//       blocked over 4 rows x 2 columns per thread (15 ring loads and 24
//       weight loads feed 96 packed FP32x2 FMAs).  G is exactly quadratic in
//       azimuth time per column, so its azimuth interpolation is
//       M0 G(L0) + g2 P1 + g1 P2 with the LUT row moments -- no taps.
//   [D] Range pass, reramp, store.  A thread owns 2 adjacent output columns
//       for 4 rows.  A column's range key (p0, bin) changes only every ~100
//       rows, so its 12 range weights stay in registers; the 14 v samples of
//       a column pair are 7 16-byte shared loads, and the phase residuals of
//       2 rows are range-interpolated together with packed FMAs.
// The interpolated phase is (1 + sp1) Psi_row + sum_i kRg[i] vg(x_i), where
// Psi_row = sum_j kAz[j] phi_ref(y_j) is FP64 (reduced mod 2 pi) and
// 1 + sp1 = sum kRg: equal to the reference's 144-tap FP64 phase sum in exact
// arithmetic.  Rows or pixels outside these cases (several keys in a row,
// edge and outside pixels, supports beyond the ring) take per-pixel paths
// that compute the same formula.
//
// Precision modes: TOPS_PREC_SPLIT (default) forms G and the reduced phase of
// each ring sample in FP32 from per-column coefficients about the burst's
// centre time, with the FP64 reference-row phase reduced mod 2 pi once per
// row (double-single).  TOPS_PREC_FP64 evaluates every sample's deramp phase
// and its reduction in FP64.  Positions, LUT bins and Psi_row are FP64 in
// both.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"
#include "launch.h"

namespace tops {

constexpr int RS_NT = 256;   // threads per CTA
constexpr int RS_TW = 112;   // output columns per strip
constexpr int RS_GR = 16;    // output rows per group
constexpr int RS_FR = 32;    // ring rows (power of two)
constexpr int RS_FW = 128;   // ring columns
constexpr int RS_SEG = 256;  // output rows per work item
constexpr int RS_MAXJOBS = 32;
constexpr int RS_DP = RS_TW / 2;   // column pairs of the range pass
constexpr int RS_DT = RS_DP * 4;   // range-pass threads (4 row quarters of 4 rows)
static_assert(RS_DT == RS_NT - 32, "warp 7 prepares the next group during the range pass");
static_assert(RS_GR == 16 && RS_FW == 128 && RS_NT == 256 && RS_FR == 32,
              "the thread mappings assume these sizes");

enum : int { REG_OUT = 0, REG_EDGE = 1, REG_IN = 2 };

using RsLut = LutPtrs;

struct RsBatch {
  int njobs;
  int total_items;
  int *counter;            // persistent launch: work-item queue (else null)
  ResampleJob jobs[RS_MAXJOBS];
};

struct RsRows {
  int v[RS_GR];                       // 1: shared azimuth pass valid for the row
  int L0[RS_GR], bL[RS_GR];           // its azimuth line and LUT bin
  float rho[RS_GR], psif[RS_GR];      // row phase Psi reduced mod 2 pi, and as float
};

struct __align__(16) RsShared {
  float2 ring_d[RS_FR][RS_FW];        // deramped slave rows
  float ring_g[RS_FR][RS_FW];         // G = phi - phi_ref of each ring sample
  float2 vd[RS_GR][RS_FW];            // azimuth-interpolated d
  float2 vgp[RS_GR / 2][RS_FW];       // azimuth-interpolated G of rows (2k, 2k+1)
  float4 wpair[RS_GR][6];             // azimuth taps duplicated: (w0,w0,w1,w1), ...
  double ring_phiref[RS_FR];          // FP64 reference-column phase of the ring row
  double ring_ta[RS_FR];              // burst-local azimuth time of the ring row
  float ring_rho[RS_FR];              // ring_phiref reduced mod 2 pi
  float ring_tc[RS_FR];               // ring_ta - tm (FP32, split mode)
  double rowA_az[RS_SEG], rowB_az[RS_SEG], rowA_rg[RS_SEG], rowB_rg[RS_SEG];
  // per-column P^ and c5 P^2 terms; a range-pass thread reads its two
  // columns with one 16-byte load (conflict-free across the warp)
  alignas(16) double col_phat[RS_TW];
  alignas(16) double col_qaz[RS_TW];
  alignas(16) double col_qrg[RS_TW];
  // per-row tables of a group; the range pass of one group reads one copy
  // while warp 7 prepares the other for the next group
  RsRows rows[2];
  float row_M0[RS_GR], row_P1[RS_GR], row_P2[RS_GR];
  int g_lmin, g_lmax;                 // slave lines the group's interior pixels use
  double caz[6], crg[6], shift;
  int xw;                             // absolute slave column of ring column 0
  double ref_a0, ref_a1, ref_a2;      // deramp quadratic of the reference column
  double tm;                          // centre time of the split-mode coefficients
  int next_item;                      // persistent launch: the item just taken
  // per-row key statistics of the whole work item, computed once up front:
  // azimuth line / LUT bin of a row with one key (bin -1: none) and the
  // slave lines its interior pixels use
  int ri_L0[RS_SEG], ri_bL[RS_SEG], ri_lmin[RS_SEG], ri_lmax[RS_SEG];
  // raw slave rows of the next group, copied asynchronously (cp.async)
  // while the current group computes; each thread reads back only the
  // elements it copied
  alignas(16) short2 stage[RS_FR][RS_FW];
  int pf_lo, pf_hi;                   // rows staged for this group
  int nx_lo, nx_hi;                   // rows the next group brings
};

// Asynchronous global -> shared copies of 4 or 8 bytes to a shared-window
// address; src_bytes 0 fills the destination with zeros without reading.
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async_8s(unsigned d, const void *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_4s(unsigned d, const void *src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Deramp + demodulation phase (DerampAndResample.cu:151-158), FP64, as the
// quadratic a2 ta^2 + a1 ta + a0 of the burst-local azimuth time ta:
//   -pi kt (ta - tref)^2 - 2 pi fdc ta.
struct DerampQuad {
  double a0, a1, a2;
};
__device__ __forceinline__ DerampQuad deramp_quad(double kt, double tref, double fdc) {
  DerampQuad q;
  q.a2 = -kPi * kt;
  q.a1 = 2.0 * kPi * kt * tref - 2.0 * kPi * fdc;
  q.a0 = -kPi * kt * tref * tref;
  return q;
}
__device__ __forceinline__ double quad_eval(const DerampQuad &q, double ta) {
  return fma(fma(q.a2, ta, q.a1), ta, q.a0);
}
__device__ __forceinline__ double deramp_phase(double ta, double kt, double tref, double fdc) {
  const double e = ta - tref;
  return -kPi * kt * (e * e) - 2.0 * kPi * fdc * ta;
}

__device__ __forceinline__ float2 cmul_conj_phase(float2 a, float phi) {
  // a * exp(-i phi)
  float s, c;
  __sincosf(reduce_2pi_f(phi), &s, &c);
  return make_float2(a.x * c + a.y * s, a.y * c - a.x * s);
}

// Integer index and LUT bin of a position (GetIndexes, DerampAndResample.cu:
// 108-112): trunc, then int(frac * 2047 + 0.5) without FMA contraction; the
// bin is clamped as the reference's texture fetch clamps.
__device__ __forceinline__ void split_pos(double v, int &i0, int &bin) {
  i0 = __double2int_rz(v);
  const int b = __double2int_rz(__dadd_rn(__dmul_rn(v - (double)i0, (double)kInterval), 0.5));
  bin = min(max(b, 0), kLutBins - 1);
}

__device__ __forceinline__ int region_of(const ResampleJob &J, int l0, int p0) {
  if (l0 > J.sy1 || l0 < J.sy0 || p0 > J.sx1 || p0 < J.sx0) return REG_OUT;
  if (l0 > J.sy1 - 7 || l0 < J.sy0 + 5 || p0 > J.sx1 - 7 || p0 < J.sx0 + 5) return REG_EDGE;
  return REG_IN;
}

// Range [lo, hi] of f(p) = fma(b, p, a + c p^2) -- the per-pixel form -- over
// p in [p0, p1]: the ends and, when inside, the vertex.  Widened by 1e-9 so
// that rounding of the per-pixel evaluation cannot leave it.
__device__ __forceinline__ void quad_span(double a, double b, double c, double p0, double p1,
                                          double &lo, double &hi) {
  const double f0 = fma(b, p0, a + c * p0 * p0);
  const double f1 = fma(b, p1, a + c * p1 * p1);
  lo = fmin(f0, f1);
  hi = fmax(f0, f1);
  // the vertex lies inside only if the slope changes sign over [p0, p1]
  const double s0 = fma(2.0 * c, p0, b), s1 = fma(2.0 * c, p1, b);
  if ((s0 < 0.0) != (s1 < 0.0)) {
    const double pv = -b / (2.0 * c);
    const double fv = fma(b, pv, a + c * pv * pv);
    lo = fmin(lo, fv);
    hi = fmax(hi, fv);
  }
  lo -= 1e-9;
  hi += 1e-9;
}

// ---------------------------------------------------- HBM slow path
// Per-pixel interior resample straight from the CInt16 slave in HBM (used
// only when the support does not fit the ring window).
__device__ float2 interior_from_global(const ResampleJob &J, const RsLut &lut, int L0, int bL,
                                       int P0, int bP) {
  const float *kl = lut.kaz + bL * kTaps;
  const float *kp = lut.krg + bP * kTaps;
  float sre = 0.f, sim = 0.f;
  double ph = 0.0;
  for (int j = 0; j < kTaps; j++) {
    int y = L0 - 5 + j;
    double ta = (double)(y - J.s_first_line) * J.dt;
    float tre = 0.f, tim = 0.f;
    double tph = 0.0;
    for (int i = 0; i < kTaps; i++) {
      int x = P0 - 5 + i;
      short2 s = J.slave[(long)(y - J.sy0) * J.slave_pitch + (x - J.sx0)];
      double phi = deramp_phase(ta, J.kt[x], J.tref[x], J.fdc[x]);
      float sn, cs;
      __sincosf(reduce_2pi(phi), &sn, &cs);
      float dre = (float)s.x * cs - (float)s.y * sn;
      float dim = (float)s.x * sn + (float)s.y * cs;
      tre = fmaf(kp[i], dre, tre);
      tim = fmaf(kp[i], dim, tim);
      tph = fma((double)kp[i], phi, tph);
    }
    sre = fmaf(kl[j], tre, sre);
    sim = fmaf(kl[j], tim, sim);
    ph = fma((double)kl[j], tph, ph);
  }
  float s, c;
  __sincosf(reduce_2pi(ph), &s, &c);
  return make_float2(sre * c + sim * s, sim * c - sre * s);
}

// ---------------------------------------------------- ring per-pixel path
__device__ float2 interior_from_ring(const RsShared &S, const RsLut &lut, const ResampleJob &J,
                                     const DerampQuad &refq, int L0, int bL, int P0, int bP) {
  const float *kl = lut.kaz + bL * kTaps;
  const float *kp = lut.krg + bP * kTaps;
  float kpr[kTaps];
#pragma unroll
  for (int i = 0; i < kTaps; i++) kpr[i] = __ldg(kp + i);
  const int xc = P0 - 5 - S.xw;
  float sre = 0.f, sim = 0.f, sg = 0.f;
  double psi = 0.0;
#pragma unroll 1
  for (int j = 0; j < kTaps; j++) {
    int slot = (L0 - 5 + j) & (RS_FR - 1);
    float w = __ldg(kl + j);
    float tre = 0.f, tim = 0.f, tg = 0.f;
#pragma unroll
    for (int i = 0; i < kTaps; i++) {
      float2 d = S.ring_d[slot][xc + i];
      tre = fmaf(kpr[i], d.x, tre);
      tim = fmaf(kpr[i], d.y, tim);
      tg = fmaf(kpr[i], S.ring_g[slot][xc + i], tg);
    }
    sre = fmaf(w, tre, sre);
    sim = fmaf(w, tim, sim);
    sg = fmaf(w, tg, sg);
    // the reference-column phase of the line, as the ring-row table holds it
    const double phref = quad_eval(refq, (double)(L0 - 5 + j - J.s_first_line) * J.dt);
    psi = fma((double)w, phref, psi);
  }
  float phi = reduce_2pi(psi) + __ldg(lut.sp1 + bP) * (float)psi + sg;
  return cmul_conj_phase(make_float2(sre, sim), phi);
}

// Range weights of one output column, held in registers while its key holds.
struct ColW {
  float4 w[6];   // (w0,w0,w1,w1), (w2,w2,w3,w3), ...
  float sp1;
  int key;       // p0 << 12 | bin of the loaded weights (-1: none)
};

__device__ __forceinline__ void colw_load(ColW &cw, const RsLut &lut, int key) {
  if (cw.key == key) return;
  const int bp = key & 0xfff;
  const float4 *kp4 = lut.krg2 + bp * (kTaps / 2);
#pragma unroll
  for (int q = 0; q < kTaps / 2; q++) cw.w[q] = __ldg(kp4 + q);
  cw.sp1 = __ldg(lut.sp1 + bp);
  cw.key = key;
}

__device__ __forceinline__ float2 wtap(const ColW &cw, int i) {
  const float4 q = cw.w[i >> 1];
  return (i & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
}

// One interior pixel of a row with a shared azimuth pass: 12-tap range pass
// over vd / vg of the row (single column).
__device__ __forceinline__ float2 range_pixel(const RsShared &S, const RsRows &R, const ColW &cw,
                                              int r, int xb) {
  float2 acc = make_float2(0.f, 0.f);
  float sg = 0.f;
  const float *vgrow = reinterpret_cast<const float *>(&S.vgp[r >> 1][0]) + (r & 1);
#pragma unroll
  for (int i = 0; i < kTaps; i++) {
    const float2 w = wtap(cw, i);
    acc = __ffma2_rn(w, S.vd[r][xb + i], acc);
    sg = fmaf(w.x, vgrow[2 * (xb + i)], sg);
  }
  const float phi = R.rho[r] + cw.sp1 * R.psif[r] + sg;
  return cmul_conj_phase(acc, phi);
}

// 12-tap range pass of two adjacent columns over the 14 samples V (the first
// column's taps start at V[odd], the second's at V[odd + 1]).
__device__ __forceinline__ void range_pair(const ColW &c0, const ColW &c1, const float2 (&V)[14],
                                           bool odd, float2 &s0, float2 &s1) {
  s0 = make_float2(0.f, 0.f);
  s1 = s0;
  if (odd) {
#pragma unroll
    for (int i = 0; i < kTaps; i++) {
      s0 = __ffma2_rn(wtap(c0, i), V[i + 1], s0);
      s1 = __ffma2_rn(wtap(c1, i), V[i + 2], s1);
    }
  } else {
#pragma unroll
    for (int i = 0; i < kTaps; i++) {
      s0 = __ffma2_rn(wtap(c0, i), V[i], s0);
      s1 = __ffma2_rn(wtap(c1, i), V[i + 1], s1);
    }
  }
}

__device__ __forceinline__ void load14(const float2 *row, int base, float2 (&V)[14]) {
  const float4 *p = reinterpret_cast<const float4 *>(row + base);
#pragma unroll
  for (int m = 0; m < 7; m++) {
    const float4 t = p[m];
    V[2 * m] = make_float2(t.x, t.y);
    V[2 * m + 1] = make_float2(t.z, t.w);
  }
}

// One work item (strip x segment of one job); all threads of the CTA call it
// with the same item.
template <bool kSplit>
__device__ __forceinline__ void resample_item(RsShared &S, const RsBatch &B, int item) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;

  // ---- locate the work item (job, strip, segment)
  int jb = 0;
  while (jb + 1 < B.njobs && B.jobs[jb + 1].item_begin <= item) jb++;
  const ResampleJob &J = B.jobs[jb];
  const RsLut &lut = J.lut;
  const int local = item - J.item_begin;
  const int strip = local % J.strips;
  const int seg = local / J.strips;
  const int mpix = J.mx1 - J.mx0 + 1;
  const int c0 = strip * RS_TW;
  const int cN = min(RS_TW, mpix - c0);
  const int r_begin = J.row0 + seg * J.seg_rows;
  const int r_end = min(r_begin + J.seg_rows, J.row0 + J.nrows);

  // ---- per work item setup: polynomials, shift, per-row and per-column terms
  if (tid < 12) {
    const double v = J.cpm_dev ? J.cpm_dev[tid] : (tid < 6 ? J.caz[tid] : J.crg[tid - 6]);
    if (tid < 6)
      S.caz[tid] = v;
    else
      S.crg[tid - 6] = v;
  }
  if (tid == 12) {
    double sh = J.az_shift;
    if (J.az_shift_dev) {
      // a device-provided ESD shift above 100 px is invalid and reset to 0,
      // as the reference driver does (Func.cpp:2612-2621)
      sh = *J.az_shift_dev;
      if (!(fabs(sh) <= 100.0)) sh = 0.0;
    }
    S.shift = sh;
  }
  __syncthreads();
  {
    // y = A(row) + B(row) P^ + c5 P^2 (the terms of my_polyval grouped by row)
    const int r = r_begin + tid;
    if (r < r_end) {
      const double L = ((double)(r + J.my0) - J.midL) * J.invL;
      const double *a = S.caz, *g = S.crg;
      S.rowA_az[tid] = a[0] + a[1] * L + a[3] * L * L + S.shift;
      S.rowB_az[tid] = a[2] + a[4] * L;
      S.rowA_rg[tid] = g[0] + g[1] * L + g[3] * L * L;
      S.rowB_rg[tid] = g[2] + g[4] * L;
    }
    if (tid < RS_TW) {
      const double P = ((double)(c0 + min(tid, cN - 1)) - J.midP) * J.invP;
      S.col_phat[tid] = P;
      S.col_qaz[tid] = S.caz[5] * P * P;
      S.col_qrg[tid] = S.crg[5] * P * P;
    }
  }
  if (tid == 0) {
    // range position at the segment corners and edge midpoints -> ring window
    double pmin = 1e300, pmax = -1e300;
    for (int a = 0; a < 3; a++) {
      int rr = (a == 0) ? r_begin : (a == 1 ? (r_begin + r_end - 1) / 2 : r_end - 1);
      double L = ((double)(rr + J.my0) - J.midL) * J.invL;
      for (int b = 0; b < 3; b++) {
        int cc = (b == 0) ? c0 : (b == 1 ? c0 + (cN - 1) / 2 : c0 + cN - 1);
        double P = ((double)cc - J.midP) * J.invP;
        const double *c = S.crg;
        double x = c[0] + c[1] * L + c[2] * P + c[3] * L * L + c[4] * L * P + c[5] * P * P;
        pmin = fmin(pmin, x);
        pmax = fmax(pmax, x);
      }
    }
    // The range pass reads ring columns [p0 - 6, p0 + 8]: the window starts
    // at the leftmost such column, one column lower when needed for an even
    // offset from the box edge (8-byte pair loads).  A strip spanning up to
    // RS_FW - 16 samples then fits; wider spans fall back per pixel.
    const int lo = (int)floor(pmin) - 6;
    const int xw = lo - ((lo - J.sx0) & 1);
    S.xw = xw;
    int xr = min(max(xw + RS_FW / 2, J.sx0), J.sx1);
    const DerampQuad q = deramp_quad(J.kt[xr], J.tref[xr], J.fdc[xr]);
    S.ref_a0 = q.a0;
    S.ref_a1 = q.a1;
    S.ref_a2 = q.a2;
    S.tm = 0.5 * (double)(J.sy0 + J.sy1 - 2 * J.s_first_line) * J.dt;
    S.nx_lo = 1;   // nothing staged for the first group
    S.nx_hi = 0;
  }
  __syncthreads();

  // ---- per-row key statistics of the whole item (one thread per row):
  // along the strip y and x are quadratics in the column, so their ranges
  // follow from the ends and the vertex.  A row whose strip maps to one
  // (azimuth line, LUT bin) key, whose azimuth support is interior and whose
  // range support fits the ring window gets the shared azimuth pass.
  if (tid < r_end - r_begin) {
    const int ri = tid;
    const double p0 = S.col_phat[0], p1 = S.col_phat[cN - 1];
    double ylo, yhi, xlo, xhi;
    quad_span(S.rowA_az[ri], S.rowB_az[ri], S.caz[5], p0, p1, ylo, yhi);
    quad_span(S.rowA_rg[ri], S.rowB_rg[ri], S.crg[5], p0, p1, xlo, xhi);
    int l0lo, blo, l0hi, bhi, x0lo, xblo, x0hi, xbhi;
    split_pos(ylo, l0lo, blo);
    split_pos(yhi, l0hi, bhi);
    split_pos(xlo, x0lo, xblo);
    split_pos(xhi, x0hi, xbhi);
    const bool az_any = !(l0hi < J.sy0 + 5 || l0lo > J.sy1 - 7);
    const bool rg_any = !(x0hi < J.sx0 + 5 || x0lo > J.sx1 - 7);
    int lmin = INT32_MAX, lmax = INT32_MIN;
    if (az_any && rg_any) {
      lmin = max(l0lo, J.sy0 + 5);
      lmax = min(l0hi, J.sy1 - 7);
    }
    const bool uniform = (l0lo == l0hi) && (blo == bhi);
    const bool az_in = l0lo >= J.sy0 + 5 && l0hi <= J.sy1 - 7;
    // the range pass reads ring columns [p0 - 6, p0 + 8] of its pixels
    const bool win = (x0lo - 6 - S.xw >= 0) && (x0hi + 8 - S.xw < RS_FW);
    S.ri_L0[ri] = l0lo;
    S.ri_bL[ri] = (uniform && az_in && rg_any && win) ? blo : -1;
    S.ri_lmin[ri] = lmin;
    S.ri_lmax[ri] = lmax;
  }

  // ---- per-thread constants of the ring / azimuth-pass column pair
  const int xr0 = 2 * (tid & 63);            // ring columns xr0, xr0 + 1
  const int xa0 = S.xw + xr0;                // absolute slave columns xa0, xa0 + 1
  const bool xin0 = xa0 >= J.sx0 && xa0 <= J.sx1;
  const bool xin1 = xa0 + 1 >= J.sx0 && xa0 + 1 <= J.sx1;
  const bool pair8 = xin0 && xin1 && J.slave_al8;   // one 8-byte copy per staged row
  const DerampQuad refq = {S.ref_a0, S.ref_a1, S.ref_a2};
  const double tm = S.tm;
  DerampQuad cq0 = refq, cq1 = refq;
  if (xin0) cq0 = deramp_quad(J.kt[xa0], J.tref[xa0], J.fdc[xa0]);
  if (xin1) cq1 = deramp_quad(J.kt[xa0 + 1], J.tref[xa0 + 1], J.fdc[xa0 + 1]);
  // G = phi - phi_ref about tm: g2 tc^2 + g1 tc + g0 (tc = ta - tm)
  float g2c0, g1c0, g0c0, g2c1, g1c1, g0c1;
  {
    const double d2 = cq0.a2 - refq.a2, d1 = cq0.a1 - refq.a1, d0 = cq0.a0 - refq.a0;
    g2c0 = (float)d2;
    g1c0 = (float)(2.0 * d2 * tm + d1);
    g0c0 = (float)((d2 * tm + d1) * tm + d0);
    const double e2 = cq1.a2 - refq.a2, e1 = cq1.a1 - refq.a1, e0 = cq1.a0 - refq.a0;
    g2c1 = (float)e2;
    g1c1 = (float)(2.0 * e2 * tm + e1);
    g0c1 = (float)((e2 * tm + e1) * tm + e0);
  }

  // ---- per-thread constants of the range pass (2 columns x 4 rows)
  const int dcp = tid % RS_DP, drq = tid / RS_DP;
  const bool dthread = tid < RS_DT;
  const int dc = 2 * dcp;                    // strip-local columns dc, dc + 1
  const bool dval0 = dthread && dc < cN, dval1 = dthread && dc + 1 < cN;
  ColW cw0, cw1;   // range weights of the two columns, kept across groups
  cw0.key = -1;
  cw1.key = -1;
  const bool out16 = J.out_al16 != 0;

  int loaded_lo = INT32_MIN, loaded_hi = INT32_MIN;  // valid ring rows (uniform)
  // ---- [A] + row setup of the group starting at row rgp into row table nb,
  // run by warp 7 (idle in the range pass) one group ahead: the group's row
  // keys, the ring-row table of the slave lines it brings, the rows the group
  // after it brings (staged while it computes), and per row the azimuth taps,
  // their moments and the row phase.  Lanes 0..15 take the rows of group
  // rgp, lanes 16..31 those of the group after it.
  auto prep_group = [&](int rgp, int nb) {
    RsRows &Q = S.rows[nb];
    {
      const int half = lane >> 4, r = lane & 15;
      const int rgx = rgp + half * RS_GR;
      int v = 0, lmin = INT32_MAX, lmax = INT32_MIN, L0 = 0, bL = 0;
      if (rgx + r < r_end) {
        const int ri = rgx - r_begin + r;
        L0 = S.ri_L0[ri];
        bL = S.ri_bL[ri];
        lmin = S.ri_lmin[ri];
        lmax = S.ri_lmax[ri];
        v = bL >= 0;
      }
      int gmin = lmin, gmax = lmax;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {   // within each half
        gmin = min(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
        gmax = max(gmax, __shfl_xor_sync(0xffffffffu, gmax, o));
      }
      const int cmin = __shfl_sync(0xffffffffu, gmin, 0);
      const int cmax = __shfl_sync(0xffffffffu, gmax, 0);
      const int nmin = __shfl_sync(0xffffffffu, gmin, 16);
      const int nmax = __shfl_sync(0xffffffffu, gmax, 16);
      const bool cok = cmin <= cmax && (cmax - cmin + 12 <= RS_FR);
      const bool nok = rgp + RS_GR < r_end && nmin <= nmax && (nmax - nmin + 12 <= RS_FR);
      if (half == 0) {
        Q.v[r] = v && cok;
        Q.L0[r] = L0;
        Q.bL[r] = max(bL, 0);
      }
      if (lane == 0) {
        S.g_lmin = cok ? cmin : 1;
        S.g_lmax = cok ? cmax : 0;
        S.pf_lo = S.nx_lo;   // the rows staged for this group
        S.pf_hi = S.nx_hi;
      }
      // ring-row table of the rows this group brings (at most RS_FR rows),
      // and the ring state after it
      int ll = loaded_lo, lh = loaded_hi;
      if (cok) {
        const int need_lo = cmin - 5, need_hi = cmax + 6;
        const bool cont = need_lo >= ll && need_lo <= lh + 1;
        const int new_lo = cont ? lh + 1 : need_lo;
        const int y = new_lo + lane;
        if (y <= need_hi) {
          const int slot = y & (RS_FR - 1);
          const double ta = (double)(y - J.s_first_line) * J.dt;
          const double phref = quad_eval(refq, ta);
          S.ring_phiref[slot] = phref;
          S.ring_ta[slot] = ta;
          S.ring_rho[slot] = reduce_2pi(phref);
          S.ring_tc[slot] = (float)(ta - tm);
        }
        if (!cont) ll = need_lo;
        lh = max(lh, need_hi);
        ll = max(ll, lh - RS_FR + 1);
      }
      if (lane == 0) {
        int lo = 1, hi = 0;
        if (nok) {
          const int need_lo = nmin - 5, need_hi = nmax + 6;
          const bool cont = need_lo >= ll && need_lo <= lh + 1;
          lo = cont ? lh + 1 : need_lo;
          hi = need_hi;
        }
        S.nx_lo = lo;
        S.nx_hi = hi;
      }
    }
    __syncwarp();
    // azimuth taps (w, w) pairs, their moments M0..M2 and the row phase
    // Psi = sum_j kAz[j] phi_ref(L0 - 5 + j): 8 lanes per row, 4 rows per
    // pass; lane j < 6 takes taps 2j, 2j+1
#pragma unroll 1
    for (int r = lane >> 3; r < RS_GR; r += 4) {
      const int j = lane & 7;
      const bool rv = Q.v[r] != 0;
      float m0 = 0.f, m1 = 0.f, m2 = 0.f;
      double psi = 0.0;
      if (rv && j < kTaps / 2) {
        const int L0 = Q.L0[r];
        const float *kl = lut.kaz + Q.bL[r] * kTaps + 2 * j;
        const float w0 = __ldg(kl), w1 = __ldg(kl + 1);
        S.wpair[r][j] = make_float4(w0, w0, w1, w1);
        const float u0 = (float)(2 * j - 5), u1 = (float)(2 * j - 4);
        m0 = w0 + w1;
        m1 = fmaf(w0, u0, w1 * u1);
        m2 = fmaf(w0, u0 * u0, w1 * (u1 * u1));
        psi = fma((double)w0, S.ring_phiref[(L0 - 5 + 2 * j) & (RS_FR - 1)],
                  (double)w1 * S.ring_phiref[(L0 - 4 + 2 * j) & (RS_FR - 1)]);
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        m0 += __shfl_xor_sync(0xffffffffu, m0, o);
        m1 += __shfl_xor_sync(0xffffffffu, m1, o);
        m2 += __shfl_xor_sync(0xffffffffu, m2, o);
        psi += __shfl_xor_sync(0xffffffffu, psi, o);
      }
      if (rv && j == 0) {
        const double tc = (double)(Q.L0[r] - J.s_first_line) * J.dt - tm;
        S.row_M0[r] = m0;
        S.row_P1[r] = (float)(2.0 * tc * J.dt * m1 + J.dt * J.dt * m2);
        S.row_P2[r] = (float)(J.dt * m1);
        Q.rho[r] = reduce_2pi(psi);
        Q.psif[r] = (float)psi;
      }
    }
  };
  __syncthreads();
  if (tid >= RS_DT) prep_group(r_begin, 0);
  __syncthreads();

  int buf = 0;   // row table of the current group
  for (int rg = r_begin; rg < r_end; rg += RS_GR, buf ^= 1) {
    const int gr = min(RS_GR, r_end - rg);
    const RsRows &R = S.rows[buf];
    // ---- [B] ring loads of the new slave rows (2 columns per thread)
    const int glmin = S.g_lmin, glmax = S.g_lmax;
    const bool ring_ok = glmin <= glmax;
    // Raw slave rows [lo, hi] (at most RS_FR) into the staging rows: this
    // thread copies its column pair of rows lo + rp + 4u to stage[4u + rp];
    // zeros outside the slave box.  The job fields are read once per call;
    // the source offset and the destination step by 4 rows per copy.
    const int rp = tid >> 6;   // row phase
    auto stage_rows = [&](int lo, int hi) {
      hi = min(hi, lo + RS_FR - 1);
      int y = lo + rp;
      if (y <= hi) {
        const short2 *const sl = J.slave;
        const long pitch = J.slave_pitch;
        const int sy0 = J.sy0;
        const unsigned rows_in = (unsigned)(J.sy1 - J.sy0);
        long off = (long)(y - sy0) * pitch + (xa0 - J.sx0);
        unsigned dst = smem_u32(&S.stage[rp][xr0]);
        constexpr unsigned kStep = 4u * RS_FW * sizeof(short2);
        if (pair8) {
#pragma unroll 4
          for (; y <= hi; y += 4, off += 4 * pitch, dst += kStep) {
            const bool yin = (unsigned)(y - sy0) <= rows_in;
            cp_async_8s(dst, sl + (yin ? off : 0), yin ? 8 : 0);
          }
        } else {
#pragma unroll 1
          for (; y <= hi; y += 4, off += 4 * pitch, dst += kStep) {
            const bool yin = (unsigned)(y - sy0) <= rows_in;
            const bool i0 = yin && xin0, i1 = yin && xin1;
            cp_async_4s(dst, sl + (i0 ? off : 0), i0 ? 4 : 0);
            cp_async_4s(dst + 4, sl + (i1 ? off + 1 : 0), i1 ? 4 : 0);
          }
        }
      }
      cp_async_commit();
    };
    // this thread's copies for the group (staged during the previous one)
    cp_async_wait_all();
    if (ring_ok) {
      const int need_lo = glmin - 5, need_hi = glmax + 6;
      const bool cont = need_lo >= loaded_lo && need_lo <= loaded_hi + 1;
      const int new_lo = cont ? loaded_hi + 1 : need_lo;
      if (S.pf_lo != new_lo || S.pf_hi != need_hi) {
        // not staged (first group of the item): copy now and wait
        stage_rows(new_lo, need_hi);
        cp_async_wait_all();
      }
      // deramp of the new rows (column pair of this thread) into the ring
      const int sy0 = J.sy0;
      const unsigned rows_in = (unsigned)(J.sy1 - J.sy0);
      const int last = min(need_hi, new_lo + RS_FR - 1);
#pragma unroll 2
      for (int y = new_lo + rp, u4 = rp; y <= last; y += 4, u4 += 4) {
        const int slot = y & (RS_FR - 1);
        const short4 ab = *reinterpret_cast<const short4 *>(&S.stage[u4][xr0]);
        const short2 a = make_short2(ab.x, ab.y), b = make_short2(ab.z, ab.w);
        float2 d0 = make_float2(0.f, 0.f), d1 = d0;
        float G0 = 0.f, G1 = 0.f;
        if ((unsigned)(y - sy0) <= rows_in) {
          float r0, r1;
          if (kSplit) {
            const float tc = S.ring_tc[slot], rho = S.ring_rho[slot];
            G0 = fmaf(fmaf(g2c0, tc, g1c0), tc, g0c0);
            G1 = fmaf(fmaf(g2c1, tc, g1c1), tc, g0c1);
            r0 = reduce_2pi_f(rho + G0);
            r1 = reduce_2pi_f(rho + G1);
          } else {
            const double ta = S.ring_ta[slot], phref = S.ring_phiref[slot];
            const double p0 = quad_eval(cq0, ta), p1 = quad_eval(cq1, ta);
            G0 = (float)(p0 - phref);
            G1 = (float)(p1 - phref);
            r0 = reduce_2pi(p0);
            r1 = reduce_2pi(p1);
          }
          float sn, cs;
          if (xin0) {
            __sincosf(r0, &sn, &cs);
            d0.x = (float)a.x * cs - (float)a.y * sn;
            d0.y = (float)a.x * sn + (float)a.y * cs;
          } else {
            G0 = 0.f;
          }
          if (xin1) {
            __sincosf(r1, &sn, &cs);
            d1.x = (float)b.x * cs - (float)b.y * sn;
            d1.y = (float)b.x * sn + (float)b.y * cs;
          } else {
            G1 = 0.f;
          }
        }
        *reinterpret_cast<float4 *>(&S.ring_d[slot][xr0]) = make_float4(d0.x, d0.y, d1.x, d1.y);
        *reinterpret_cast<float2 *>(&S.ring_g[slot][xr0]) = make_float2(G0, G1);
      }
      if (!cont) loaded_lo = need_lo;
      loaded_hi = max(loaded_hi, need_hi);
      loaded_lo = max(loaded_lo, loaded_hi - RS_FR + 1);
    }
    // stage the next group's new rows (the staged values above are consumed:
    // their ring stores are issued); they land while this group computes
    if (S.nx_lo <= S.nx_hi) stage_rows(S.nx_lo, S.nx_hi);
    __syncthreads();

    // ---- [C] shared azimuth pass: 2 ring columns x 4 rows per thread
    {
      const int q = tid >> 6;      // rows 4q .. 4q+3
      const int r0 = 4 * q;
      if (r0 < gr) {
        const int L00 = R.L0[r0];
        bool blk = r0 + 4 <= gr;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int r = min(r0 + k, RS_GR - 1);
          blk = blk && R.v[r] && R.L0[r] == L00 + k;
        }
        if (blk) {
          float2 a0[4], a1[4];
#pragma unroll
          for (int k = 0; k < 4; k++) a0[k] = a1[k] = make_float2(0.f, 0.f);
#pragma unroll
          for (int jj = 0; jj < kTaps + 3; jj++) {
            const float4 dd =
                *reinterpret_cast<const float4 *>(&S.ring_d[(L00 - 5 + jj) & (RS_FR - 1)][xr0]);
            const float2 e0 = make_float2(dd.x, dd.y), e1 = make_float2(dd.z, dd.w);
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const int j = jj - k;
              if (j >= 0 && j < kTaps) {
                const float4 wp = S.wpair[r0 + k][j >> 1];
                const float2 w = (j & 1) ? make_float2(wp.z, wp.w) : make_float2(wp.x, wp.y);
                a0[k] = __ffma2_rn(w, e0, a0[k]);
                a1[k] = __ffma2_rn(w, e1, a1[k]);
              }
            }
          }
          float vg0[4], vg1[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const int r = r0 + k;
            const float2 gc =
                *reinterpret_cast<const float2 *>(&S.ring_g[(L00 + k) & (RS_FR - 1)][xr0]);
            const float M0 = S.row_M0[r], P1 = S.row_P1[r], P2 = S.row_P2[r];
            vg0[k] = fmaf(M0, gc.x, fmaf(g2c0, P1, g1c0 * P2));
            vg1[k] = fmaf(M0, gc.y, fmaf(g2c1, P1, g1c1 * P2));
            *reinterpret_cast<float4 *>(&S.vd[r][xr0]) =
                make_float4(a0[k].x, a0[k].y, a1[k].x, a1[k].y);
          }
          *reinterpret_cast<float4 *>(&S.vgp[2 * q][xr0]) =
              make_float4(vg0[0], vg0[1], vg1[0], vg1[1]);
          *reinterpret_cast<float4 *>(&S.vgp[2 * q + 1][xr0]) =
              make_float4(vg0[2], vg0[3], vg1[2], vg1[3]);
        } else {
#pragma unroll 1
          for (int k = 0; k < 4 && r0 + k < gr; k++) {
            const int r = r0 + k;
            if (!R.v[r]) continue;
            const int L0 = R.L0[r];
            float2 a0 = make_float2(0.f, 0.f), a1 = a0;
#pragma unroll
            for (int j = 0; j < kTaps; j++) {
              const float4 wp = S.wpair[r][j >> 1];
              const float2 w = (j & 1) ? make_float2(wp.z, wp.w) : make_float2(wp.x, wp.y);
              const float4 dd =
                  *reinterpret_cast<const float4 *>(&S.ring_d[(L0 - 5 + j) & (RS_FR - 1)][xr0]);
              a0 = __ffma2_rn(w, make_float2(dd.x, dd.y), a0);
              a1 = __ffma2_rn(w, make_float2(dd.z, dd.w), a1);
            }
            const float2 gc =
                *reinterpret_cast<const float2 *>(&S.ring_g[L0 & (RS_FR - 1)][xr0]);
            const float M0 = S.row_M0[r], P1 = S.row_P1[r], P2 = S.row_P2[r];
            float *vg = reinterpret_cast<float *>(&S.vgp[r >> 1][xr0]) + (r & 1);
            vg[0] = fmaf(M0, gc.x, fmaf(g2c0, P1, g1c0 * P2));
            vg[2] = fmaf(M0, gc.y, fmaf(g2c1, P1, g1c1 * P2));
            *reinterpret_cast<float4 *>(&S.vd[r][xr0]) = make_float4(a0.x, a0.y, a1.x, a1.y);
          }
        }
      }
    }
    __syncthreads();

    // ---- [D] range pass, reramp, store: 2 columns x 4 rows per thread
    if (dthread) {
#pragma unroll 2
      for (int h = 0; h < 2; h++) {
        const int ra = 4 * drq + 2 * h;     // rows ra, ra + 1 (ra even)
        if (ra >= gr) break;
        const bool two = ra + 1 < gr;
        // range keys of the 2 x 2 pixels
        // (entries beyond cN - 1 hold the last column's terms)
        int p0v[2][2], bpv[2][2];
        const double2 cph = *reinterpret_cast<const double2 *>(&S.col_phat[dc]);
        const double2 cq = *reinterpret_cast<const double2 *>(&S.col_qrg[dc]);
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const int ri = rg - r_begin + ra + k;
          const double A = S.rowA_rg[ri], Bc = S.rowB_rg[ri];
          split_pos(fma(Bc, cph.x, A + cq.x), p0v[k][0], bpv[k][0]);
          split_pos(fma(Bc, cph.y, A + cq.y), p0v[k][1], bpv[k][1]);
        }
        // Fast pair: both rows with a shared azimuth pass, each row's two
        // pixels interior, adjacent (p0 steps by one) and inside the ring
        // window.  A column's range key may change between the two rows
        // (about once per 100 rows); its weights are then reloaded for the
        // second row and its phase residual is interpolated per row.
        bool fast = two && dval1 && out16 && R.v[ra] && R.v[ra + 1];
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const int xbk = p0v[k][0] - 5 - S.xw;
          fast = fast && p0v[k][1] == p0v[k][0] + 1 && p0v[k][0] >= J.sx0 + 5 &&
                 p0v[k][1] <= J.sx1 - 7 && xbk >= 1 && xbk + 13 < RS_FW;
        }
        if (fast) {
          const int key00 = (p0v[0][0] << 12) | bpv[0][0], key01 = (p0v[0][1] << 12) | bpv[0][1];
          const int key10 = (p0v[1][0] << 12) | bpv[1][0], key11 = (p0v[1][1] << 12) | bpv[1][1];
          const bool same = key00 == key10 && key01 == key11;
          float2 acc[2][2];
          float sg[2][2];
#pragma unroll
          for (int k = 0; k < 2; k++) {
            colw_load(cw0, lut, k ? key10 : key00);
            colw_load(cw1, lut, k ? key11 : key01);
            const int xb = p0v[k][0] - 5 - S.xw;   // ring column of the first tap
            const int base = xb & ~1;              // 16-byte aligned start
            const bool odd = (xb & 1) != 0;
            {
              float2 V[14];
              load14(&S.vd[ra + k][0], base, V);
              range_pair(cw0, cw1, V, odd, acc[k][0], acc[k][1]);
            }
            // phase residuals from the (row ra, row ra+1) pairs: both rows
            // at once when the keys agree, else each row with its weights
            if (k == 0 || !same) {
              float2 Gp[14], g0, g1;
              load14(&S.vgp[ra >> 1][0], base, Gp);
              range_pair(cw0, cw1, Gp, odd, g0, g1);
              if (k == 0) {
                sg[0][0] = g0.x;
                sg[0][1] = g1.x;
                sg[1][0] = g0.y;
                sg[1][1] = g1.y;
              } else {
                sg[1][0] = g0.y;
                sg[1][1] = g1.y;
              }
            }
          }
#pragma unroll
          for (int k = 0; k < 2; k++) {
            const int r = ra + k;
            const float rho = R.rho[r], psif = R.psif[r];
            // sp1 of the column's row-k bin (cw holds row 1's weights now)
            const float sp0 = (k == 0 && !same) ? __ldg(lut.sp1 + bpv[0][0]) : cw0.sp1;
            const float sp1 = (k == 0 && !same) ? __ldg(lut.sp1 + bpv[0][1]) : cw1.sp1;
            const float2 o0 = cmul_conj_phase(acc[k][0], rho + sp0 * psif + sg[k][0]);
            const float2 o1 = cmul_conj_phase(acc[k][1], rho + sp1 * psif + sg[k][1]);
            float2 *orow = J.out + (long)(rg + r - J.row0) * J.out_pitch + c0 + dc;
            *reinterpret_cast<float4 *>(orow) = make_float4(o0.x, o0.y, o1.x, o1.y);
          }
        } else {
          // per pixel: any region, any key
#pragma unroll 1
          for (int k = 0; k < 2; k++) {
            const int r = ra + k;
            if (r >= gr) break;
            const int ri = rg - r_begin + r;
            const bool rv = R.v[r];
#pragma unroll 1
            for (int c = 0; c < 2; c++) {
              if (!(c ? dval1 : dval0)) continue;
              const int col = dc + c;
              int l0, bl;
              if (rv) {
                l0 = R.L0[r];
                bl = R.bL[r];
              } else {
                const double y =
                    fma(S.rowB_az[ri], S.col_phat[col], S.rowA_az[ri] + S.col_qaz[col]);
                split_pos(y, l0, bl);
              }
              // (selects, not a dynamic index: keeps p0v / bpv in registers)
              const int p0 = k ? (c ? p0v[1][1] : p0v[1][0]) : (c ? p0v[0][1] : p0v[0][0]);
              const int bp = k ? (c ? bpv[1][1] : bpv[1][0]) : (c ? bpv[0][1] : bpv[0][0]);
              const int reg = region_of(J, l0, p0);
              float2 res = make_float2(0.f, 0.f);
              if (reg == REG_EDGE) {
                const short2 sv = J.slave[(long)(l0 - J.sy0) * J.slave_pitch + (p0 - J.sx0)];
                res = make_float2((float)sv.x, (float)sv.y);
              } else if (reg == REG_IN) {
                const int xbp = p0 - 5 - S.xw;
                const bool in_win = xbp >= 0 && xbp + kTaps <= RS_FW;
                if (rv && in_win) {
                  if (c) {
                    colw_load(cw1, lut, (p0 << 12) | bp);
                    res = range_pixel(S, R, cw1, r, xbp);
                  } else {
                    colw_load(cw0, lut, (p0 << 12) | bp);
                    res = range_pixel(S, R, cw0, r, xbp);
                  }
                } else if (ring_ok && in_win && l0 - 5 >= loaded_lo && l0 + 6 <= loaded_hi) {
                  res = interior_from_ring(S, lut, J, refq, l0, bl, p0, bp);
                } else {
                  res = interior_from_global(J, lut, l0, bl, p0, bp);
                }
              }
              J.out[(long)(rg + r - J.row0) * J.out_pitch + c0 + col] = res;
            }
          }
        }
      }
    } else if (rg + RS_GR < r_end) {
      prep_group(rg + RS_GR, buf ^ 1);
    }
    __syncthreads();
  }
}

template <bool kSplit>
__global__ void __launch_bounds__(RS_NT, 2)
    resample_kernel(const __grid_constant__ RsBatch B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsShared &S = *reinterpret_cast<RsShared *>(smem_raw);
  // one work item per CTA, or (persistent) items from the queue until it
  // is empty; a single call site keeps one inlined copy of the item code
  int item = blockIdx.x;
  if (B.counter) {
    if (threadIdx.x == 0) S.next_item = atomicAdd(B.counter, 1);
    __syncthreads();
    item = S.next_item;
    __syncthreads();
  }
  while (item < B.total_items) {
    resample_item<kSplit>(S, B, item);
    if (!B.counter) break;
    if (threadIdx.x == 0) S.next_item = atomicAdd(B.counter, 1);
    __syncthreads();
    item = S.next_item;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host
struct LutDev {
  float *kaz = nullptr, *krg = nullptr, *sp1 = nullptr;
  float4 *krg2 = nullptr;
};

}  // namespace tops

struct tops_lut_dev {
  tops::LutDev d;
};

using namespace tops;

extern "C" int tops_lut_create(const float *kaz, const float *krg, tops_lut_dev **out) {
  if (!kaz || !krg || !out) return TOPS_E_INVALID;
  tops_lut_dev *L = new tops_lut_dev();
  std::vector<float> sp1(kLutBins), krg2((size_t)kLutBins * kTaps * 2);
  for (int b = 0; b < kLutBins; b++) {
    double s = 0.0;
    for (int i = 0; i < kTaps; i++) {
      s += (double)krg[b * kTaps + i];
      krg2[(size_t)b * kTaps * 2 + 2 * i] = krg[b * kTaps + i];
      krg2[(size_t)b * kTaps * 2 + 2 * i + 1] = krg[b * kTaps + i];
    }
    sp1[b] = (float)(s - 1.0);
  }
  size_t nb = sizeof(float) * kLutBins * kTaps;
  cudaError_t e = cudaMalloc(&L->d.kaz, nb);
  if (e == cudaSuccess) e = cudaMalloc(&L->d.krg, nb);
  if (e == cudaSuccess) e = cudaMalloc(&L->d.krg2, 2 * nb);
  if (e == cudaSuccess) e = cudaMalloc(&L->d.sp1, sizeof(float) * kLutBins);
  if (e == cudaSuccess) e = cudaMemcpy(L->d.kaz, kaz, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(L->d.krg, krg, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(L->d.krg2, krg2.data(), 2 * nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(L->d.sp1, sp1.data(), sizeof(float) * kLutBins, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    cudaFree(L->d.kaz);
    cudaFree(L->d.krg);
    cudaFree(L->d.krg2);
    cudaFree(L->d.sp1);
    delete L;
    return e == cudaErrorMemoryAllocation ? TOPS_E_NOMEM : TOPS_E_CUDA;
  }
  *out = L;
  return TOPS_OK;
}

extern "C" int tops_lut_destroy(tops_lut_dev *L) {
  if (!L) return TOPS_OK;
  cudaFree(L->d.kaz);
  cudaFree(L->d.krg);
  cudaFree(L->d.krg2);
  cudaFree(L->d.sp1);
  delete L;
  return TOPS_OK;
}

namespace tops {

static int check_box(const int b[4]) { return b[1] >= b[0] && b[3] >= b[2]; }

int fill_resample_job(const tops_resample_job &u, ResampleJob &J) {
  if (!u.slave || !u.out || !u.kt || !u.tref || !u.fdc) return TOPS_E_INVALID;
  if (!check_box(u.mbox) || !check_box(u.sbox)) return TOPS_E_INVALID;
  if ((u.slave_pitch % sizeof(short2)) || (u.out_pitch % sizeof(float2))) return TOPS_E_INVALID;
  const int mlines = u.mbox[3] - u.mbox[2] + 1;
  J.slave = static_cast<const short2 *>(u.slave);
  J.slave_pitch = (long)(u.slave_pitch / sizeof(short2));
  J.out = static_cast<float2 *>(u.out);
  J.out_pitch = (long)(u.out_pitch / sizeof(float2));
  if (J.slave_pitch < u.sbox[1] - u.sbox[0] + 1 || J.out_pitch < u.mbox[1] - u.mbox[0] + 1)
    return TOPS_E_INVALID;
  // vector access needs aligned bases and pitches: 8-byte slave pairs and
  // 16-byte output pairs (scalar access otherwise)
  J.slave_al8 = ((reinterpret_cast<uintptr_t>(u.slave) & 7) == 0) && (u.slave_pitch % 8 == 0);
  J.out_al16 = ((reinterpret_cast<uintptr_t>(u.out) & 15) == 0) && (u.out_pitch % 16 == 0);
  J.kt = u.kt;
  J.tref = u.tref;
  J.fdc = u.fdc;
  J.mx0 = u.mbox[0];
  J.mx1 = u.mbox[1];
  J.my0 = u.mbox[2];
  J.my1 = u.mbox[3];
  J.sx0 = u.sbox[0];
  J.sx1 = u.sbox[1];
  J.sy0 = u.sbox[2];
  J.sy1 = u.sbox[3];
  for (int i = 0; i < 6; i++) {
    J.caz[i] = u.cpm_az[i];
    J.crg[i] = u.cpm_rg[i];
  }
  J.az_shift = u.az_shift;
  J.az_shift_dev = u.az_shift_dev;
  J.cpm_dev = u.cpm_dev;
  J.s_first_line = u.s_first_line;
  J.dt = u.dt;
  J.row0 = u.out_rows < 0 ? 0 : u.out_row0;
  J.nrows = u.out_rows < 0 ? mlines : u.out_rows;
  if (J.row0 < 0 || J.nrows < 0 || J.row0 + J.nrows > mlines) return TOPS_E_INVALID;
  // normalizeWarp(v, lo, hi) = (v - 0.5*(lo+hi)) / (0.25*(hi-lo))
  J.midP = 0.5 * ((double)u.mbox[0] + (double)u.mbox[1]);
  J.invP = 1.0 / (0.25 * ((double)u.mbox[1] - (double)u.mbox[0]));
  J.midL = 0.5 * ((double)u.mbox[2] + (double)u.mbox[3]);
  J.invL = 1.0 / (0.25 * ((double)u.mbox[3] - (double)u.mbox[2]));
  const int mpix = u.mbox[1] - u.mbox[0] + 1;
  J.strips = (mpix + RS_TW - 1) / RS_TW;
  J.seg_rows = RS_SEG;
  J.segs = (J.nrows + RS_SEG - 1) / RS_SEG;
  return TOPS_OK;
}

template <bool kSplit>
static int launch_resample_t(const ResampleJob *jobs, int njobs, const TileCfg &cfg,
                             cudaStream_t st) {
  // the shared-memory opt-in is a per-device function attribute; the
  // persistent grid is the number of CTAs resident at once
  static PerDeviceOnce setup;
  int dev = 0, resident = 0;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  const int s0 = once_per_device(
      setup, dev,
      [&](int &v) -> int {
        TOPS_CUDA_TRY(cudaFuncSetAttribute(resample_kernel<kSplit>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sizeof(RsShared)));
        int per_sm = 0, sms = 0;
        TOPS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, resample_kernel<kSplit>, RS_NT, sizeof(RsShared)));
        TOPS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        v = per_sm * sms;
        return TOPS_OK;
      },
      &resident);
  if (s0 != TOPS_OK) return s0;
  if (cfg.seg_rows < 0 || cfg.seg_rows > RS_SEG || (cfg.seg_rows && cfg.seg_rows < RS_GR))
    return TOPS_E_INVALID;
  for (int j0 = 0, k = 0; j0 < njobs; j0 += RS_MAXJOBS, k++) {
    RsBatch B;
    B.njobs = 0;
    B.counter = cfg.counters ? cfg.counters + k : nullptr;
    int items = 0;
    for (int j = j0; j < njobs && j < j0 + RS_MAXJOBS; j++) {
      ResampleJob &J = B.jobs[B.njobs];
      J = jobs[j];
      if (cfg.seg_rows) {
        J.seg_rows = cfg.seg_rows;
        J.segs = (J.nrows + cfg.seg_rows - 1) / cfg.seg_rows;
      }
      J.item_begin = items;
      items += J.strips * J.segs;
      B.njobs++;
    }
    B.total_items = items;
    if (items == 0) continue;
    int grid = items;
    if (B.counter) {
      TOPS_CUDA_TRY(cudaMemsetAsync(B.counter, 0, sizeof(int), st));
      grid = min(items, cfg.grid > 0 ? cfg.grid : resident);
    }
    resample_kernel<kSplit><<<grid, RS_NT, sizeof(RsShared), st>>>(B);
    TOPS_CUDA_TRY(cudaGetLastError());
  }
  return TOPS_OK;
}

int launch_resample(const ResampleJob *jobs, int njobs, int precision, const TileCfg &cfg,
                    cudaStream_t st) {
  if (precision == TOPS_PREC_FP64) return launch_resample_t<false>(jobs, njobs, cfg, st);
  if (precision == TOPS_PREC_SPLIT) return launch_resample_t<true>(jobs, njobs, cfg, st);
  return TOPS_E_INVALID;
}

int resample_launch_multi(const tops_lut_dev *const *luts, const tops_resample_job *jobs,
                          int njobs, int precision, const TileCfg &cfg, cudaStream_t st) {
  if (!luts || (!jobs && njobs > 0) || njobs < 0) return TOPS_E_INVALID;
  std::vector<ResampleJob> J(njobs);
  for (int j = 0; j < njobs; j++) {
    if (!luts[j]) return TOPS_E_INVALID;
    int s = fill_resample_job(jobs[j], J[j]);
    if (s != TOPS_OK) return s;
    const LutDev &L = luts[j]->d;
    J[j].lut = LutPtrs{L.kaz, L.krg, L.krg2, L.sp1};
  }
  return launch_resample(J.data(), njobs, precision, cfg, st);
}

int resample_launch(const tops_lut_dev *lut, const tops_resample_job *jobs, int njobs,
                    int precision, const TileCfg &cfg, cudaStream_t st) {
  if (!lut || (!jobs && njobs > 0) || njobs < 0) return TOPS_E_INVALID;
  std::vector<const tops_lut_dev *> luts(njobs, lut);
  return resample_launch_multi(luts.data(), jobs, njobs, precision, cfg, st);
}

}  // namespace tops

extern "C" int tops_resample_ex(const tops_lut_dev *lut, const tops_resample_job *jobs,
                                int njobs, int precision, void *stream) {
  return resample_launch(lut, jobs, njobs, precision, TileCfg(),
                         static_cast<cudaStream_t>(stream));
}

extern "C" int tops_resample(const tops_lut_dev *lut, const tops_resample_job *jobs, int njobs,
                             void *stream) {
  return tops_resample_ex(lut, jobs, njobs, TOPS_PREC_SPLIT, stream);
}

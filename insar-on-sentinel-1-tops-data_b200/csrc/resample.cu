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
// B200 design (no textures, no phase array in HBM).  A CTA of 128 threads
// owns a strip of RS_TW = 112 output columns and a segment of up to 252
// output rows (a work item), swept in groups of RS_GR = 12 rows.
//
// Item prologue (all threads): per-row statistics from the offset
// polynomials -- along the strip y is a quadratic in the column, so a row
// whose whole strip maps to one (azimuth line, LUT bin) key (nearly every
// row of a TOPS pair) gets one shared azimuth pass -- with the row's FP64
// phase terms; per output column the runs of its range key (p0, bin) over
// the item, found by bisection of the exact per-pixel position (keys change
// every ~100+ rows), each run with its range weights' phase moments.
//
// Per group:
//   [A] azimuth pass, thread = ring column (RS_FW = 128 slave columns): the
//       thread's raw slave lines were staged in shared memory with cp.async
//       during the previous group; each new line is deramped in registers
//       and pushed into a 12-line register window (the window's slots rotate
//       with the row index, so a steady row costs one deramp and no moves);
//       v = sum_j kAz[j] d(L0-5+j) is 12 packed FP32x2 FMAs, written to the
//       group's 12 x 128 tile; then the next group's raw lines are staged,
//       so their copies land while [B] runs.
//   [B] range pass, thread = 2 adjacent output columns x 6 rows: the 14
//       tile samples of the pair are 7 16-byte loads, the 12 range weights
//       of each column stay in registers for its key run, and the reramp
//       phase is a dot product of row terms and column-run terms (below).
// A barrier separates [A] and [B]; the deferred passes [C1] (columns
// without run tables), [C2] (the second bin of two-bin rows) and [C] (the
// per-pixel path) follow [B] when the group has such pixels.
//
// The phase.  The reference reramps with the 144-tap FP64 sum
// Phi = sum_j sum_i kAz[j] kRg[i] phi(y_j, x_i).  With phi = phi_ref(y) +
// G(y, x), phi_ref the deramp phase of one reference column and G exactly
// quadratic in the burst-local time tc (G = g2 tc^2 + g1 tc + g0 per
// column), Phi = (1 + sp) Psi + G2 R2 + G1 R1 + G0 R0, with
//   Psi = sum_j kAz[j] phi_ref(y_j)                   (row, FP64, reduced)
//   sp  = sum_i kRg[i] - 1, Gk = sum_i kRg[i] gk(x_i)  (column key run)
//   R2 = M0 tc0^2 + 2 tc0 dt M1 + dt^2 M2, R1 = M0 tc0 + dt M1, R0 = M0
//        (row; M0..M2 the azimuth taps' moments, tc0 = tc(L0)),
// equal to the reference's sum in exact arithmetic.
//
// Every row whose strip maps to one azimuth key takes the shared pass: from
// the register window when its line is the window's, else (the row-to-line
// map skipped a line inside a group) by the same 12-line sum over lines
// deramped anew.  A row whose strip spans two adjacent bins of one line
// takes it for the first bin; the second bin's sums follow the range pass
// over the freed tile rows, and its columns (found by bisection in the
// prologue) go through the keyed path.  A column with more than RS_MAXRUN
// key runs in the item finds each pixel's key and run terms with the
// functions that build the run tables.  Rows with more azimuth keys, and
// pixels whose range support leaves the ring window, take a per-pixel path
// that computes the reference's formula from the slave in HBM; edge and
// outside pixels take the nearest sample and 0.  Which path a pixel takes depends on its row,
// its column and its strip only, never on the work item, so a job that
// produces a subset of the rows gives those rows bit for bit.
//
// Precision modes: TOPS_PREC_SPLIT (default) forms each sample's deramp
// phase in FP32 as rho(y) + G(y, x), rho the FP64 reference phase reduced
// once per slave line and G the FP32 quadratic about the burst's centre
// time, both in turns (cycles), so that the sum is reduced exactly by
// t - rint(t) before the sine and cosine.  TOPS_PREC_FP64 evaluates every
// sample's deramp phase and its reduction in FP64.  The reramp phase is
// formed in turns in both modes.  Positions, LUT bins and Psi are FP64 in
// both.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"
#include "launch.h"

namespace tops {

constexpr int RS_NT = 128;                 // threads per CTA
constexpr int RS_TW = 112;                 // output columns per strip
constexpr int RS_FW = 128;                 // ring (slave) columns of a strip
constexpr int RS_GR = 12;                  // rows per group (= azimuth taps)
constexpr int RS_HR = RS_GR / 2;           // rows per range-pass thread
constexpr int RS_SEG = 252;                // default rows per work item
constexpr int RS_MAXSEG = 252;             // per-item tables are sized for this
constexpr int RS_NGRP = (RS_MAXSEG + RS_GR - 1) / RS_GR;
constexpr int RS_SR = 32;                  // staged slave lines (power of two)
constexpr int RS_NSR = RS_MAXSEG + 44;     // slave-line phase table
constexpr int RS_MAXRUN = 6;               // range-key runs per column and item
constexpr int RS_MAXBIN = 16;              // distinct azimuth bins per item
constexpr int RS_NOSLOT = 0x7fff;          // azimuth bin outside the bin table
constexpr int RS_MAXJOBS = 32;
constexpr int RS_DP = RS_TW / 2;           // column pairs of the range pass
constexpr int RS_DT = 2 * RS_DP;           // range-pass threads
static_assert(RS_FW == RS_NT, "one ring column per thread in the azimuth pass");
static_assert(RS_DT <= RS_NT && RS_GR == 12 && RS_HR * 2 == RS_GR,
              "thread mappings assume these sizes");

enum : int { REG_OUT = 0, REG_EDGE = 1, REG_IN = 2 };
enum : int { RM_PIXEL = 0, RM_SHARED = 1, RM_TWO = 2 };

using RsLut = LutPtrs;

struct RsBatch {
  int njobs;
  int total_items;
  int *counter;            // persistent launch: work-item queue (else null)
  ResampleJob jobs[RS_MAXJOBS];
};

// One output row of a work item.
struct __align__(16) RsRow {
  float rho, psif, R2, R1;   // Psi mod 2 pi, Psi as float, residual-phase row terms
  float R0;
  int L0;                    // azimuth line of the shared azimuth pass
  int bin;                   // its LUT bin | bin-table slot << 16
  int mode;                  // RM_SHARED: the row takes the shared azimuth pass;
                             // RM_TWO | lo << 8 | hi << 16: the same, but columns
                             // [lo, hi) have the next LUT bin of the same line;
                             // RM_PIXEL: its pixels take the per-pixel path
};

// Deramp terms of one slave line: the burst-local azimuth time (FP64
// mode), or the reference-column phase mod 2 pi and ta - tm (split mode).
union RsSlaveRow {
  double ta;
  struct {
    float rho, tc;
  } f;
};

struct __align__(16) RsShared {
  float2 vd[RS_GR][RS_FW];            // azimuth-interpolated rows of the group
  short2 stage[RS_SR][RS_FW];         // raw slave lines, ring indexed by line & 31
  RsRow rows[RS_MAXSEG];
  RsSlaveRow srow[RS_NSR];            // slave lines ys0 .. ys0 + RS_NSR - 1
  float4 run_g[RS_TW][RS_MAXRUN];     // per range-key run: (sp, G2, G1, G0)
  int2 run_rk[RS_TW][RS_MAXRUN];      // (first item row, key = p0 * 4096 + bin)
  int run_n[RS_TW];                   // runs of the column (-1: more than RS_MAXRUN)
  float4 ring_gc[RS_FW];              // per ring column (g2, g1, g0, 0)
  float4 bin_w[RS_MAXBIN][6];         // azimuth taps as (w0,w0,w1,w1), ...
  int bin_id[RS_MAXBIN];
  alignas(16) double col_phat[RS_TW];
  double col_qaz[RS_TW], col_qrg[RS_TW];
  int4 gplan[RS_NGRP];                // per group: lines to stage before it, staged window
  int4 gwin[RS_NGRP];                 // per group: window on, filled at its start, line of row 0,
                                      // rows without a shared azimuth pass (bit mask)
  int2 grange[RS_NGRP];               // per group: lines its window pushes need
  RsRow r2[RS_GR];                    // row terms of the second bin of the group's two-bin rows
  int gen_n[RS_NGRP];                 // per group: pixels deferred to the per-pixel pass
  int gen_d[RS_NGRP];                 // per group: pixels of columns without a run table
  unsigned short gen[RS_GR * RS_TW];  // their (row in group) * 128 + column: the first
                                      // from the bottom, the second from the top
  int scan[RS_NT / 32];               // per-warp totals of the bin-change scan
  double caz[6], crg[6], shift;
  double ref_a0, ref_a1, ref_a2, tm;
  int xw, ys0, nbins, ngrp, next_item;
};

// Asynchronous 4-byte global -> shared copy; src_bytes 0 fills zeros.
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
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

// Phases of the split arithmetic are carried in turns (cycles): a turn is
// reduced to [-1/2, 1/2] by t - rint(t), exact for |t| < 2^22, and scaled
// by 2 pi once for the sine and cosine.
constexpr float kTwoPiF = 6.28318530717958647692f;
__device__ __forceinline__ float turns_reduce(float t) { return t - rintf(t); }
// An FP64 phase in radians as turns reduced to [-1/2, 1/2].
__device__ __forceinline__ float to_turns(double phi) {
  const double u = phi * kInvTwoPi;
  return (float)(u - rint(u));
}
// a * exp(-i 2 pi t), t in turns
__device__ __forceinline__ float2 cmul_conj_turns(float2 a, float t) {
  float s, c;
  __sincosf(turns_reduce(t) * kTwoPiF, &s, &c);
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

// my_polyval grouped by row: position = fma(B(row), P^, A(row) + c5 P^2)
// with A = c0 + c1 L^ + c3 L^2 and B = c2 + c4 L^.  Every path of the kernel
// evaluates positions with these functions, so their keys agree bit for bit.
__device__ __forceinline__ double row_L(const ResampleJob &J, int r) {
  return ((double)(r + J.my0) - J.midL) * J.invL;
}
__device__ __forceinline__ double row_a(const double *c, double L) {
  return fma(fma(c[3], L, c[1]), L, c[0]);
}
__device__ __forceinline__ double row_b(const double *c, double L) { return fma(c[4], L, c[2]); }
__device__ __forceinline__ double pix_pos(double A, double B, double P, double Q) {
  return fma(B, P, A + Q);
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

// Range key (p0 * 4096 + bin) of pixel (box row r, strip column c).
__device__ __forceinline__ int rg_key(const RsShared &S, const ResampleJob &J, int r, int c) {
  const double L = row_L(J, r);
  const double x = pix_pos(row_a(S.crg, L), row_b(S.crg, L), S.col_phat[c], S.col_qrg[c]);
  int p0, b;
  split_pos(x, p0, b);
  return p0 * 4096 + b;
}

// ---------------------------------------------------- HBM slow path
// Per-pixel interior resample straight from the CInt16 slave in HBM (rows
// and pixels the shared passes do not cover).
__device__ float2 interior_from_global(const ResampleJob &J, const RsLut &lut, int L0, int bL,
                                       int P0, int bP) {
  const float *kl = lut.kaz + bL * kTaps;
  const float *kp = lut.krg + bP * kTaps;
  float sre = 0.f, sim = 0.f;
  double ph = 0.0;
#pragma unroll 1
  for (int j = 0; j < kTaps; j++) {
    int y = L0 - 5 + j;
    double ta = (double)(y - J.s_first_line) * J.dt;
    float tre = 0.f, tim = 0.f;
    double tph = 0.0;
#pragma unroll 1
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

// Any pixel (box row r, strip column c) by the per-pixel definition.
__device__ __forceinline__ float2 pixel_generic(const RsShared &S, const ResampleJob &J, int r,
                                             int c) {
  const double L = row_L(J, r);
  const double P = S.col_phat[c];
  const double y = pix_pos(row_a(S.caz, L) + S.shift, row_b(S.caz, L), P, S.col_qaz[c]);
  const double x = pix_pos(row_a(S.crg, L), row_b(S.crg, L), P, S.col_qrg[c]);
  int l0, bl, p0, bp;
  split_pos(y, l0, bl);
  split_pos(x, p0, bp);
  const int reg = region_of(J, l0, p0);
  if (reg == REG_OUT) return make_float2(0.f, 0.f);
  if (reg == REG_EDGE) {
    const short2 sv = J.slave[(long)(l0 - J.sy0) * J.slave_pitch + (p0 - J.sx0)];
    return make_float2((float)sv.x, (float)sv.y);
  }
  return interior_from_global(J, J.lut, l0, bl, p0, bp);
}

// Range weights and phase terms of one output column's current key run.
struct ColRun {
  float4 w[6];    // (w0,w0,w1,w1), (w2,w2,w3,w3), ...
  float sp, G2, G1, G0;
  int key;        // p0 * 4096 + bin
  int next;       // first item row of the next run
  int m;          // run index
  bool ok;        // range-interior and inside the ring window: fast range pass
};

__device__ __forceinline__ void run_load(ColRun &cr, const RsShared &S, const ResampleJob &J,
                                         int c, int m) {
  const int n = S.run_n[c];
  const int2 rk = S.run_rk[c][m];
  const float4 g = S.run_g[c][m];
  cr.m = m;
  cr.key = rk.y;
  cr.next = (m + 1 < n) ? S.run_rk[c][m + 1].x : INT32_MAX;
  cr.sp = g.x;
  cr.G2 = g.y;
  cr.G1 = g.z;
  cr.G0 = g.w;
  const int p0 = rk.y >> 12;
  const int xb = p0 - 5 - S.xw;
  cr.ok = p0 >= J.sx0 + 5 && p0 <= J.sx1 - 7 && xb >= 0 && xb + 13 < RS_FW;
}

// The range weights of the column's current run (fast runs only).  They are
// loaded at the start of each group's range pass and after a run change, so
// they hold no registers during the azimuth pass.
__device__ __forceinline__ void run_weights(ColRun &cr, const ResampleJob &J) {
  if (cr.ok) {
    const float4 *kp4 = J.lut.krg2 + (cr.key & 4095) * (kTaps / 2);
#pragma unroll
    for (int q = 0; q < kTaps / 2; q++) cr.w[q] = __ldg(kp4 + q);
  }
}

__device__ __forceinline__ float2 wtap(const ColRun &cr, int i) {
  const float4 q = cr.w[i >> 1];
  return (i & 1) ? make_float2(q.z, q.w) : make_float2(q.x, q.y);
}

// 12-tap range pass of two adjacent columns over the 14 samples V (the first
// column's taps start at V[odd], the second's at V[odd + 1]); two partial
// sums per column shorten the FMA chains.
__device__ __forceinline__ void range_pair(const ColRun &c0, const ColRun &c1,
                                           const float2 (&V)[14], bool odd, float2 &s0,
                                           float2 &s1) {
  float2 a0 = make_float2(0.f, 0.f), b0 = a0, a1 = a0, b1 = a0;
  if (odd) {
#pragma unroll
    for (int i = 0; i < kTaps; i += 2) {
      a0 = __ffma2_rn(wtap(c0, i), V[i + 1], a0);
      b0 = __ffma2_rn(wtap(c0, i + 1), V[i + 2], b0);
      a1 = __ffma2_rn(wtap(c1, i), V[i + 2], a1);
      b1 = __ffma2_rn(wtap(c1, i + 1), V[i + 3], b1);
    }
  } else {
#pragma unroll
    for (int i = 0; i < kTaps; i += 2) {
      a0 = __ffma2_rn(wtap(c0, i), V[i], a0);
      b0 = __ffma2_rn(wtap(c0, i + 1), V[i + 1], b0);
      a1 = __ffma2_rn(wtap(c1, i), V[i + 1], a1);
      b1 = __ffma2_rn(wtap(c1, i + 1), V[i + 2], b1);
    }
  }
  s0 = __fadd2_rn(a0, b0);
  s1 = __fadd2_rn(a1, b1);
}

// 12-tap range pass of one column from a tile row (8-byte loads).
__device__ __forceinline__ float2 range_single(const float2 *row, int xb, const ColRun &cr) {
  float2 a = make_float2(0.f, 0.f), b = a;
#pragma unroll
  for (int i = 0; i < kTaps; i += 2) {
    a = __ffma2_rn(wtap(cr, i), row[xb + i], a);
    b = __ffma2_rn(wtap(cr, i + 1), row[xb + i + 1], b);
  }
  return __fadd2_rn(a, b);
}

// Reramp phase of a pixel: (1 + sp) Psi + G2 R2 + G1 R1 + G0 R0, with Psi
// as its reduced value plus sp times its float value.
__device__ __forceinline__ float run_phase(const RsRow &R, const ColRun &cr) {
  return fmaf(cr.sp, R.psif, R.rho) + fmaf(cr.G2, R.R2, fmaf(cr.G1, R.R1, cr.G0 * R.R0));
}

// Deramped slave sample (line y, this thread's ring column) for the
// azimuth-pass window: from the staged lines when the line is staged, else
// from HBM.
template <bool kSplit>
__device__ __forceinline__ float2 deramp_at(const RsShared &S, const ResampleJob &J, int x,
                                            int xa, bool xin, int y, int win_lo, int win_hi,
                                            float g2c, float g1c, float g0c,
                                            const DerampQuad &cq) {
  float sx, sy;
  if (y >= win_lo && y <= win_hi) {
    const short2 v = S.stage[y & (RS_SR - 1)][x];
    sx = (float)v.x;
    sy = (float)v.y;
  } else {
    if (!xin || y < J.sy0 || y > J.sy1) return make_float2(0.f, 0.f);
    const short2 v = J.slave[(long)(y - J.sy0) * J.slave_pitch + (xa - J.sx0)];
    sx = (float)v.x;
    sy = (float)v.y;
  }
  const int iy = y - S.ys0;
  float r;
  if (kSplit) {
    float rho, tc;
    if ((unsigned)iy < (unsigned)RS_NSR) {
      rho = S.srow[iy].f.rho;
      tc = S.srow[iy].f.tc;
    } else {
      const DerampQuad refq = {S.ref_a0, S.ref_a1, S.ref_a2};
      const double ta = (double)(y - J.s_first_line) * J.dt;
      rho = to_turns(quad_eval(refq, ta));
      tc = (float)(ta - S.tm);
    }
    const float G = fmaf(fmaf(g2c, tc, g1c), tc, g0c);
    r = turns_reduce(rho + G) * kTwoPiF;
  } else {
    const double ta = ((unsigned)iy < (unsigned)RS_NSR) ? S.srow[iy].ta
                                                         : (double)(y - J.s_first_line) * J.dt;
    r = reduce_2pi(quad_eval(cq, ta));
  }
  float sn, cs;
  __sincosf(r, &sn, &cs);
  return make_float2(sx * cs - sy * sn, sx * sn + sy * cs);
}

// deramp_at for a line known to be staged and in the slave-line table.
template <bool kSplit>
__device__ __forceinline__ float2 deramp_staged(const RsShared &S, int x, int y, int ys0,
                                                float g2c, float g1c, float g0c,
                                                const DerampQuad &cq) {
  const short2 v = S.stage[y & (RS_SR - 1)][x];
  const float sx = (float)v.x, sy = (float)v.y;
  const RsSlaveRow sr = S.srow[y - ys0];
  float r;
  if (kSplit) {
    const float G = fmaf(fmaf(g2c, sr.f.tc, g1c), sr.f.tc, g0c);
    r = turns_reduce(sr.f.rho + G) * kTwoPiF;
  } else {
    r = reduce_2pi(quad_eval(cq, sr.ta));
  }
  float sn, cs;
  __sincosf(r, &sn, &cs);
  return make_float2(sx * cs - sy * sn, sx * sn + sy * cs);
}

// Azimuth taps of a row (bin | slot << 16) as (w, w) pairs.
__device__ __forceinline__ void load_az_taps(const RsShared &S, const RsLut &lut, int bin,
                                             float4 (&wz)[6]) {
  const int slot = bin >> 16;
  if (slot < RS_MAXBIN) {
#pragma unroll
    for (int q = 0; q < 6; q++) wz[q] = S.bin_w[slot][q];
  } else {
    const float *kl = lut.kaz + (bin & 0xffff) * kTaps;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const float a = __ldg(kl + 2 * q), b = __ldg(kl + 2 * q + 1);
      wz[q] = make_float4(a, a, b, b);
    }
  }
}

// Stage this thread's ring column of slave lines [lo, hi] (zeros outside
// the slave box) into the line ring.
__device__ __forceinline__ void stage_rows(RsShared &S, const ResampleJob &J, int x, int xa,
                                           bool xin, int lo, int hi) {
  const short2 *const sl = J.slave;
  const long pitch = J.slave_pitch;
  const unsigned base = smem_u32(&S.stage[0][x]);
  constexpr unsigned kRow = RS_FW * sizeof(short2);
  if (xin && lo >= J.sy0 && hi <= J.sy1) {
    // every line inside the slave box (the usual case): no per-line checks
    const short2 *src = sl + (long)(lo - J.sy0) * pitch + (xa - J.sx0);
#pragma unroll 4
    for (int y = lo; y <= hi; y++, src += pitch)
      cp_async_4s(base + (unsigned)(y & (RS_SR - 1)) * kRow, src, 4);
  } else {
    const unsigned rows_in = (unsigned)(J.sy1 - J.sy0);
    long off = (long)(lo - J.sy0) * pitch + (xa - J.sx0);
#pragma unroll 1
    for (int y = lo; y <= hi; y++, off += pitch) {
      const bool in = xin && (unsigned)(y - J.sy0) <= rows_in;
      cp_async_4s(base + (unsigned)(y & (RS_SR - 1)) * kRow, sl + (in ? off : 0), in ? 4 : 0);
    }
  }
  cp_async_commit();
}

// Phase terms of a range-key run: (sp, G2, G1, G0) with Gk = sum_i kRg[i]
// gk(x_i) over the ring columns of its taps (0 when they leave the window).
__device__ __forceinline__ float4 run_terms(const RsShared &S, const RsLut &lut, int xw,
                                            int key) {
  const int p0 = key >> 12, bp = key & 4095;
  const int xb = p0 - 5 - xw;
  float4 gg = make_float4(__ldg(lut.sp1 + bp), 0.f, 0.f, 0.f);
  if (xb >= 0 && xb + kTaps <= RS_FW) {
    const float *kp = lut.krg + bp * kTaps;
    float G2 = 0.f, G1 = 0.f, G0 = 0.f;
#pragma unroll
    for (int i = 0; i < kTaps; i++) {
      const float w = __ldg(kp + i);
      const float4 gc = S.ring_gc[xb + i];
      G2 = fmaf(w, gc.x, G2);
      G1 = fmaf(w, gc.y, G1);
      G0 = fmaf(w, gc.z, G0);
    }
    gg.y = G2;
    gg.z = G1;
    gg.w = G0;
  }
  return gg;
}

// A pixel of a shared row (its azimuth-interpolated row in vrow) whose
// column has no run table: its range key and the key's run terms are found
// here, by the same functions the run tables are built with, so the result
// is the one the run path gives.
__device__ __forceinline__ float2 pixel_keyed(const RsShared &S, const ResampleJob &J,
                                           const RsRow &R, const float2 *vrow, int r, int c) {
  ColRun cr;
  cr.key = rg_key(S, J, r, c);
  const float4 g = run_terms(S, J.lut, S.xw, cr.key);
  cr.sp = g.x;
  cr.G2 = g.y;
  cr.G1 = g.z;
  cr.G0 = g.w;
  const int p0 = cr.key >> 12;
  const int xb = p0 - 5 - S.xw;
  cr.ok = p0 >= J.sx0 + 5 && p0 <= J.sx1 - 7 && xb >= 0 && xb + 13 < RS_FW;
  if (cr.ok) {
    run_weights(cr, J);
    return cmul_conj_turns(range_single(vrow, xb, cr), run_phase(R, cr));
  }
  if (p0 < J.sx0 || p0 > J.sx1) return make_float2(0.f, 0.f);
  if (p0 < J.sx0 + 5 || p0 > J.sx1 - 7) {
    const short2 sv = J.slave[(long)(R.L0 - J.sy0) * J.slave_pitch + (p0 - J.sx0)];
    return make_float2((float)sv.x, (float)sv.y);
  }
  return pixel_generic(S, J, r, c);
}

// Azimuth sum of this thread's ring column for the key (L0, bin) over
// lines deramped anew (staged lines in [win_lo, win_hi] from shared memory,
// others from HBM), in the order of the register-window sum.
template <bool kSplit>
__device__ __forceinline__ float2 az_direct(const RsShared &S, const ResampleJob &J,
                                            const RsLut &lut, int x, int xa, bool xin, int L0,
                                            int bin, int win_lo, int win_hi, float g2c,
                                            float g1c, float g0c, const DerampQuad &cq) {
  const float *kl = lut.kaz + bin * kTaps;
  float2 a = make_float2(0.f, 0.f), b = a;
#pragma unroll 1
  for (int j = 0; j < RS_GR; j += 2) {
    const float wa = __ldg(kl + j), wb = __ldg(kl + j + 1);
    const float2 d0 =
        deramp_at<kSplit>(S, J, x, xa, xin, L0 - 5 + j, win_lo, win_hi, g2c, g1c, g0c, cq);
    const float2 d1 =
        deramp_at<kSplit>(S, J, x, xa, xin, L0 - 4 + j, win_lo, win_hi, g2c, g1c, g0c, cq);
    a = __ffma2_rn(make_float2(wa, wa), d0, a);
    b = __ffma2_rn(make_float2(wb, wb), d1, b);
  }
  return __fadd2_rn(a, b);
}

// Reramp row terms of the azimuth key (L0, bin): Psi = sum_j kAz[j]
// phi_ref(L0 - 5 + j) (FP64) and the taps' moments about the burst centre
// time.
__device__ __forceinline__ void row_terms(const RsShared &S, const ResampleJob &J,
                                          const RsLut &lut, int L0, int bin, RsRow &R) {
  const DerampQuad refq = {S.ref_a0, S.ref_a1, S.ref_a2};
  const float *kl = lut.kaz + bin * kTaps;
  double psi = 0.0, m0 = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll 4
  for (int j = 0; j < kTaps; j++) {
    const double w = (double)__ldg(kl + j), u = (double)(j - 5);
    const double ta = (double)(L0 - 5 + j - J.s_first_line) * J.dt;
    psi = fma(w, quad_eval(refq, ta), psi);
    m0 += w;
    m1 = fma(w, u, m1);
    m2 = fma(w, u * u, m2);
  }
  const double tc0 = (double)(L0 - J.s_first_line) * J.dt - S.tm;
  const double dt = J.dt;
  R.rho = to_turns(psi);
  R.psif = (float)(psi * kInvTwoPi);
  R.R2 = (float)(m0 * tc0 * tc0 + 2.0 * tc0 * dt * m1 + dt * dt * m2);
  R.R1 = (float)(m0 * tc0 + dt * m1);
  R.R0 = (float)m0;
}

// One work item (strip x segment of one job); all threads of the CTA call it
// with the same item.
template <bool kSplit>
__device__ __forceinline__ void resample_item(RsShared &S, const RsBatch &B, int item) {
  const int tid = threadIdx.x;

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
  const int nr = r_end - r_begin;

  // ---- [P1] polynomials and shift
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

  // ---- [P2] column terms; the ring window and the reference column
  if (tid < RS_TW) {
    const double P = ((double)(c0 + min(tid, cN - 1)) - J.midP) * J.invP;
    S.col_phat[tid] = P;
    S.col_qaz[tid] = S.caz[5] * P * P;
    S.col_qrg[tid] = S.crg[5] * P * P;
  }
  if (tid == RS_NT - 1) {
    // range position at the corners and edge midpoints of the strip over
    // the whole master box -> window.  The window, and with it the reference
    // column of the phase split, depends on the strip only, so a job that
    // produces a subset of the rows gives those rows bit for bit as the
    // whole job does.
    double pmin = 1e300;
    const int box_rows = J.my1 - J.my0 + 1;
    for (int a = 0; a < 3; a++) {
      const int rr = (a == 0) ? 0 : (a == 1 ? (box_rows - 1) / 2 : box_rows - 1);
      const double L = row_L(J, rr);
      for (int b = 0; b < 3; b++) {
        const int cc = (b == 0) ? c0 : (b == 1 ? c0 + (cN - 1) / 2 : c0 + cN - 1);
        const double P = ((double)cc - J.midP) * J.invP;
        const double *c = S.crg;
        const double x = c[0] + c[1] * L + c[2] * P + c[3] * L * L + c[4] * L * P + c[5] * P * P;
        pmin = fmin(pmin, x);
      }
    }
    // the range pass reads ring columns [p0 - 5, p0 + 8] of a column pair;
    // one column of margin for the position's variation inside the strip
    const int xw = (int)floor(pmin) - 6;
    S.xw = xw;
    S.ys0 = INT32_MAX;   // first slave line used: minimum taken in [P6a]
    const int xr = min(max(xw + RS_FW / 2, J.sx0), J.sx1);
    const DerampQuad q = deramp_quad(J.kt[xr], J.tref[xr], J.fdc[xr]);
    S.ref_a0 = q.a0;
    S.ref_a1 = q.a1;
    S.ref_a2 = q.a2;
    S.tm = 0.5 * (double)(J.sy0 + J.sy1 - 2 * J.s_first_line) * J.dt;
  }
  __syncthreads();

  // ---- [P3] this thread's ring column: deramp coefficients
  const int xw = S.xw;
  const int x = tid;                     // ring column
  const int xa = xw + x;                 // absolute slave column
  const bool xin = xa >= J.sx0 && xa <= J.sx1;
  const double tm = S.tm;
  DerampQuad cq;
  float g2c, g1c, g0c;   // G = phi - phi_ref about tm: g2 tc^2 + g1 tc + g0
  {
    const DerampQuad refq = {S.ref_a0, S.ref_a1, S.ref_a2};
    cq = refq;
    if (xin) cq = deramp_quad(J.kt[xa], J.tref[xa], J.fdc[xa]);
    const double d2 = cq.a2 - refq.a2, d1 = cq.a1 - refq.a1, d0 = cq.a0 - refq.a0;
    g2c = (float)(d2 * kInvTwoPi);   // in turns
    g1c = (float)((2.0 * d2 * tm + d1) * kInvTwoPi);
    g0c = (float)(((d2 * tm + d1) * tm + d0) * kInvTwoPi);
  }
  S.ring_gc[x] = make_float4(g2c, g1c, g0c, 0.f);

  // ---- [P4] per-row statistics: one shared azimuth pass where the whole
  // strip maps to one (line, bin) key inside the slave box's interior; where
  // it maps to two adjacent bins of one line and the position is monotone
  // along the strip, the columns of the second bin are found by bisection of
  // the exact per-pixel key
  for (int ri = tid; ri < nr; ri += RS_NT) {
    const double L = row_L(J, r_begin + ri);
    const double Aaz = row_a(S.caz, L) + S.shift, Baz = row_b(S.caz, L);
    double ylo, yhi;
    quad_span(Aaz, Baz, S.caz[5], S.col_phat[0], S.col_phat[cN - 1], ylo, yhi);
    int l0lo, blo, l0hi, bhi;
    split_pos(ylo, l0lo, blo);
    split_pos(yhi, l0hi, bhi);
    const bool inter = l0lo >= J.sy0 + 5 && l0hi <= J.sy1 - 7;
    const bool fast = (l0lo == l0hi) && (blo == bhi) && inter;
    int mode = fast ? RM_SHARED : RM_PIXEL;
    if (!fast && inter && l0lo == l0hi && bhi == blo + 1) {
      const double c2 = 2.0 * S.caz[5];
      const double s0 = fma(c2, S.col_phat[0], Baz), s1 = fma(c2, S.col_phat[cN - 1], Baz);
      if ((s0 < 0.0) == (s1 < 0.0)) {
        auto is_hi = [&](int c) {
          int l, b;
          split_pos(pix_pos(Aaz, Baz, S.col_phat[c], S.col_qaz[c]), l, b);
          return b == bhi;
        };
        const bool f0 = is_hi(0);
        int t = cN;   // first column whose bin differs from column 0's
        if (is_hi(cN - 1) != f0) {
          int lo = 0, hi = cN - 1;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (is_hi(mid) == f0)
              lo = mid;
            else
              hi = mid;
          }
          t = hi;
        }
        const int c_lo = f0 ? 0 : t, c_hi = f0 ? t : cN;
        mode = RM_TWO | (c_lo << 8) | (c_hi << 16);
      }
    }
    RsRow R;
    R.L0 = l0lo;
    R.bin = blo | (RS_NOSLOT << 16);
    R.rho = R.psif = R.R2 = R.R1 = R.R0 = 0.f;
    if (mode != RM_PIXEL) row_terms(S, J, lut, l0lo, blo, R);
    R.mode = mode;
    S.rows[ri] = R;
  }
  __syncthreads();

  // ---- [P5] the window of the azimuth pass over the groups.  The window
  // advances one line per row; a group whose first row with a single key
  // finds another line than the window expects (or no window yet) fills it
  // anew at the group's start, with the line of that row extrapolated back
  // one line per row.  A row takes the shared pass when it has a single key
  // and its line is the window's.  Thread g finds group g's first
  // single-key row; thread 0 then chains the groups.
  {
    const int ngrp = (nr + RS_GR - 1) / RS_GR;
    if (tid < ngrp) {
      int k1 = -1, l1 = 0;
      for (int k = 0; k < RS_GR && tid * RS_GR + k < nr; k++) {
        const RsRow &R = S.rows[tid * RS_GR + k];
        if (R.mode) {
          k1 = k;
          l1 = R.L0;
          break;
        }
      }
      S.grange[tid] = make_int2(k1, l1);
    }
  }
  __syncthreads();
  if (tid == 0) {
    const int ngrp = (nr + RS_GR - 1) / RS_GR;
    bool on = false;
    int base_row = 0, base_L0 = 0;
    for (int g = 0; g < ngrp; g++) {
      const int p = g * RS_GR;
      const int2 f = S.grange[g];   // first single-key row of the group, its line
      bool fill = false;
      if (f.x >= 0 && (!on || f.y != base_L0 + (p + f.x - base_row))) {
        fill = true;
        on = true;
        base_row = p + f.x;
        base_L0 = f.y;
      }
      // (window on, bit 0: filled here | bit 1: check-free loop, line of
      // row 0, per-pixel rows)
      S.gwin[g] = make_int4(on ? 1 : 0, fill ? 1 : 0, on ? base_L0 + (p - base_row) : 0, 0);
      S.gen_n[g] = 0;
      S.gen_d[g] = 0;
    }
    S.ngrp = ngrp;
  }
  __syncthreads();

  // ---- [P6a] row modes; azimuth-bin table (a slot per change of the bin
  // between consecutive shared rows, ranked by a block-wide scan); each
  // group's line range and per-pixel rows; the first slave line used.
  // Thread t takes rows 2t and 2t + 1.
  {
    const int lane = tid & 31, warp = tid >> 5;
    const int r0 = 2 * tid, r1 = r0 + 1;
    auto shared_row = [&](int ri) -> bool { return ri < nr && S.rows[ri].mode; };
    const bool h0 = shared_row(r0), h1 = shared_row(r1);
    const bool p0 = r0 > 0 && shared_row(r0 - 1);
    auto bin_of = [&](int ri) { return S.rows[ri].bin & 0xffff; };
    const int f0 = h0 && (!p0 || bin_of(r0 - 1) != bin_of(r0)) ? 1 : 0;
    const int f1 = h1 && (!h0 || bin_of(r0) != bin_of(r1)) ? 1 : 0;
    int v = f0 + f1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) S.scan[warp] = v;
    int ymin = INT32_MAX;
    const int ngrp = S.ngrp;
    if (tid < ngrp) {
      const int4 gw = S.gwin[tid];
      const int gr = min(RS_GR, nr - tid * RS_GR);
      if (gw.x) ymin = gw.z - (gw.y ? 5 : -6);
      // rows without a shared pass (bits 0..11) and shared rows whose line
      // is not the window's, summed directly (bits 16..27)
      int mask = 0, two = 0;
      for (int k = 0; k < gr; k++) {
        const int ri = tid * RS_GR + k;
        if (!shared_row(ri))
          mask |= 1 << k;
        else if (!gw.x || S.rows[ri].L0 != gw.z + k)
          mask |= 1 << (16 + k);
        if (shared_row(ri) && (S.rows[ri].mode & 0xff) == RM_TWO) two |= 1 << k;
      }
      // rows with a second bin (bits 4..15 of the flags)
      S.gwin[tid].y = gw.y | (two << 4);
      S.grange[tid] = gw.x ? make_int2(gw.y ? gw.z - 5 : gw.z + 6, gw.z + gr - 1 + 6)
                           : make_int2(1, 0);
      S.gwin[tid].w = mask;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
    if (lane == 0 && ymin != INT32_MAX) atomicMin(&S.ys0, ymin);
    __syncthreads();
    int off = 0, total = 0;
#pragma unroll
    for (int q = 0; q < RS_NT / 32; q++) {
      const int t = S.scan[q];
      off += q < warp ? t : 0;
      total += t;
    }
    const int incl0 = off + v - f1, incl1 = incl0 + f1;   // inclusive ranks
    auto set_row = [&](int ri, bool h, int incl, int f) {
      if (ri >= nr) return;
      RsRow &R = S.rows[ri];
      if (!h) {
        R.mode = RM_PIXEL;
        return;
      }
      const int b = R.bin & 0xffff;
      const int slot = incl - 1 < RS_MAXBIN ? incl - 1 : RS_NOSLOT;
      R.bin = b | (slot << 16);
      if (f && slot < RS_MAXBIN) S.bin_id[slot] = b;
    };
    set_row(r0, h0, incl0, f0);
    set_row(r1, h1, incl1, f1);
    if (tid == 0) S.nbins = min(total, RS_MAXBIN);
  }
  __syncthreads();

  // ---- [P6b] thread 0: the staging plan (a short chain over the groups);
  // threads 16..127: range-key runs of the columns
  if (tid == 0) {
    if (S.ys0 == INT32_MAX) S.ys0 = 0;
    // the lines each group's window pushes need, copied before the group
    // (at most RS_SR lines kept)
    int st_lo = 1, st_hi = 0;
    for (int g = 0; g < S.ngrp; g++) {
      int lo = S.grange[g].x;
      const int hi = S.grange[g].y;
      int c_lo = 1, c_hi = 0;
      if (lo <= hi) {
        lo = max(lo, hi - (RS_SR - 1));
        if (st_lo <= st_hi && lo >= st_lo && lo <= st_hi + 1) {
          c_lo = st_hi + 1;   // extend the staged window
          c_hi = hi;
          st_hi = max(st_hi, hi);
          st_lo = max(st_lo, st_hi - (RS_SR - 1));
        } else {
          c_lo = lo;          // restart it
          c_hi = hi;
          st_lo = lo;
          st_hi = hi;
        }
      }
      S.gplan[g] = make_int4(c_lo, c_hi, st_lo, st_hi);
      // a full group whose rows all take the shared pass and whose lines are
      // all staged and in the slave-line table takes the check-free loop
      const int4 gw = S.gwin[g];
      const int lo_need = (gw.y & 1) ? gw.z - 5 : gw.z + 6;
      const bool simple = gw.x && g * RS_GR + RS_GR <= nr && gw.w == 0 && lo_need >= st_lo &&
                          hi <= st_hi && lo_need >= S.ys0 && hi < S.ys0 + RS_NSR;
      if (simple) S.gwin[g].y = gw.y | 2;
    }
  } else if (tid >= RS_NT - RS_TW) {
    const int c = tid - (RS_NT - RS_TW);
    if (c < cN) {
      // runs of the range key over the item rows, by bisection of the exact
      // per-pixel key on the pieces where the position is monotone in the
      // row; a piece that starts with the key the previous one ended with
      // continues its run
      auto keyat = [&](int ri) { return rg_key(S, J, r_begin + ri, c); };
      int ends[2] = {nr - 1, nr - 1};
      int np = 1;
      {
        // x(L) = g0 + g2 P + g5 P^2 + (g1 + g4 P) L + g3 L^2: vertex in L
        const double *g = S.crg;
        const double P = S.col_phat[c];
        if (g[3] != 0.0) {
          const double Lv = -(g[1] + g[4] * P) / (2.0 * g[3]);
          const double rv = Lv / J.invL + J.midL - (double)J.my0 - (double)r_begin;
          if (rv > 0.0 && rv < (double)(nr - 1)) {
            ends[0] = (int)rv;
            np = 2;
          }
        }
      }
      int n = 0, last_key = INT32_MIN;
      bool dense = false;
      int a = 0;
      for (int pc = 0; pc < np && !dense; pc++) {
        const int bend = ends[pc];
        int r = a, k = keyat(a);
        const int kb = keyat(bend);
        for (;;) {
          if (k != last_key) {
            if (n == RS_MAXRUN) {
              dense = true;
              break;
            }
            S.run_rk[c][n] = make_int2(r, k);
            S.run_g[c][n] = run_terms(S, lut, xw, k);
            n++;
            last_key = k;
          }
          if (k == kb) break;   // monotone: the rest of the piece has this key
          int lo = r, hi = bend, khi = kb;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            const int km = keyat(mid);
            if (km == k) {
              lo = mid;
            } else {
              hi = mid;
              khi = km;
            }
          }
          r = hi;
          k = khi;
        }
        a = bend + 1;
      }
      S.run_n[c] = dense ? -1 : n;
    }
  }
  __syncthreads();

  // ---- [P7] stage the first group's lines; slave-line phase table; the
  // azimuth taps of the bin table
  {
    const int4 p = S.gplan[0];
    if (p.x <= p.y) stage_rows(S, J, x, xa, xin, p.x, p.y);
  }
  {
    const DerampQuad refq = {S.ref_a0, S.ref_a1, S.ref_a2};
    for (int i = tid; i < RS_NSR; i += RS_NT) {
      const int y = S.ys0 + i;
      const double ta = (double)(y - J.s_first_line) * J.dt;
      RsSlaveRow sr;
      if (kSplit) {
        sr.f.rho = to_turns(quad_eval(refq, ta));
        sr.f.tc = (float)(ta - tm);
      } else {
        sr.ta = ta;
      }
      S.srow[i] = sr;
    }
  }
  for (int e = tid; e < S.nbins * 6; e += RS_NT) {
    const int slot = e / 6, q = e - slot * 6;
    const float *kl = lut.kaz + S.bin_id[slot] * kTaps + 2 * q;
    const float a = __ldg(kl), b = __ldg(kl + 1);
    S.bin_w[slot][q] = make_float4(a, a, b, b);
  }
  __syncthreads();

  // ---- range-pass thread: column pair (dc, dc + 1), rows 6h .. 6h + 5 of a group
  const int dp = tid % RS_DP, dh = tid / RS_DP;
  const bool dthread = tid < RS_DT;
  const int dc = 2 * dp;
  const bool dval0 = dthread && dc < cN, dval1 = dthread && dc + 1 < cN;
  const bool dense0 = dval0 && S.run_n[dc] < 0, dense1 = dval1 && S.run_n[dc + 1] < 0;
  ColRun cr0, cr1;
  cr0.ok = cr1.ok = false;
  cr0.next = cr1.next = INT32_MAX;
  cr0.key = cr1.key = 0;
  cr0.m = cr1.m = 0;
  if (dval0 && !dense0) run_load(cr0, S, J, dc, 0);
  if (dval1 && !dense1) run_load(cr1, S, J, dc + 1, 0);
  const bool out16 = J.out_al16 != 0;

  // azimuth-pass state: the 12-line window of this ring column (line
  // wl0 + k - 5 + j of group row k in slot (k + j) % 12) and the taps
  float2 w[RS_GR];
#pragma unroll
  for (int j = 0; j < RS_GR; j++) w[j] = make_float2(0.f, 0.f);
  float4 wz[6];
#pragma unroll
  for (int q = 0; q < 6; q++) wz[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  int wz_bin = -1;

  const int ngrp = S.ngrp;
  for (int g = 0; g < ngrp; g++) {
    const int rg0 = g * RS_GR;            // first item row of the group
    const int gr = min(RS_GR, nr - rg0);
    const int4 plan = S.gplan[g];
    const int4 gw = S.gwin[g];
    const int pixmask = gw.w & 0xfff;     // rows without a shared pass ([A] only)
    const int dirmask = gw.w >> 16;       // shared rows off the window's line
    cp_async_wait_all();                  // this thread's staged lines of the group
    // ---- [A] azimuth pass of the group's rows (the taps are loaded anew per
    // group, so they hold no registers during [B] and [C])
    wz_bin = -1;
    if (gw.y & 2) {
      // every row takes the shared pass, every line is staged
      const int wl0 = gw.z;
      const int ys0 = S.ys0;
      if (gw.y & 1) {
#pragma unroll
        for (int j = 0; j < RS_GR - 1; j++)
          w[j] = deramp_staged<kSplit>(S, x, wl0 - 5 + j, ys0, g2c, g1c, g0c, cq);
      }
#pragma unroll
      for (int k = 0; k < RS_GR; k++) {
        w[(k + 11) % RS_GR] = deramp_staged<kSplit>(S, x, wl0 + k + 6, ys0, g2c, g1c, g0c, cq);
        const int bin = S.rows[rg0 + k].bin;
        if (bin != wz_bin) {
          load_az_taps(S, lut, bin, wz);
          wz_bin = bin;
        }
        float2 a = make_float2(0.f, 0.f), b = a;
#pragma unroll
        for (int j = 0; j < RS_GR; j += 2) {
          const float4 q = wz[j >> 1];
          a = __ffma2_rn(make_float2(q.x, q.y), w[(k + j) % RS_GR], a);
          b = __ffma2_rn(make_float2(q.z, q.w), w[(k + j + 1) % RS_GR], b);
        }
        S.vd[k][x] = __fadd2_rn(a, b);
      }
    } else if (gw.x) {
      const int wl0 = gw.z;
      if (gw.y & 1) {
        // fill the window of row 0 (slots 0..10; row 0 pushes slot 11)
#pragma unroll
        for (int j = 0; j < RS_GR - 1; j++)
          w[j] = deramp_at<kSplit>(S, J, x, xa, xin, wl0 - 5 + j, plan.z, plan.w, g2c, g1c,
                                   g0c, cq);
      }
#pragma unroll
      for (int k = 0; k < RS_GR; k++) {
        if (k < gr) {
          w[(k + 11) % RS_GR] = deramp_at<kSplit>(S, J, x, xa, xin, wl0 + k + 6, plan.z, plan.w,
                                                  g2c, g1c, g0c, cq);
          if (!(((pixmask | dirmask) >> k) & 1)) {
            const int bin = S.rows[rg0 + k].bin;
            if (bin != wz_bin) {
              load_az_taps(S, lut, bin, wz);
              wz_bin = bin;
            }
            float2 a = make_float2(0.f, 0.f), b = a;
#pragma unroll
            for (int j = 0; j < RS_GR; j += 2) {
              const float4 q = wz[j >> 1];
              a = __ffma2_rn(make_float2(q.x, q.y), w[(k + j) % RS_GR], a);
              b = __ffma2_rn(make_float2(q.z, q.w), w[(k + j + 1) % RS_GR], b);
            }
            S.vd[k][x] = __fadd2_rn(a, b);
          }
        }
      }
    }
    if (dirmask) {
      // shared rows whose line is not the window's (the row-to-line map
      // skipped a line inside the group): the same sum, in the same order,
      // over lines deramped anew
#pragma unroll 1
      for (int m = dirmask; m; m &= m - 1) {
        const int k = __ffs(m) - 1;
        const RsRow &R = S.rows[rg0 + k];
        S.vd[k][x] = az_direct<kSplit>(S, J, lut, x, xa, xin, R.L0, R.bin & 0xffff, plan.z,
                                       plan.w, g2c, g1c, g0c, cq);
      }
    }
    // stage the next group's new lines; they land while [B] runs
    if (g + 1 < ngrp) {
      const int4 pn = S.gplan[g + 1];
      if (pn.x <= pn.y) stage_rows(S, J, x, xa, xin, pn.x, pn.y);
    }
    __syncthreads();

    // ---- [B] range pass, reramp, store: 2 columns x 6 rows per thread;
    // pixels the shared passes do not cover are listed for [C]
    // rows without a shared pass and two-bin rows (read again here, so the
    // group's flags hold no registers during [B])
    const int bskip = (S.gwin[g].w & 0xfff) | ((S.gwin[g].y >> 4) & 0xfff);
    if (dval0) {
      run_weights(cr0, J);
      run_weights(cr1, J);
#pragma unroll 1
      for (int kk = 0; kk < RS_HR; kk++) {
        const int k = dh * RS_HR + kk;
        if (k >= gr) break;
        if ((bskip >> k) & 1) continue;     // the whole row is done in [C2] or [C]
        const int ri = rg0 + k;
        if (ri >= cr0.next) {
          while (ri >= cr0.next) run_load(cr0, S, J, dc, cr0.m + 1);
          run_weights(cr0, J);
        }
        if (ri >= cr1.next) {
          while (ri >= cr1.next) run_load(cr1, S, J, dc + 1, cr1.m + 1);
          run_weights(cr1, J);
        }
        const int r = r_begin + ri;       // box row
        float2 *orow = J.out + (long)(r - J.row0) * J.out_pitch + c0 + dc;
        const float2 *vrow = &S.vd[k][0];
        const int xb0 = (cr0.key >> 12) - 5 - xw;
        if (cr0.ok && cr1.ok && dval1 && (cr1.key >> 12) == (cr0.key >> 12) + 1) {
          const RsRow R = S.rows[ri];
          const int base = xb0 & ~1;
          const bool odd = (xb0 & 1) != 0;
          float2 V[14];
          const float4 *p = reinterpret_cast<const float4 *>(vrow + base);
#pragma unroll
          for (int m = 0; m < 7; m++) {
            const float4 t = p[m];
            V[2 * m] = make_float2(t.x, t.y);
            V[2 * m + 1] = make_float2(t.z, t.w);
          }
          float2 s0, s1;
          range_pair(cr0, cr1, V, odd, s0, s1);
          const float2 o0 = cmul_conj_turns(s0, run_phase(R, cr0));
          const float2 o1 = cmul_conj_turns(s1, run_phase(R, cr1));
          if (out16) {
            *reinterpret_cast<float4 *>(orow) = make_float4(o0.x, o0.y, o1.x, o1.y);
          } else {
            orow[0] = o0;
            orow[1] = o1;
          }
        } else {
          // per column, from the run key: outside the slave box 0, at its
          // edge the nearest sample, inside the window the tile's range
          // pass, else [C]
          const RsRow R = S.rows[ri];
#pragma unroll
          for (int cc = 0; cc < 2; cc++) {
            if (cc == 1 && !dval1) break;
            const ColRun &cr = cc ? cr1 : cr0;
            const bool dense = cc ? dense1 : dense0;
            const int p0 = cr.key >> 12;
            if (dense) {
              const int e = atomicAdd(&S.gen_d[g], 1);
              S.gen[RS_GR * RS_TW - 1 - e] = (unsigned short)(k * 128 + dc + cc);
            } else if (p0 >= J.sx0 + 5 && p0 <= J.sx1 - 7 && !cr.ok) {
              const int e = atomicAdd(&S.gen_n[g], 1);
              S.gen[e] = (unsigned short)(k * 128 + dc + cc);
            } else if (cr.ok) {
              orow[cc] = cmul_conj_turns(range_single(vrow, p0 - 5 - xw, cr), run_phase(R, cr));
            } else if (p0 < J.sx0 || p0 > J.sx1) {
              orow[cc] = make_float2(0.f, 0.f);
            } else {
              const short2 sv = J.slave[(long)(R.L0 - J.sy0) * J.slave_pitch + (p0 - J.sx0)];
              orow[cc] = make_float2((float)sv.x, (float)sv.y);
            }
          }
        }
      }
    }
    __syncthreads();

    // ---- [C1] pixels of shared rows in columns without a run table, all
    // threads: the range key and its run terms per pixel, then the range
    // pass over the tile as in [B]
    {
      const int nd = S.gen_d[g];
      if (nd > 0) {
        for (int u = tid; u < nd; u += RS_NT) {
          const int code = S.gen[RS_GR * RS_TW - 1 - u];
          const int k = code >> 7, c = code & 127;
          const int r = r_begin + rg0 + k;
          J.out[(long)(r - J.row0) * J.out_pitch + c0 + c] =
              pixel_keyed(S, J, S.rows[rg0 + k], &S.vd[k][0], r, c);
        }
        __syncthreads();
      }
    }

    // ---- [C2] two-bin rows, all threads, by the keyed path: the columns of
    // the first bin from the tile; then the rows' azimuth sums with the
    // second bin, over lines deramped anew from HBM (the line ring already
    // holds the next group's lines), into their tile rows, and the row terms
    // of that key; then the columns of the second bin
    {
      const int two = (S.gwin[g].y >> 4) & 0xfff;
      if (two) {
#pragma unroll 1
        for (int m = two; m; m &= m - 1) {
          const int k = __ffs(m) - 1;
          const int md = S.rows[rg0 + k].mode;
          const int lo = (md >> 8) & 0xff, hi = (md >> 16) & 0xff;
          const int r = r_begin + rg0 + k;
          for (int c = tid; c < cN; c += RS_NT)
            if (c < lo || c >= hi)
              J.out[(long)(r - J.row0) * J.out_pitch + c0 + c] =
                  pixel_keyed(S, J, S.rows[rg0 + k], &S.vd[k][0], r, c);
        }
        __syncthreads();
#pragma unroll 1
        for (int m = two; m; m &= m - 1) {
          const int k = __ffs(m) - 1;
          const RsRow &R = S.rows[rg0 + k];
          S.vd[k][x] = az_direct<kSplit>(S, J, lut, x, xa, xin, R.L0, (R.bin & 0xffff) + 1, 1,
                                         0, g2c, g1c, g0c, cq);
        }
        if (tid < RS_GR && ((two >> tid) & 1)) {
          const RsRow &R = S.rows[rg0 + tid];
          RsRow R2 = R;
          row_terms(S, J, lut, R.L0, (R.bin & 0xffff) + 1, R2);
          S.r2[tid] = R2;
        }
        __syncthreads();
#pragma unroll 1
        for (int m = two; m; m &= m - 1) {
          const int k = __ffs(m) - 1;
          const int md = S.rows[rg0 + k].mode;
          const int r = r_begin + rg0 + k;
          for (int c = ((md >> 8) & 0xff) + tid; c < ((md >> 16) & 0xff); c += RS_NT)
            J.out[(long)(r - J.row0) * J.out_pitch + c0 + c] =
                pixel_keyed(S, J, S.r2[k], &S.vd[k][0], r, c);
        }
        __syncthreads();
      }
    }

    // ---- [C] per-pixel path, all threads: the rows without a shared pass,
    // then the listed pixels
    {
      const int pixmask = S.gwin[g].w & 0xfff;
      const int npr = __popc(pixmask);
      const int nrow_units = npr * cN;
      const int total = nrow_units + S.gen_n[g];
      // the tile is free after [B]: each thread parks its column of the
      // window there while the per-pixel path runs, so the window holds no
      // registers during it
      if (total > 0) {
#pragma unroll
        for (int j = 0; j < RS_GR; j++) S.vd[j][x] = w[j];
      }
      for (int u = tid; u < total; u += RS_NT) {
        int k, c;
        if (u < nrow_units) {
          int nth = u / cN;
          c = u - nth * cN;
          int m = pixmask;
          while (nth-- > 0) m &= m - 1;   // drop the lower set bits
          k = __ffs(m) - 1;
        } else {
          const int code = S.gen[u - nrow_units];
          k = code >> 7;
          c = code & 127;
        }
        const int r = r_begin + rg0 + k;
        J.out[(long)(r - J.row0) * J.out_pitch + c0 + c] = pixel_generic(S, J, r, c);
      }
      if (total > 0) {
#pragma unroll
        for (int j = 0; j < RS_GR; j++) w[j] = S.vd[j][x];
      }
    }
  }
  __syncthreads();   // the next item's prologue rewrites the tables
}

template <bool kSplit>
__global__ void __launch_bounds__(RS_NT, 3)
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
  if (cfg.seg_rows < 0 || cfg.seg_rows > RS_MAXSEG || (cfg.seg_rows && cfg.seg_rows < RS_GR))
    return TOPS_E_INVALID;
  // default segment rows: the longest (least prologue per output row) that
  // still gives every SM two waves of items; small launches (a narrow burst,
  // a single burst) take shorter segments.  Outputs do not depend on it.
  int seg_rows = cfg.seg_rows;
  if (!seg_rows) {
    static const int kSegs[] = {RS_SEG, 168, 120, 84};
    for (int sr : kSegs) {
      long items = 0;
      for (int j = 0; j < njobs; j++)
        items += (long)jobs[j].strips * ((jobs[j].nrows + sr - 1) / sr);
      seg_rows = sr;
      if (items >= 2L * resident) break;
    }
  }
  for (int j0 = 0, k = 0; j0 < njobs; j0 += RS_MAXJOBS, k++) {
    RsBatch B;
    B.njobs = 0;
    B.counter = cfg.counters ? cfg.counters + k : nullptr;
    int items = 0;
    for (int j = j0; j < njobs && j < j0 + RS_MAXJOBS; j++) {
      ResampleJob &J = B.jobs[B.njobs];
      J = jobs[j];
      J.seg_rows = seg_rows;
      J.segs = (J.nrows + seg_rows - 1) / seg_rows;
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

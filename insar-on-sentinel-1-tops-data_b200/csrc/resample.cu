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
// B200 design (no textures, no phase array in HBM):
//   * A CTA owns a strip of RS_TW output columns and sweeps a segment of
//     output rows in groups of RS_GR rows.  Slave rows are deramped once
//     into a ring of RS_FR rows x RS_FW columns in shared memory (complex
//     float + a float phase residual), so the slave is read from HBM about
//     once (the ring keeps the 11-row azimuth halo between groups).
//   * Azimuth-first separable filtering shared across the row: when every
//     interior pixel of a row segment uses the same (azimuth line, LUT bin),
//     v(x) = sum_j kAz[j] d(L0-5+j, x) is computed once per slave column and
//     reused by the 12 range taps of all pixels; the azimuth pass is
//     register-blocked over 4 consecutive rows (15 ring loads serve 4 rows)
//     and uses the packed FP32x2 FMA of sm_100 for the complex samples.
//   * Phase: phi(y,x) = phi_ref(y) + G(y,x), phi_ref the FP64 phase of a
//     reference column, G an FP32 residual of a few radians.  For a column,
//     G is exactly quadratic in azimuth time, so its azimuth interpolation
//     is sum_j kAz[j] G(y_j) = M0 G(L0) + dG/dt(L0) dt M1 + d2G dt^2 M2 with
//     the LUT row moments M0..M2 -- three FMAs instead of twelve taps.  The
//     interpolated phase is (1 + sp1) Psi_row + sum_i kRg[i] gamma(x_i),
//     where Psi_row = sum_j kAz[j] phi_ref(y_j) is FP64 (reduced mod 2 pi)
//     and 1 + sp1 = sum kRg.  This equals the reference's 144-tap FP64 phase
//     sum in exact arithmetic with FP32 only on few-radian quantities.
//   * Rows whose bins are not uniform, or pixels whose support leaves the
//     ring window, take per-pixel paths (from the ring, else from HBM) that
//     compute the same formula.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace tops {

constexpr int RS_NT = 256;   // threads per CTA
constexpr int RS_TW = 112;   // output columns per strip
constexpr int RS_GR = 16;    // output rows per group
constexpr int RS_FR = 32;    // ring rows (power of two)
constexpr int RS_FW = 128;   // ring columns (= threads per half CTA)
constexpr int RS_SEG = 256;  // output rows per work item
constexpr int RS_CPI = 8;    // output columns per range-pass item
constexpr int RS_MAXJOBS = 32;
constexpr int KEY_NONE = 0x7fffffff;

enum : int { REG_OUT = 0, REG_EDGE = 1, REG_IN = 2 };

struct RsLut {
  const float *kaz, *krg;  // [2048][12]
  const float4 *krg2;      // [2048][6]: range taps duplicated (w0,w0,w1,w1), ...
  const float *sp1;        // [2048]: sum(krg row) - 1
};

struct RsBatch {
  int njobs;
  int total_items;
  ResampleJob jobs[RS_MAXJOBS];
};

struct __align__(16) RsShared {
  float2 ring_d[RS_FR][RS_FW];
  float ring_g[RS_FR][RS_FW];
  float2 vd[RS_GR][pad8(RS_FW)];   // indexed with pad8(x)
  float vg[RS_GR][pad8(RS_FW)];
  float4 wpair[RS_GR][6];        // azimuth taps duplicated: (w0,w0,w1,w1), ...
  double ring_phiref[RS_FR];
  double rowA_az[RS_SEG], rowB_az[RS_SEG], rowA_rg[RS_SEG], rowB_rg[RS_SEG];
  int kl0[RS_GR][pad8(RS_TW)];     // indexed with pad8(column)
  int kp0[RS_GR][pad8(RS_TW)];
  int kb[RS_GR][pad8(RS_TW)];      // binL | binP << 12 | region << 24
  // per-row statistics of the group (interior pixels)
  int st_kmin[RS_GR], st_kmax[RS_GR], st_pmin[RS_GR], st_pmax[RS_GR];
  int row_flag[RS_GR];           // 1: shared azimuth pass
  int row_L0[RS_GR], row_xlo[RS_GR], row_xhi[RS_GR];
  float row_M0[RS_GR], row_P1[RS_GR], row_P2[RS_GR];
  float row_rho[RS_GR], row_psif[RS_GR];
  double caz[6], crg[6], shift;
  int xw;                        // absolute slave column of ring column 0
  double ref_a0, ref_a1, ref_a2; // deramp quadratic of the reference column
};

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
__device__ float2 interior_from_ring(const RsShared &S, const RsLut &lut, int L0, int bL, int P0,
                                     int bP) {
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
    psi = fma((double)w, S.ring_phiref[slot], psi);
  }
  float phi = reduce_2pi(psi) + __ldg(lut.sp1 + bP) * (float)psi + sg;
  return cmul_conj_phase(make_float2(sre, sim), phi);
}

__device__ __forceinline__ int warp_min(int v) { return __reduce_min_sync(0xffffffffu, v); }
__device__ __forceinline__ int warp_max(int v) { return __reduce_max_sync(0xffffffffu, v); }

__global__ void __launch_bounds__(RS_NT, 2)
    resample_kernel(const __grid_constant__ RsBatch B, RsLut lut) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsShared &S = *reinterpret_cast<RsShared *>(smem_raw);
  const int tid = threadIdx.x;
  const int ct = tid & (RS_FW - 1);  // column of this thread (key, ring, azimuth passes)
  const int half = tid >> 7;         // 0 / 1

  // ---- locate the work item (job, strip, segment)
  const int item = blockIdx.x;
  if (item >= B.total_items) return;
  int jb = 0;
  while (jb + 1 < B.njobs && B.jobs[jb + 1].item_begin <= item) jb++;
  const ResampleJob &J = B.jobs[jb];
  const int local = item - J.item_begin;
  const int strip = local % J.strips;
  const int seg = local / J.strips;
  const int mpix = J.mx1 - J.mx0 + 1;
  const int c0 = strip * RS_TW;
  const int cN = min(RS_TW, mpix - c0);
  const int r_begin = J.row0 + seg * J.seg_rows;
  const int r_end = min(r_begin + J.seg_rows, J.row0 + J.nrows);

  // ---- per work item setup: polynomials, shift, statistics
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
  if (tid < RS_GR) {
    S.st_kmin[tid] = KEY_NONE;
    S.st_kmax[tid] = -1;
    S.st_pmin[tid] = KEY_NONE;
    S.st_pmax[tid] = -KEY_NONE;
  }
  __syncthreads();
  // per-row polynomial terms: y = A(row) + B(row) P^ + c5 P^2
  {
    const int r = r_begin + tid;
    if (r < r_end) {
      const double L = ((double)(r + J.my0) - J.midL) * J.invL;
      const double *a = S.caz, *g = S.crg;
      S.rowA_az[tid] = a[0] + a[1] * L + a[3] * L * L + S.shift;
      S.rowB_az[tid] = a[2] + a[4] * L;
      S.rowA_rg[tid] = g[0] + g[1] * L + g[3] * L * L;
      S.rowB_rg[tid] = g[2] + g[4] * L;
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
    int lo = (int)floor(pmin) - 5, hi = (int)floor(pmax) + 6;
    int slack = RS_FW - (hi - lo + 1);
    int xw = lo - (slack > 0 ? slack / 2 : 0);
    S.xw = xw;
    int xr = min(max(xw + RS_FW / 2, J.sx0), J.sx1);
    const DerampQuad q = deramp_quad(J.kt[xr], J.tref[xr], J.fdc[xr]);
    S.ref_a0 = q.a0;
    S.ref_a1 = q.a1;
    S.ref_a2 = q.a2;
  }
  __syncthreads();

  // per-thread column constants
  const bool kcol = ct < cN;                         // key column
  const double phat = ((double)(c0 + min(ct, cN - 1)) - J.midP) * J.invP;
  const double q_az = S.caz[5] * phat * phat, q_rg = S.crg[5] * phat * phat;
  const int xabs = S.xw + ct;                        // ring column
  const bool xin = (xabs >= J.sx0 && xabs <= J.sx1);
  DerampQuad colq = {0.0, 0.0, 0.0};
  if (xin) colq = deramp_quad(J.kt[xabs], J.tref[xabs], J.fdc[xabs]);
  const float da2 = (float)(colq.a2 - S.ref_a2), da1 = (float)(colq.a1 - S.ref_a1);
  const DerampQuad refq = {S.ref_a0, S.ref_a1, S.ref_a2};
  int loaded_lo = INT32_MIN, loaded_hi = INT32_MIN;  // valid ring rows (uniform)

  for (int rg = r_begin; rg < r_end; rg += RS_GR) {
    const int gr = min(RS_GR, r_end - rg);
    // ---- [A] indexes, bins and regions; per-row statistics
#pragma unroll 2
    for (int k = 0; k < RS_GR / 2; k++) {
      const int r = half + 2 * k;
      int key = KEY_NONE, kmx = -1, pmn = KEY_NONE, pmx = -KEY_NONE;
      if (r < gr && kcol) {
        const int ri = rg - r_begin + r;
        const double y = fma(S.rowB_az[ri], phat, S.rowA_az[ri] + q_az);
        const double x = fma(S.rowB_rg[ri], phat, S.rowA_rg[ri] + q_rg);
        const int l0 = __double2int_rz(y);
        int bl = __double2int_rz(__dadd_rn(__dmul_rn(y - (double)l0, (double)kInterval), 0.5));
        const int p0 = __double2int_rz(x);
        int bp = __double2int_rz(__dadd_rn(__dmul_rn(x - (double)p0, (double)kInterval), 0.5));
        int reg;
        if (l0 > J.sy1 || l0 < J.sy0 || p0 > J.sx1 || p0 < J.sx0)
          reg = REG_OUT;
        else if (l0 > J.sy1 - 7 || l0 < J.sy0 + 5 || p0 > J.sx1 - 7 || p0 < J.sx0 + 5)
          reg = REG_EDGE;
        else
          reg = REG_IN;
        bl = min(max(bl, 0), kLutBins - 1);  // the reference's texture clamps
        bp = min(max(bp, 0), kLutBins - 1);
        S.kl0[r][pad8(ct)] = l0;
        S.kp0[r][pad8(ct)] = p0;
        S.kb[r][pad8(ct)] = bl | (bp << 12) | (reg << 24);
        if (reg == REG_IN) {
          key = (l0 << 12) | bl;
          kmx = key;
          pmn = pmx = p0;
        }
      }
      if (r < gr) {
        key = warp_min(key);
        kmx = warp_max(kmx);
        pmn = warp_min(pmn);
        pmx = warp_max(pmx);
        if ((tid & 31) == 0 && key != KEY_NONE) {
          atomicMin(&S.st_kmin[r], key);
          atomicMax(&S.st_kmax[r], kmx);
          atomicMin(&S.st_pmin[r], pmn);
          atomicMax(&S.st_pmax[r], pmx);
        }
      }
    }
    __syncthreads();

    // ---- [B] group extent, per-row setup, ring loads
    int lmin = INT32_MAX, lmax = INT32_MIN;
#pragma unroll
    for (int r = 0; r < RS_GR; r++) {
      const int km = S.st_kmin[r];
      if (km != KEY_NONE) {
        lmin = min(lmin, km >> 12);
        lmax = max(lmax, S.st_kmax[r] >> 12);
      }
    }
    const bool ring_ok = (lmax >= lmin) && (lmax - lmin + 12 <= RS_FR);
    if (tid < RS_GR) {
      const int r = tid;
      const int km = S.st_kmin[r];
      int flag = 0;
      if (r < gr && km != KEY_NONE) {
        const int L0 = km >> 12, bL = km & 0xfff;
        const int xlo = S.st_pmin[r] - 5 - S.xw, xhi = S.st_pmax[r] + 6 - S.xw;
        flag = ring_ok && (km == S.st_kmax[r]) && xlo >= 0 && xhi < RS_FW;
        S.row_L0[r] = L0;
        S.row_xlo[r] = xlo;
        S.row_xhi[r] = xhi;
        if (flag) {
          const float *kl = lut.kaz + bL * kTaps;
          float m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll
          for (int j = 0; j < kTaps; j += 2) {
            const float w0 = __ldg(kl + j), w1 = __ldg(kl + j + 1);
            S.wpair[r][j / 2] = make_float4(w0, w0, w1, w1);
            const float u0 = (float)(j - 5), u1 = (float)(j - 4);
            m0 += w0 + w1;
            m1 = fmaf(w0, u0, fmaf(w1, u1, m1));
            m2 = fmaf(w0, u0 * u0, fmaf(w1, u1 * u1, m2));
          }
          const double ta_c = (double)(L0 - J.s_first_line) * J.dt;
          S.row_M0[r] = m0;
          S.row_P1[r] = (float)(2.0 * ta_c * J.dt * m1 + J.dt * J.dt * m2);
          S.row_P2[r] = (float)(J.dt * m1);
        }
      }
      S.row_flag[r] = flag;
    }
    if (ring_ok) {
      const int need_lo = lmin - 5, need_hi = lmax + 6;
      // rows [need_lo, loaded_hi] are already in the ring when the ring holds
      // them contiguously; otherwise (a jump) the whole range is reloaded
      const bool cont = need_lo >= loaded_lo && need_lo <= loaded_hi + 1;
      const int new_lo = cont ? loaded_hi + 1 : need_lo;
      // loads of up to RS_LB rows are issued before any of the math, so the
      // HBM latency of a group's new rows is paid once
      constexpr int RS_LB = 8;
      for (int y0 = new_lo + half; y0 <= need_hi; y0 += 2 * RS_LB) {
        short2 sv[RS_LB];
#pragma unroll
        for (int u = 0; u < RS_LB; u++) {
          const int y = y0 + 2 * u;
          sv[u] = make_short2(0, 0);
          if (y <= need_hi && xin && y >= J.sy0 && y <= J.sy1)
            sv[u] = J.slave[(long)(y - J.sy0) * J.slave_pitch + (xabs - J.sx0)];
        }
#pragma unroll
        for (int u = 0; u < RS_LB; u++) {
          const int y = y0 + 2 * u;
          if (y > need_hi) break;
          const int slot = y & (RS_FR - 1);
          const double ta = (double)(y - J.s_first_line) * J.dt;
          const double phref = quad_eval(refq, ta);
          float2 d = make_float2(0.f, 0.f);
          float g = 0.f;
          if (xin && y >= J.sy0 && y <= J.sy1) {
            const double phi = quad_eval(colq, ta);
            g = (float)(phi - phref);
            float sn, cs;
            __sincosf(reduce_2pi(phi), &sn, &cs);
            d.x = (float)sv[u].x * cs - (float)sv[u].y * sn;
            d.y = (float)sv[u].x * sn + (float)sv[u].y * cs;
          }
          S.ring_d[slot][ct] = d;
          S.ring_g[slot][ct] = g;
          if (ct == 0) S.ring_phiref[slot] = phref;
        }
      }
      if (!cont) loaded_lo = need_lo;
      loaded_hi = max(loaded_hi, need_hi);
      loaded_lo = max(loaded_lo, loaded_hi - RS_FR + 1);
    }
    __syncthreads();

    // ---- [C] shared azimuth pass v(x) and the row phases
    if (tid < RS_GR && S.row_flag[tid]) {
      const int r = tid;
      const int bL = S.st_kmin[r] & 0xfff, L0 = S.row_L0[r];
      const float *kl = lut.kaz + bL * kTaps;
      double psi = 0.0;
#pragma unroll
      for (int j = 0; j < kTaps; j++)
        psi = fma((double)__ldg(kl + j), S.ring_phiref[(L0 - 5 + j) & (RS_FR - 1)], psi);
      S.row_rho[r] = reduce_2pi(psi);
      S.row_psif[r] = (float)psi;
    }
    {
      const int x = ct;
#pragma unroll 1
      for (int qq = 0; qq < 2; qq++) {
        const int q = half + 2 * qq;  // quad of rows 4q..4q+3
        const int r0 = 4 * q;
        if (r0 >= gr) continue;
        bool blk = r0 + 4 <= gr;
        int xl = INT32_MAX, xh = INT32_MIN;
        const int L00 = S.row_L0[r0];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int r = min(r0 + k, RS_GR - 1);
          blk = blk && S.row_flag[r] && S.row_L0[r] == L00 + k;
          xl = min(xl, S.row_xlo[r]);
          xh = max(xh, S.row_xhi[r]);
        }
        if (blk) {
          if (x < xl || x > xh) continue;
          float2 acc[4];
#pragma unroll
          for (int k = 0; k < 4; k++) acc[k] = make_float2(0.f, 0.f);
          const int ybase = L00 - 5;
#pragma unroll
          for (int jj = 0; jj < kTaps + 3; jj++) {
            const float2 d = S.ring_d[(ybase + jj) & (RS_FR - 1)][x];
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const int j = jj - k;
              if (j >= 0 && j < kTaps) {
                const float4 wp = S.wpair[r0 + k][j >> 1];
                const float2 w = (j & 1) ? make_float2(wp.z, wp.w) : make_float2(wp.x, wp.y);
                acc[k] = __ffma2_rn(w, d, acc[k]);
              }
            }
          }
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const int r = r0 + k;
            const float gc = S.ring_g[(L00 + k) & (RS_FR - 1)][x];
            S.vd[r][pad8(x)] = acc[k];
            S.vg[r][pad8(x)] = fmaf(S.row_M0[r], gc, fmaf(da2, S.row_P1[r], da1 * S.row_P2[r]));
          }
        } else {
#pragma unroll 1
          for (int k = 0; k < 4 && r0 + k < gr; k++) {
            const int r = r0 + k;
            if (!S.row_flag[r] || x < S.row_xlo[r] || x > S.row_xhi[r]) continue;
            const int L0 = S.row_L0[r];
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < kTaps; j++) {
              const float4 wp = S.wpair[r][j >> 1];
              const float2 w = (j & 1) ? make_float2(wp.z, wp.w) : make_float2(wp.x, wp.y);
              acc = __ffma2_rn(w, S.ring_d[(L0 - 5 + j) & (RS_FR - 1)][x], acc);
            }
            const float gc = S.ring_g[L0 & (RS_FR - 1)][x];
            S.vd[r][pad8(x)] = acc;
            S.vg[r][pad8(x)] = fmaf(S.row_M0[r], gc, fmaf(da2, S.row_P1[r], da1 * S.row_P2[r]));
          }
        }
      }
    }
    __syncthreads();

    // ---- [D] range pass, reramp, store: RS_CPI consecutive columns per item
    constexpr int NG = RS_TW / RS_CPI;
    for (int it = tid; it < gr * NG; it += RS_NT) {
      const int r = it / NG;
      const int cg = (it - r * NG) * RS_CPI;
      if (cg >= cN) continue;
      const int mr = rg + r;
      float2 *orow = J.out + (long)(mr - J.row0) * J.out_pitch + c0 + cg;
      int kbv[RS_CPI], p0v[RS_CPI];
#pragma unroll
      for (int k = 0; k < RS_CPI; k++) {
        const int c = pad8(min(cg + k, cN - 1));
        kbv[k] = S.kb[r][c];
        p0v[k] = S.kp0[r][c];
      }
      const bool uni = S.row_flag[r];
      bool fast = uni && (cg + RS_CPI <= cN) && ((reinterpret_cast<uintptr_t>(orow) & 15) == 0);
#pragma unroll
      for (int k = 0; k < RS_CPI; k++)
        fast = fast && ((kbv[k] >> 24) == REG_IN) && (p0v[k] == p0v[0] + k);
      if (fast) {
        // 19 shared v loads serve 8 pixels x 12 taps; 16-byte stores
        const int xb = p0v[0] - 5 - S.xw;
        float2 vd[kTaps + RS_CPI - 1];
        float vg[kTaps + RS_CPI - 1];
#pragma unroll
        for (int i = 0; i < kTaps + RS_CPI - 1; i++) {
          vd[i] = S.vd[r][pad8(xb + i)];
          vg[i] = S.vg[r][pad8(xb + i)];
        }
        const float rho = S.row_rho[r], psif = S.row_psif[r];
        float4 *o4 = reinterpret_cast<float4 *>(orow);
#pragma unroll
        for (int k = 0; k < RS_CPI; k += 2) {
          float2 res[2];
#pragma unroll
          for (int u = 0; u < 2; u++) {
            const int bp = (kbv[k + u] >> 12) & 0xfff;
            const float4 *kp4 = lut.krg2 + bp * (kTaps / 2);
            float2 acc = make_float2(0.f, 0.f);
            float sg = 0.f;
#pragma unroll
            for (int q = 0; q < kTaps / 2; q++) {
              const float4 w = __ldg(kp4 + q);
              acc = __ffma2_rn(make_float2(w.x, w.y), vd[k + u + 2 * q], acc);
              acc = __ffma2_rn(make_float2(w.z, w.w), vd[k + u + 2 * q + 1], acc);
              sg = fmaf(w.x, vg[k + u + 2 * q], sg);
              sg = fmaf(w.z, vg[k + u + 2 * q + 1], sg);
            }
            const float phi = rho + __ldg(lut.sp1 + bp) * psif + sg;
            res[u] = cmul_conj_phase(acc, phi);
          }
          o4[k / 2] = make_float4(res[0].x, res[0].y, res[1].x, res[1].y);
        }
      } else {
#pragma unroll 1
        for (int k = 0; k < RS_CPI && cg + k < cN; k++) {
          const int c = pad8(cg + k);
          const int kb = S.kb[r][c], reg = kb >> 24;
          const int l0 = S.kl0[r][c], p0 = S.kp0[r][c];
          float2 res = make_float2(0.f, 0.f);
          if (reg == REG_EDGE) {
            const short2 sv = J.slave[(long)(l0 - J.sy0) * J.slave_pitch + (p0 - J.sx0)];
            res = make_float2((float)sv.x, (float)sv.y);
          } else if (reg == REG_IN) {
            const int bl = kb & 0xfff, bp = (kb >> 12) & 0xfff;
            const int xb = p0 - 5 - S.xw;
            const bool in_win = xb >= 0 && xb + kTaps <= RS_FW;
            if (uni && in_win) {
              const float4 *kp4 = lut.krg2 + bp * (kTaps / 2);
              float2 acc = make_float2(0.f, 0.f);
              float sg = 0.f;
#pragma unroll
              for (int q = 0; q < kTaps / 2; q++) {
                const float4 w = __ldg(kp4 + q);
                acc = __ffma2_rn(make_float2(w.x, w.y), S.vd[r][pad8(xb + 2 * q)], acc);
                acc = __ffma2_rn(make_float2(w.z, w.w), S.vd[r][pad8(xb + 2 * q + 1)], acc);
                sg = fmaf(w.x, S.vg[r][pad8(xb + 2 * q)], sg);
                sg = fmaf(w.z, S.vg[r][pad8(xb + 2 * q + 1)], sg);
              }
              const float phi = S.row_rho[r] + __ldg(lut.sp1 + bp) * S.row_psif[r] + sg;
              res = cmul_conj_phase(acc, phi);
            } else if (ring_ok && in_win) {
              res = interior_from_ring(S, lut, l0, bl, p0, bp);
            } else {
              res = interior_from_global(J, lut, l0, bl, p0, bp);
            }
          }
          orow[k] = res;
        }
      }
    }
    if (tid < RS_GR) {
      S.st_kmin[tid] = KEY_NONE;
      S.st_kmax[tid] = -1;
      S.st_pmin[tid] = KEY_NONE;
      S.st_pmax[tid] = -KEY_NONE;
    }
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

int launch_resample(const LutDev &L, const ResampleJob *jobs, int njobs, cudaStream_t st) {
  static bool attr_done = false;
  if (!attr_done) {
    TOPS_CUDA_TRY(cudaFuncSetAttribute(resample_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(RsShared)));
    attr_done = true;
  }
  RsLut lut{L.kaz, L.krg, L.krg2, L.sp1};
  for (int j0 = 0; j0 < njobs; j0 += RS_MAXJOBS) {
    RsBatch B;
    B.njobs = 0;
    int items = 0;
    for (int j = j0; j < njobs && j < j0 + RS_MAXJOBS; j++) {
      B.jobs[B.njobs] = jobs[j];
      B.jobs[B.njobs].item_begin = items;
      items += jobs[j].strips * jobs[j].segs;
      B.njobs++;
    }
    B.total_items = items;
    if (items == 0) continue;
    resample_kernel<<<items, RS_NT, sizeof(RsShared), st>>>(B, lut);
    TOPS_CUDA_TRY(cudaGetLastError());
  }
  return TOPS_OK;
}

}  // namespace tops

extern "C" int tops_resample(const tops_lut_dev *lut, const tops_resample_job *jobs, int njobs,
                             void *stream) {
  if (!lut || (!jobs && njobs > 0) || njobs < 0) return TOPS_E_INVALID;
  std::vector<ResampleJob> J(njobs);
  for (int j = 0; j < njobs; j++) {
    int st = fill_resample_job(jobs[j], J[j]);
    if (st != TOPS_OK) return st;
  }
  return launch_resample(lut->d, J.data(), njobs, static_cast<cudaStream_t>(stream));
}

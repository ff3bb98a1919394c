// resample.cu -- TOPS deramp + demodulation + 12-point LUT sinc resampling
// + reramp of slave bursts onto the master grid (sm_100a).
//
// Computes exactly the reference algorithm of DerampDemod_Shared
// (DerampAndResample.cu:117-183) followed by Interpolation_12p
// (DerampAndResample.cu:349-520), GetIndexes (:108-112) and my_polyval /
// normalizeWarp (cuConstants.cuh:53-65):
//   position  y = polyAz(L^, P^) + shift,  x = polyRg(L^, P^)
//   index     L0 = trunc(y), bin = int(frac * 2047 + 0.5)  (same for x)
//   regions   outside the slave box -> 0; within 5/7 samples of its edge ->
//             the nearest sample; interior -> separable 12x12 LUT sinc of the
//             deramped slave, reramped with the interpolated deramp phase.
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
//     register-blocked over 4 consecutive rows (15 ring loads for 4 rows).
//   * Phase: phi(y,x) = phi_ref(y) + G(y,x), with phi_ref(y) the FP64 phase
//     of a reference column and G a small FP32 residual (|G| < a few rad).
//     The interpolated phase is S_P * Psi_row + sum kRg*gamma(x), where
//     Psi_row = sum_j kAz[j] phi_ref(y_j) is FP64 per row (reduced mod 2*pi)
//     and S_P = sum kRg = 1 + sp1 per LUT bin.  This equals the reference's
//     144-tap FP64 phase sum in exact arithmetic with FP32 only on
//     few-radian quantities.
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
constexpr int RS_GR = 8;     // output rows per group
constexpr int RS_FR = 32;    // ring rows (power of two)
constexpr int RS_FW = 128;   // ring columns
constexpr int RS_SEG = 256;  // output rows per work item
constexpr int RS_MAXJOBS = 32;

enum : int { REG_OUT = 0, REG_EDGE = 1, REG_IN = 2 };

struct RsLut {
  const float *kaz, *krg;  // [2048][12]
  const float *sp1;        // [2048]: sum(krg row) - 1
};

struct RsBatch {
  int njobs;
  int total_items;
  ResampleJob jobs[RS_MAXJOBS];
};

struct RsTask {
  int kind;      // 4: four-row blocked, 1: single row
  int row;       // first row
  int xlo, n;    // ring-relative first column, count
  int begin;     // first item index
};

struct RsShared {
  float2 ring_d[RS_FR][RS_FW];
  float ring_g[RS_FR][RS_FW];
  double ring_phiref[RS_FR];
  int ring_row[RS_FR];
  float2 vd[RS_GR][RS_FW];
  float vg[RS_GR][RS_FW];
  int kl0[RS_GR][RS_TW];
  int kp0[RS_GR][RS_TW];
  int kb[RS_GR][RS_TW];          // binL | binP << 12 | region << 24
  double phat[RS_TW];            // normalised master column per strip column
  int row_uniform[RS_GR];
  int row_L0[RS_GR], row_bL[RS_GR];
  int row_xlo[RS_GR], row_xhi[RS_GR];   // ring-relative, inclusive
  double row_lhat[RS_GR];         // normalised master line of each row
  double row_psi[RS_GR];
  float row_rho[RS_GR], row_psif[RS_GR];
  RsTask tasks[RS_GR];
  int ntasks, nitems;
  int grp_lmin, grp_lmax, grp_ring_ok;
  int xw;                        // absolute slave column of ring column 0
  double ref_kt, ref_tref, ref_fdc;
  double caz[6], crg[6];         // offset polynomials of this job
  double shift;                  // azimuth shift of this job
};

// Deramp + demodulation phase (DerampAndResample.cu:151-158), FP64.
__device__ __forceinline__ double deramp_phase(double ta, double kt, double tref, double fdc) {
  double e = ta - tref;
  double deramp = -kPi * kt * (e * e);
  double demod = -2.0 * kPi * fdc * ta;
  return deramp + demod;
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

__global__ void __launch_bounds__(RS_NT, 2)
    resample_kernel(const __grid_constant__ RsBatch B, RsLut lut) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RsShared &S = *reinterpret_cast<RsShared *>(smem_raw);
  const int tid = threadIdx.x;

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
  // ---- per-strip setup: coefficients, normalised columns, ring window
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
  for (int c = tid; c < RS_TW; c += RS_NT)
    S.phat[c] = ((double)(c0 + min(c, cN - 1)) - J.midP) * J.invP;
  if (tid < RS_FR) S.ring_row[tid] = INT32_MIN;
  __syncthreads();
  const double shift = S.shift;
  if (tid == 0) {
    // range position at the segment corners and edge midpoints
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
    S.ref_kt = J.kt[xr];
    S.ref_tref = J.tref[xr];
    S.ref_fdc = J.fdc[xr];
  }
  __syncthreads();

  // per-thread ring column (fixed for the work item) and its deramp params
  const int rcol = tid & (RS_FW - 1);
  const int rpar = tid >> 7;  // 0 or 1: which half of the new rows
  const int xabs = S.xw + rcol;
  const bool xin = (xabs >= J.sx0 && xabs <= J.sx1);
  double col_kt = 0, col_tref = 0, col_fdc = 0;
  if (xin) {
    col_kt = J.kt[xabs];
    col_tref = J.tref[xabs];
    col_fdc = J.fdc[xabs];
  }

  for (int rg = r_begin; rg < r_end; rg += RS_GR) {
    const int gr = min(RS_GR, r_end - rg);
    if (tid == 0) {
      S.grp_lmin = INT32_MAX;
      S.grp_lmax = INT32_MIN;
    }
    if (tid < RS_GR) {
      int r = tid;
      double L = ((double)(rg + r + J.my0) - J.midL) * J.invL;
      S.row_lhat[r] = L;
    }
    __syncthreads();

    // ---- phase A: indexes, bins and regions of the group's pixels
    for (int p = tid; p < RS_GR * RS_TW; p += RS_NT) {
      int r = p / RS_TW, c = p - r * RS_TW;
      if (r >= gr || c >= cN) continue;
      double L = S.row_lhat[r];
      double P = S.phat[c];
      const double *ca = S.caz, *cr = S.crg;
      double y = ca[0] + ca[1] * L + ca[2] * P + ca[3] * L * L + ca[4] * L * P + ca[5] * P * P;
      y += shift;
      double x = cr[0] + cr[1] * L + cr[2] * P + cr[3] * L * L + cr[4] * L * P + cr[5] * P * P;
      int l0 = (int)trunc(y);
      int bl = (int)__dadd_rn(__dmul_rn(y - (double)l0, (double)kInterval), 0.5);
      int p0 = (int)trunc(x);
      int bp = (int)__dadd_rn(__dmul_rn(x - (double)p0, (double)kInterval), 0.5);
      int reg;
      if (l0 > J.sy1 || l0 < J.sy0 || p0 > J.sx1 || p0 < J.sx0)
        reg = REG_OUT;
      else if (l0 > J.sy1 - 7 || l0 < J.sy0 + 5 || p0 > J.sx1 - 7 || p0 < J.sx0 + 5)
        reg = REG_EDGE;
      else
        reg = REG_IN;
      bl = min(max(bl, 0), kLutBins - 1);  // the reference's texture clamps
      bp = min(max(bp, 0), kLutBins - 1);
      S.kl0[r][c] = l0;
      S.kp0[r][c] = p0;
      S.kb[r][c] = bl | (bp << 12) | (reg << 24);
      if (reg == REG_IN) {
        atomicMin(&S.grp_lmin, l0);
        atomicMax(&S.grp_lmax, l0);
      }
    }
    __syncthreads();

    // ---- phase A2: row analysis (one warp per row)
    {
      const int w = tid >> 5, lane = tid & 31;
      if (w < RS_GR) {
        int r = w;
        int first = -1;
        int pmin = INT32_MAX, pmax = INT32_MIN;
        int uni = 1;
        int L0 = 0, bL = 0;
        if (r < gr) {
          // first interior pixel of the row (warp-wide)
          for (int c0i = 0; c0i < cN && first < 0; c0i += 32) {
            int c = c0i + lane;
            int in = (c < cN) && ((S.kb[r][c] >> 24) == REG_IN);
            unsigned m = __ballot_sync(0xffffffffu, in);
            if (m) first = c0i + __ffs(m) - 1;
          }
          if (first >= 0) {
            L0 = S.kl0[r][first];
            bL = S.kb[r][first] & 0xfff;
            for (int c = lane; c < cN; c += 32) {
              int kb = S.kb[r][c];
              if ((kb >> 24) != REG_IN) continue;
              if (S.kl0[r][c] != L0 || (kb & 0xfff) != bL) uni = 0;
              pmin = min(pmin, S.kp0[r][c]);
              pmax = max(pmax, S.kp0[r][c]);
            }
          }
          uni = __all_sync(0xffffffffu, uni);
          for (int o = 16; o > 0; o >>= 1) {
            pmin = min(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
            pmax = max(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
          }
        }
        if (lane == 0) {
          int xlo = pmin - 5 - S.xw, xhi = pmax + 6 - S.xw;
          bool ok = (first >= 0) && uni && xlo >= 0 && xhi < RS_FW;
          S.row_uniform[r] = ok ? 1 : 0;
          S.row_L0[r] = L0;
          S.row_bL[r] = bL;
          S.row_xlo[r] = xlo;
          S.row_xhi[r] = xhi;
        }
      }
      if (tid == RS_NT - 1) {
        int lmin = S.grp_lmin, lmax = S.grp_lmax;
        S.grp_ring_ok = (lmax >= lmin) && (lmax - lmin + 12 <= RS_FR);
      }
    }
    __syncthreads();

    // ---- phase B: bring the needed slave rows into the ring (deramped)
    if (S.grp_ring_ok) {
      const int need_lo = S.grp_lmin - 5, need_hi = S.grp_lmax + 6;
      int k = 0;  // index among rows to load
      for (int y = need_lo; y <= need_hi; y++) {
        const int slot = y & (RS_FR - 1);
        if (S.ring_row[slot] == y) continue;  // uniform across the block
        if ((k & 1) == rpar) {
          double ta = (double)(y - J.s_first_line) * J.dt;
          double phref = deramp_phase(ta, S.ref_kt, S.ref_tref, S.ref_fdc);
          float2 d = make_float2(0.f, 0.f);
          float g = 0.f;
          if (xin && y >= J.sy0 && y <= J.sy1) {
            short2 s = J.slave[(long)(y - J.sy0) * J.slave_pitch + (xabs - J.sx0)];
            double phi = deramp_phase(ta, col_kt, col_tref, col_fdc);
            g = (float)(phi - phref);
            float sn, cs;
            __sincosf(reduce_2pi(phi), &sn, &cs);
            d.x = (float)s.x * cs - (float)s.y * sn;
            d.y = (float)s.x * sn + (float)s.y * cs;
          }
          S.ring_d[slot][rcol] = d;
          S.ring_g[slot][rcol] = g;
          if (rcol == 0) S.ring_phiref[slot] = phref;
        }
        k++;
      }
    }
    __syncthreads();
    if (S.grp_ring_ok && tid == 0) {
      for (int y = S.grp_lmin - 5; y <= S.grp_lmax + 6; y++) S.ring_row[y & (RS_FR - 1)] = y;
    }

    // ---- phase C0: task list for the shared azimuth pass + row phases
    if (tid == 0) {
      int nt = 0, ni = 0;
      for (int sub = 0; sub < RS_GR; sub += 4) {
        bool block4 = S.grp_ring_ok && sub + 4 <= gr;
        int xlo = INT32_MAX, xhi = INT32_MIN;
        if (block4) {
          for (int k = 0; k < 4; k++) {
            int r = sub + k;
            if (!S.row_uniform[r] || S.row_L0[r] != S.row_L0[sub] + k) block4 = false;
            xlo = min(xlo, S.row_xlo[r]);
            xhi = max(xhi, S.row_xhi[r]);
          }
        }
        if (block4) {
          S.tasks[nt] = RsTask{4, sub, xlo, xhi - xlo + 1, ni};
          ni += xhi - xlo + 1;
          nt++;
        } else if (S.grp_ring_ok) {
          for (int k = 0; k < 4 && sub + k < gr; k++) {
            int r = sub + k;
            if (!S.row_uniform[r]) continue;
            int n = S.row_xhi[r] - S.row_xlo[r] + 1;
            S.tasks[nt] = RsTask{1, r, S.row_xlo[r], n, ni};
            ni += n;
            nt++;
          }
        }
      }
      S.ntasks = nt;
      S.nitems = ni;
    }
    if (tid < gr && S.grp_ring_ok && S.row_uniform[tid]) {
      const int r = tid;
      const float *kl = lut.kaz + S.row_bL[r] * kTaps;
      double psi = 0.0;
      for (int j = 0; j < kTaps; j++)
        psi = fma((double)__ldg(kl + j), S.ring_phiref[(S.row_L0[r] - 5 + j) & (RS_FR - 1)], psi);
      S.row_psi[r] = psi;
      S.row_rho[r] = reduce_2pi(psi);
      S.row_psif[r] = (float)psi;
    }
    __syncthreads();

    // ---- phase C: azimuth pass v(x) = sum_j kAz[j] (d, G)(L0-5+j, x)
    for (int it = tid; it < S.nitems; it += RS_NT) {
      int t = 0;
      while (t + 1 < S.ntasks && S.tasks[t + 1].begin <= it) t++;
      const RsTask T = S.tasks[t];
      const int x = T.xlo + (it - T.begin);
      if (T.kind == 4) {
        float w[4][kTaps];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const float *kl = lut.kaz + S.row_bL[T.row + k] * kTaps;
#pragma unroll
          for (int j = 0; j < kTaps; j++) w[k][j] = __ldg(kl + j);
        }
        float ar[4] = {0.f, 0.f, 0.f, 0.f}, ai[4] = {0.f, 0.f, 0.f, 0.f},
              ag[4] = {0.f, 0.f, 0.f, 0.f};
        const int ybase = S.row_L0[T.row] - 5;
#pragma unroll
        for (int jj = 0; jj < kTaps + 3; jj++) {
          const int slot = (ybase + jj) & (RS_FR - 1);
          const float2 d = S.ring_d[slot][x];
          const float g = S.ring_g[slot][x];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const int j = jj - k;
            if (j >= 0 && j < kTaps) {
              ar[k] = fmaf(w[k][j], d.x, ar[k]);
              ai[k] = fmaf(w[k][j], d.y, ai[k]);
              ag[k] = fmaf(w[k][j], g, ag[k]);
            }
          }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
          S.vd[T.row + k][x] = make_float2(ar[k], ai[k]);
          S.vg[T.row + k][x] = ag[k];
        }
      } else {
        const float *kl = lut.kaz + S.row_bL[T.row] * kTaps;
        const int ybase = S.row_L0[T.row] - 5;
        float ar = 0.f, ai = 0.f, ag = 0.f;
#pragma unroll
        for (int j = 0; j < kTaps; j++) {
          const int slot = (ybase + j) & (RS_FR - 1);
          const float w = __ldg(kl + j);
          const float2 d = S.ring_d[slot][x];
          ar = fmaf(w, d.x, ar);
          ai = fmaf(w, d.y, ai);
          ag = fmaf(w, S.ring_g[slot][x], ag);
        }
        S.vd[T.row][x] = make_float2(ar, ai);
        S.vg[T.row][x] = ag;
      }
    }
    __syncthreads();

    // ---- phase D: range pass, reramp, store (4 consecutive columns/item)
    const int ngrp = (cN + 3) >> 2;
    for (int it = tid; it < gr * ngrp; it += RS_NT) {
      const int r = it / ngrp;
      const int cg = (it - r * ngrp) << 2;
      const int mr = rg + r;  // master row (0-based in box)
      float2 res[4];
      int kbv[4], p0v[4], l0v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int c = min(cg + k, cN - 1);
        kbv[k] = S.kb[r][c];
        p0v[k] = S.kp0[r][c];
        l0v[k] = S.kl0[r][c];
      }
      const bool uni = S.grp_ring_ok && S.row_uniform[r];
      bool fast = uni;
#pragma unroll
      for (int k = 0; k < 4; k++)
        fast = fast && ((kbv[k] >> 24) == REG_IN) && (p0v[k] == p0v[0] + k) && (cg + k < cN);
      if (fast) {
        // 15 shared v loads serve 4 pixels x 12 taps
        const int xb = p0v[0] - 5 - S.xw;
        float2 vd[kTaps + 3];
        float vg[kTaps + 3];
#pragma unroll
        for (int i = 0; i < kTaps + 3; i++) {
          vd[i] = S.vd[r][xb + i];
          vg[i] = S.vg[r][xb + i];
        }
        const float rho = S.row_rho[r], psif = S.row_psif[r];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const int bp = (kbv[k] >> 12) & 0xfff;
          const float4 *kp4 = reinterpret_cast<const float4 *>(lut.krg + bp * kTaps);
          float kp[kTaps];
#pragma unroll
          for (int q = 0; q < 3; q++) {
            float4 t4 = __ldg(kp4 + q);
            kp[4 * q] = t4.x;
            kp[4 * q + 1] = t4.y;
            kp[4 * q + 2] = t4.z;
            kp[4 * q + 3] = t4.w;
          }
          float sre = 0.f, sim = 0.f, sg = 0.f;
#pragma unroll
          for (int i = 0; i < kTaps; i++) {
            sre = fmaf(kp[i], vd[k + i].x, sre);
            sim = fmaf(kp[i], vd[k + i].y, sim);
            sg = fmaf(kp[i], vg[k + i], sg);
          }
          const float phi = rho + __ldg(lut.sp1 + bp) * psif + sg;
          res[k] = cmul_conj_phase(make_float2(sre, sim), phi);
        }
      } else {
#pragma unroll 1
        for (int k = 0; k < 4; k++) {
          res[k] = make_float2(0.f, 0.f);
          if (cg + k >= cN) continue;
          const int reg = kbv[k] >> 24;
          const int l0 = l0v[k], p0 = p0v[k];
          if (reg == REG_EDGE) {
            short2 s = J.slave[(long)(l0 - J.sy0) * J.slave_pitch + (p0 - J.sx0)];
            res[k] = make_float2((float)s.x, (float)s.y);
          } else if (reg == REG_IN) {
            const int bl = kbv[k] & 0xfff, bp = (kbv[k] >> 12) & 0xfff;
            const int xb = p0 - 5 - S.xw;
            const bool in_ring = S.grp_ring_ok && xb >= 0 && xb + kTaps <= RS_FW;
            if (uni && in_ring) {
              const float4 *kp4 = reinterpret_cast<const float4 *>(lut.krg + bp * kTaps);
              float sre = 0.f, sim = 0.f, sg = 0.f;
#pragma unroll
              for (int q = 0; q < 3; q++) {
                float4 t4 = __ldg(kp4 + q);
                float kq[4] = {t4.x, t4.y, t4.z, t4.w};
#pragma unroll
                for (int u = 0; u < 4; u++) {
                  const float2 v = S.vd[r][xb + 4 * q + u];
                  sre = fmaf(kq[u], v.x, sre);
                  sim = fmaf(kq[u], v.y, sim);
                  sg = fmaf(kq[u], S.vg[r][xb + 4 * q + u], sg);
                }
              }
              const float phi = S.row_rho[r] + __ldg(lut.sp1 + bp) * S.row_psif[r] + sg;
              res[k] = cmul_conj_phase(make_float2(sre, sim), phi);
            } else if (in_ring) {
              res[k] = interior_from_ring(S, lut, l0, bl, p0, bp);
            } else {
              res[k] = interior_from_global(J, lut, l0, bl, p0, bp);
            }
          }
        }
      }
      // store: vectorised when the 4 outputs are in the strip and aligned
      float2 *orow = J.out + (long)(mr - J.row0) * J.out_pitch + c0 + cg;
      if (cg + 4 <= cN && ((reinterpret_cast<uintptr_t>(orow) & 15) == 0)) {
        float4 *o4 = reinterpret_cast<float4 *>(orow);
        o4[0] = make_float4(res[0].x, res[0].y, res[1].x, res[1].y);
        o4[1] = make_float4(res[2].x, res[2].y, res[3].x, res[3].y);
      } else {
        for (int k = 0; k < 4 && cg + k < cN; k++) orow[k] = res[k];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host
struct LutDev {
  float *kaz = nullptr, *krg = nullptr, *sp1 = nullptr;
};

}  // namespace tops

struct tops_lut_dev {
  tops::LutDev d;
};

using namespace tops;

extern "C" int tops_lut_create(const float *kaz, const float *krg, tops_lut_dev **out) {
  if (!kaz || !krg || !out) return TOPS_E_INVALID;
  tops_lut_dev *L = new tops_lut_dev();
  std::vector<float> sp1(kLutBins);
  for (int b = 0; b < kLutBins; b++) {
    double s = 0.0;
    for (int i = 0; i < kTaps; i++) s += (double)krg[b * kTaps + i];
    sp1[b] = (float)(s - 1.0);
  }
  size_t nb = sizeof(float) * kLutBins * kTaps;
  cudaError_t e = cudaMalloc(&L->d.kaz, nb);
  if (e == cudaSuccess) e = cudaMalloc(&L->d.krg, nb);
  if (e == cudaSuccess) e = cudaMalloc(&L->d.sp1, sizeof(float) * kLutBins);
  if (e == cudaSuccess) e = cudaMemcpy(L->d.kaz, kaz, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(L->d.krg, krg, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(L->d.sp1, sp1.data(), sizeof(float) * kLutBins, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    set_cuda_error(e);
    cudaFree(L->d.kaz);
    cudaFree(L->d.krg);
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
  RsLut lut{L.kaz, L.krg, L.sp1};
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

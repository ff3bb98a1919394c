// coherence.cu -- windowed interferometric coherence (sm_100a).
//
// Reference: CohMatSet (EstCoh.cu:101-139) builds m*conj(s) and
// (|s|^2, |m|^2) in padded arrays; Cohbasic (EstCoh.cu:413-456) and the
// prefix-sum chain of CoherenceEst_ESD (EstCoh.cu:152-411) sum them over the
// box rows r-dy..r-dy+winAz-1, cols c-dx..c-dx+winRg-1 and output
//   gamma = |sum m s*| / sqrt(sum|s|^2 * sum|m|^2)   (0 if the product is 0)
// with gamma = 0 where |s(r,c)| < 0.001.  The reference leaves the pad
// uninitialised (EstCoh.cu:581-583); here it is zero.
//
// B200 design: one CTA per (strip of CO_TW columns, segment of rows).  Each
// thread owns one loaded column and walks the segment in groups of CO_GR
// rows.  For the common azimuth windows (template WAZ = 3 and the
// reference's 6) the products (m s*, |s|^2, |m|^2) of the last WAZ - 1 input
// rows stay in registers from one group to the next, so every input row is
// read once, and the loads of the next group are issued before the
// horizontal pass of the current one, so HBM latency overlaps the shared-
// memory work.  The vertical sums go to shared memory; the horizontal box is
// a sliding sum over CO_CPI consecutive outputs per thread, written with
// 16-byte stores.  Other window heights (WAZ = 0) reload the halo rows of
// each group.  HBM traffic is the algorithmic 4 + 8 + 4 bytes per pixel plus
// the column halo.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "launch.h"

namespace tops {

constexpr int CO_NT = 256;
constexpr int CO_TW = 224;   // output columns per strip (win_rg <= 33)
constexpr int CO_GR = 8;     // rows per group
constexpr int CO_SEG = 128;  // rows per work item
constexpr int CO_CPI = 8;    // output columns per horizontal item
constexpr int CO_MAXJOBS = 32;
constexpr int CO_MAX_WIN_RG = CO_NT - CO_TW + 1;

struct CoBatch {
  int njobs, total_items, win_rg, win_az;
  int compensated;         // 1: each output's window summed pairwise
  int *counter;            // persistent launch: work-item queue (else null)
  CohJob jobs[CO_MAXJOBS];
};

struct CoShared {
  float4 V[CO_GR][pad8(CO_NT)];      // vertical sums (re, im, |s|^2, |m|^2), pad8(x)
  float spow[CO_GR][pad8(CO_NT)];   // |s|^2 of the centre pixel, pad8(x)
  int next_item;                     // persistent launch: the item just taken
};

__device__ __forceinline__ float4 coh_product(short2 m, float2 s) {
  const float mr = m.x, mi = m.y;
  return make_float4(mr * s.x + mi * s.y,   // m * conj(s)
                     mi * s.x - mr * s.y, s.x * s.x + s.y * s.y, mr * mr + mi * mi);
}

// a += b with packed FP32x2 adds
__device__ __forceinline__ void add4(float4 &a, const float4 &b) {
  const float2 c = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  const float2 p = __fadd2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w));
  a = make_float4(c.x, c.y, p.x, p.y);
}

// Pairwise sum of n window columns V[idx(0)] .. V[idx(n - 1)] (the
// compensated mode: no sliding update, rounding error O(log n)).
template <class Idx>
__device__ __forceinline__ float4 window_pairwise(const float4 *V, int n, Idx idx) {
  float4 p[16];
  int m = 0;
  for (int i = 0; i + 1 < n; i += 2, m++) {
    p[m] = V[idx(i)];
    add4(p[m], V[idx(i + 1)]);
  }
  if (n & 1) p[m++] = V[idx(n - 1)];
  for (int h = 1; h < m; h <<= 1)
    for (int i = 0; i + h < m; i += 2 * h) add4(p[i], p[i + h]);
  return p[0];
}

// Horizontal pass of one group: CO_CPI consecutive outputs per item.  The
// amplitude mask |s| < 0.001 of the reference (EstCoh.cu:393, 446) is
// evaluated as |s|^2 < 1e-6.  WRG > 0: range window known at compile time;
// an item starts at a multiple of 8 columns, so pad8(cg + i) = pad8(cg) +
// pad8(i) and every shared-memory offset below is a constant.
template <int WRG, bool COMP>
__device__ __forceinline__ void coh_horizontal(const CoShared &S, const CohJob &J, int tid,
                                               int rg, int gr, int c0, int cN, int win_rg_rt,
                                               int dx_rt) {
  constexpr int NG = CO_TW / CO_CPI;
  static_assert(CO_CPI % 8 == 0, "items must start at multiples of 8 columns");
  const int win_rg = WRG > 0 ? WRG : win_rg_rt;
  const int dx = WRG > 0 ? (WRG - 1) / 2 : dx_rt;
  for (int it = tid; it < gr * NG; it += CO_NT) {
    const int k = it / NG;
    const int cg = (it - k * NG) * CO_CPI;
    if (cg >= cN) continue;
    const float4 *V = &S.V[k][pad8(cg)];
    const float *Jd = &S.spow[k][pad8(cg)];
    float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
    if (WRG > 0) {
#pragma unroll
      for (int i = 0; i < WRG; i++) add4(w, V[pad8(i)]);
    } else {
      for (int i = 0; i < win_rg; i++) add4(w, V[pad8(i)]);
    }
    float out[CO_CPI];
#pragma unroll
    for (int u = 0; u < CO_CPI; u++) {
      if (COMP) {
        w = window_pairwise(V, win_rg, [&](int i) { return pad8(u + i); });
      } else if (u > 0) {
        const float4 a = V[pad8(u - 1 + win_rg)];
        const float4 b = V[pad8(u - 1)];
        const float2 m1 = make_float2(-1.f, -1.f);
        const float2 wc = __fadd2_rn(make_float2(w.x, w.y),
                                     __ffma2_rn(make_float2(b.x, b.y), m1, make_float2(a.x, a.y)));
        const float2 wp = __fadd2_rn(make_float2(w.z, w.w),
                                     __ffma2_rn(make_float2(b.z, b.w), m1, make_float2(a.z, a.w)));
        w = make_float4(wc.x, wc.y, wp.x, wp.y);
      }
      // |sum m s*| / sqrt(sum |s|^2 sum |m|^2) as num rsqrt(num) rsqrt(p):
      // two MUFU reciprocal square roots instead of an IEEE square root
      // (relative error a few 1e-7)
      const float p = w.z * w.w;
      const float num = fmaf(w.x, w.x, w.y * w.y);
      float g = (p > 0.f && num > 0.f) ? num * rsqrtf(num) * rsqrtf(p) : 0.f;
      if (Jd[pad8(u + dx)] < 1e-6f) g = 0.f;
      out[u] = g;
    }
    float *orow = J.coh + (long)(rg + k) * J.coh_pitch + c0 + cg;
    if (cg + CO_CPI <= cN && ((reinterpret_cast<uintptr_t>(orow) & 15) == 0)) {
#pragma unroll
      for (int u = 0; u < CO_CPI; u += 4)
        *reinterpret_cast<float4 *>(orow + u) = make_float4(out[u], out[u + 1], out[u + 2],
                                                            out[u + 3]);
    } else {
#pragma unroll
      for (int u = 0; u < CO_CPI; u++)
        if (cg + u < cN) orow[u] = out[u];
    }
  }
}

// One work item (strip x segment of one job); all threads of the CTA call it
// with the same item.
template <int WAZ, int WRG, bool COMP>
__device__ __forceinline__ void coherence_item(CoShared &S, const CoBatch &B, int item) {
  const int tid = threadIdx.x;
  int jb = 0;
  while (jb + 1 < B.njobs && B.jobs[jb + 1].item_begin <= item) jb++;
  const CohJob &J = B.jobs[jb];
  const int local = item - J.item_begin;
  const int strip = local % J.strips, seg = local / J.strips;
  const int win_rg = B.win_rg;
  const int win_az = WAZ > 0 ? WAZ : B.win_az;
  const int dx = (win_rg - 1) / 2, dy = (win_az - 1) / 2;
  const int c0 = strip * CO_TW;
  const int cN = min(CO_TW, J.pixels - c0);
  const int nload = cN + win_rg - 1;
  const int r_begin = seg * J.seg_rows;
  const int r_end = min(r_begin + J.seg_rows, J.lines);
  const int x = c0 - dx + tid;          // this thread's loaded column
  const bool xin = tid < nload && x >= 0 && x < J.pixels;
  auto load = [&](int y, short2 &m, float2 &s) {
    m = make_short2(0, 0);
    s = make_float2(0.f, 0.f);
    if (xin && y >= 0 && y < J.lines) {
      m = J.master[(long)y * J.master_pitch + x];
      s = J.slave[(long)y * J.slave_pitch + x];
    }
  };

  if constexpr (WAZ > 0) {
    // products of input rows: q[0 .. WAZ-2] carried, then the group's rows
    constexpr int NQ = WAZ > 0 ? WAZ - 1 : 1;
    float4 q[NQ];
    {
      // rows r_begin - dy .. r_begin - dy + WAZ - 2 (the first group's halo)
#pragma unroll
      for (int j = 0; j < NQ; j++) {
        short2 m;
        float2 s;
        load(r_begin - dy + j, m, s);
        q[j] = coh_product(m, s);
      }
    }
    // loads of the first group: input rows r_begin - dy + WAZ - 1 + k
    short2 mv[CO_GR];
    float2 sv[CO_GR];
#pragma unroll
    for (int k = 0; k < CO_GR; k++) load(r_begin - dy + WAZ - 1 + k, mv[k], sv[k]);
    for (int rg = r_begin; rg < r_end; rg += CO_GR) {
      const int gr = min(CO_GR, r_end - rg);
      float4 p[NQ + CO_GR];
#pragma unroll
      for (int j = 0; j < NQ; j++) p[j] = q[j];
#pragma unroll
      for (int k = 0; k < CO_GR; k++) p[NQ + k] = coh_product(mv[k], sv[k]);
      // issue the next group's loads now; they land during the rest
      const int rn = rg + CO_GR;
      if (rn < r_end) {
#pragma unroll
        for (int k = 0; k < CO_GR; k++) load(rn - dy + WAZ - 1 + k, mv[k], sv[k]);
      }
#pragma unroll
      for (int k = 0; k < CO_GR; k++) {
        float4 a = p[k];
#pragma unroll
        for (int j = 1; j < WAZ; j++) add4(a, p[k + j]);
        S.V[k][pad8(tid)] = a;
        S.spow[k][pad8(tid)] = p[k + dy].z;
      }
#pragma unroll
      for (int j = 0; j < NQ; j++) q[j] = p[CO_GR + j];
      __syncthreads();
      coh_horizontal<WRG, COMP>(S, J, tid, rg, gr, c0, cN, win_rg, dx);
      __syncthreads();
    }
  } else {
    for (int rg = r_begin; rg < r_end; rg += CO_GR) {
      const int gr = min(CO_GR, r_end - rg);
      // vertical pass: input rows rg-dy .. rg-dy+gr+win_az-2
      float4 acc[CO_GR];
      float spow[CO_GR];
#pragma unroll
      for (int k = 0; k < CO_GR; k++) {
        acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        spow[k] = 0.f;
      }
      const int nin = gr + win_az - 1;
      for (int qi = 0; qi < nin; qi++) {
        short2 m;
        float2 sl;
        load(rg - dy + qi, m, sl);
        const float4 pr = coh_product(m, sl);
#pragma unroll
        for (int k = 0; k < CO_GR; k++) {
          const int j = qi - k;
          if (j >= 0 && j < win_az) add4(acc[k], pr);
          if (qi == k + dy) spow[k] = pr.z;
        }
      }
#pragma unroll
      for (int k = 0; k < CO_GR; k++) {
        S.V[k][pad8(tid)] = acc[k];
        S.spow[k][pad8(tid)] = spow[k];
      }
      __syncthreads();
      coh_horizontal<WRG, COMP>(S, J, tid, rg, gr, c0, cN, win_rg, dx);
      __syncthreads();
    }
  }
}

// COMP: the compensated window sums (a separate instantiation, so the plain
// kernels carry none of its code or registers)
template <int WAZ, int WRG, bool COMP>
__global__ void __launch_bounds__(CO_NT, 3) coherence_kernel(const __grid_constant__ CoBatch B) {
  __shared__ CoShared S;
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
    coherence_item<WAZ, WRG, COMP>(S, B, item);
    if (!B.counter) break;
    if (threadIdx.x == 0) S.next_item = atomicAdd(B.counter, 1);
    __syncthreads();
    item = S.next_item;
    __syncthreads();
  }
}

// ------------------------------------------------ TMA-staged variant
// For the pipeline's 10-sample and the reference driver's 24-sample range
// windows.  A CTA of CT_NT threads owns a strip of TW output columns and a
// segment of rows; its input rows come in chunks of CT_CH rows x CT_LW
// columns (master as 32-bit, slave as 64-bit elements), each chunk one
// cp.async.bulk.tensor box per image on an mbarrier, CT_NST - 1 chunks ahead
// of the one being summed.  The box starts XOFF columns left of the strip:
// dx rounded up to a multiple of 4, so every box's x coordinate is 16-byte
// aligned in both images; the copy engine fills rows and columns outside the
// image with zeros -- the zero pad.  The
// vertical sums are those of coherence_item; the horizontal sliding sum
// restarts every CT_CPI = 4 outputs instead of every CO_CPI = 8 (measured
// faster: 0.398 against 0.490 ms for 3 bursts of 1500 x 21000), so the two
// kernels agree to FP32 rounding of the window sums (a few 1e-7).
constexpr int CT_NT = 256;
constexpr int CT_LW = 256;                 // loaded columns (box width)
constexpr int CT_CH = 4;                   // rows per chunk (box height)
constexpr int CT_NST = 4;                  // chunk slots
constexpr int CT_CPI = 4;                  // outputs per horizontal item
constexpr int CT_SEG = 256;                // rows per work item
constexpr int CT_MAXJOBS = 16;
constexpr unsigned long long CT_WAIT_NS = 2000000000ull;   // a chunk is given up after 2 s
// Geometry of a range window of WRG samples: the box starts XOFF columns
// left of the strip, the window of the strip's first output starts B0
// columns into the box, and a strip has TW outputs.
template <int WRG>
struct CtWin {
  static constexpr int DX = (WRG - 1) / 2;
  static constexpr int XOFF = (DX + 3) & ~3;
  static constexpr int B0 = XOFF - DX;
  static constexpr int TW = WRG == 10 ? 240 : ((CT_LW - XOFF - (WRG - 1 - DX)) & ~(CT_CPI - 1));
  static_assert(XOFF % 4 == 0, "box x coordinates stay 16-byte aligned");
  static_assert(XOFF + TW + WRG - 1 - DX <= CT_LW, "the strip's boxes cover its windows");
  static_assert(TW % CT_CPI == 0 && CT_CH * (TW / CT_CPI) <= CT_NT, "one horizontal item per thread");
};

__host__ __device__ constexpr int pad4(int x) { return x + (x >> 2); }

struct __align__(64) CtBatch {
  CUtensorMap tm_m[CT_MAXJOBS];   // master: int32 [lines][pixels], box CT_LW x CT_CH
  CUtensorMap tm_s[CT_MAXJOBS];   // slave: 64-bit [lines][pixels], same box
  CohJob jobs[CT_MAXJOBS];
  int njobs, total_items;
  int compensated;                // 1: each output's window summed pairwise
  int *counter;                   // persistent launch: work-item queue (else null)
};

struct __align__(128) CtShared {
  int m[CT_NST][CT_CH][CT_LW];          // master chunks (CInt16 pairs)
  float2 s[CT_NST][CT_CH][CT_LW];       // slave chunks
  float4 V[CT_CH][pad4(CT_LW)];         // vertical sums (re, im, |s|^2, |m|^2)
  float spow[CT_CH][pad4(CT_LW)];       // |s|^2 of the centre pixel
  unsigned long long full[CT_NST];      // one mbarrier per slot
  int next_item;
};

__device__ int g_coh_wait_faults;       // chunks whose wait ran out (0 normally)

__device__ __forceinline__ unsigned ct_smem(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void ct_mbar_init(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ct_smem(bar)) : "memory");
}
__device__ __forceinline__ void ct_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ct_smem(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool ct_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(ct_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void ct_tma_2d(void *dst, const CUtensorMap *tm, int x, int y,
                                          unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(ct_smem(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(ct_smem(bar))
      : "memory");
}
__device__ __forceinline__ unsigned long long ct_now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the slot's chunk for at most CT_WAIT_NS of wall time (the
// bound is on time, not on polls: a poll may suspend the thread); false if
// it never arrived (recorded in g_coh_wait_faults).
__device__ __forceinline__ bool ct_wait(unsigned long long *bar, unsigned parity) {
  if (ct_try_wait(bar, parity)) return true;
  const unsigned long long t0 = ct_now_ns();
  do {
    if (ct_try_wait(bar, parity)) return true;
  } while (ct_now_ns() - t0 < CT_WAIT_NS);
  return false;
}

// One work item; returns false (all threads) when a chunk never arrived.
// `seq` counts the chunks this CTA has consumed (slot and mbarrier phase).
template <int WAZ, int WRG, bool COMP>
__device__ __forceinline__ bool coh_tma_item(CtShared &S, const CtBatch &B, int item,
                                             unsigned &seq) {
  using Win = CtWin<WRG>;
  constexpr int DY = (WAZ - 1) / 2;
  constexpr int NQ = WAZ - 1;
  constexpr int H = (NQ + CT_CH - 1) / CT_CH;   // chunks holding the first halo rows
  constexpr unsigned kChunkBytes = CT_CH * CT_LW * (4 + 8);
  const int tid = threadIdx.x;
  int jb = 0;
  while (jb + 1 < B.njobs && B.jobs[jb + 1].item_begin <= item) jb++;
  const CohJob &J = B.jobs[jb];
  const int local = item - J.item_begin;
  const int strip = local % J.strips, seg = local / J.strips;
  const int c0 = strip * Win::TW;
  const int cN = min(Win::TW, J.pixels - c0);
  const int r_begin = seg * J.seg_rows;
  const int r_end = min(r_begin + J.seg_rows, J.lines);
  const int nout = (r_end - r_begin + CT_CH - 1) / CT_CH;
  const int T = H + nout;
  const int x0 = c0 - Win::XOFF;
  // chunk u holds input rows base(u) .. base(u) + CT_CH - 1: output chunk
  // u - H's new rows, the halo rows r_begin - DY .. r_begin - DY + NQ - 1
  // at the end of the first H chunks
  auto base = [&](int u) { return r_begin + CT_CH * (u - H) + (NQ - DY); };
  auto issue = [&](int u) {
    const unsigned slot = (seq + u) % CT_NST;
    ct_expect_tx(&S.full[slot], kChunkBytes);
    ct_tma_2d(&S.m[slot][0][0], &B.tm_m[jb], x0, base(u), &S.full[slot]);
    ct_tma_2d(&S.s[slot][0][0], &B.tm_s[jb], x0, base(u), &S.full[slot]);
  };
  if (tid == 0)
    for (int u = 0; u < CT_NST - 1 && u < T; u++) issue(u);

  float4 q[NQ > 0 ? NQ : 1];
#pragma unroll
  for (int j = 0; j < NQ; j++) q[j] = make_float4(0.f, 0.f, 0.f, 0.f);
  const int t = tid;                       // loaded column
  bool ok = true;
  for (int u = 0; u < T; u++) {
    const unsigned slot = (seq + u) % CT_NST;
    const unsigned parity = ((seq + u) / CT_NST) & 1u;
    const bool got = ct_wait(&S.full[slot], parity);
    if (__syncthreads_or(!got)) {
      ok = false;
      if (tid == 0) {
        atomicAdd(&g_coh_wait_faults, 1);
        // let the copies in flight land (bounded) before the CTA moves on
        for (int v = u; v < T && v < u + CT_NST - 1; v++)
          (void)ct_wait(&S.full[(seq + v) % CT_NST], ((seq + v) / CT_NST) & 1u);
      }
      __syncthreads();
      break;
    }
    // the next chunk into the slot freed by the previous one
    if (tid == 0 && u + CT_NST - 1 < T) issue(u + CT_NST - 1);
    if (u < H) {
      // halo rows: products of input rows r_begin - DY + i
#pragma unroll
      for (int hu = 0; hu < H; hu++) {
        if (u == hu) {
#pragma unroll
          for (int k = 0; k < CT_CH; k++) {
            const int i = CT_CH * (hu - H) + NQ + k;
            if (i >= 0 && i < NQ) {
              const int mv = S.m[slot][k][t];
              q[i] = coh_product(*reinterpret_cast<const short2 *>(&mv), S.s[slot][k][t]);
            }
          }
        }
      }
      continue;
    }
    // vertical sums of the chunk's output rows (as coherence_item sums them)
#pragma unroll
    for (int k = 0; k < CT_CH; k++) {
      const int mv = S.m[slot][k][t];
      const float4 p = coh_product(*reinterpret_cast<const short2 *>(&mv), S.s[slot][k][t]);
      float4 a = NQ > 0 ? q[0] : p;
#pragma unroll
      for (int j = 1; j < NQ; j++) add4(a, q[j]);
      if (NQ > 0) add4(a, p);
      S.V[k][pad4(t)] = a;
      S.spow[k][pad4(t)] = (DY < NQ) ? q[DY < NQ ? DY : 0].z : p.z;
#pragma unroll
      for (int j = 0; j + 1 < NQ; j++) q[j] = q[j + 1];
      if (NQ > 0) q[NQ - 1] = p;
    }
    __syncthreads();
    // horizontal box: CT_CPI consecutive outputs per item; an item starts at
    // a multiple of 4 columns, so every padded offset below is a constant
    {
      constexpr int NG = Win::TW / CT_CPI;
      constexpr int B0 = Win::B0;
      const int k = tid / NG;
      const int cg = (tid - k * NG) * CT_CPI;
      const int o = r_begin + CT_CH * (u - H) + k;   // output row
      if (k < CT_CH && o < r_end && cg < cN) {
        const float4 *V = &S.V[k][pad4(cg)];
        const float *Jd = &S.spow[k][pad4(cg)];
        float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < WRG; i++) add4(w, V[pad4(B0 + i)]);
        float out[CT_CPI];
#pragma unroll
        for (int uu = 0; uu < CT_CPI; uu++) {
          if (COMP) {
            w = window_pairwise(V, WRG, [&](int i) { return pad4(B0 + uu + i); });
          } else if (uu > 0) {
            const float4 a = V[pad4(B0 + uu - 1 + WRG)];
            const float4 b = V[pad4(B0 + uu - 1)];
            const float2 m1 = make_float2(-1.f, -1.f);
            const float2 wc = __fadd2_rn(make_float2(w.x, w.y),
                                         __ffma2_rn(make_float2(b.x, b.y), m1, make_float2(a.x, a.y)));
            const float2 wp = __fadd2_rn(make_float2(w.z, w.w),
                                         __ffma2_rn(make_float2(b.z, b.w), m1, make_float2(a.z, a.w)));
            w = make_float4(wc.x, wc.y, wp.x, wp.y);
          }
          const float pp = w.z * w.w;
          const float num = fmaf(w.x, w.x, w.y * w.y);
          float g = (pp > 0.f && num > 0.f) ? num * rsqrtf(num) * rsqrtf(pp) : 0.f;
          if (Jd[pad4(uu + Win::XOFF)] < 1e-6f) g = 0.f;
          out[uu] = g;
        }
        float *orow = J.coh + (long)o * J.coh_pitch + c0 + cg;
        if (cg + CT_CPI <= cN && ((reinterpret_cast<uintptr_t>(orow) & 15) == 0)) {
#pragma unroll
          for (int v = 0; v < CT_CPI; v += 4)
            *reinterpret_cast<float4 *>(orow + v) =
                make_float4(out[v], out[v + 1], out[v + 2], out[v + 3]);
        } else {
#pragma unroll
          for (int uu = 0; uu < CT_CPI; uu++)
            if (cg + uu < cN) orow[uu] = out[uu];
        }
      }
    }
    __syncthreads();
  }
  seq += T;
  return ok;
}

template <int WAZ, int WRG, bool COMP>
__global__ void __launch_bounds__(CT_NT, 3) coh_tma_kernel(const __grid_constant__ CtBatch B) {
  extern __shared__ __align__(128) unsigned char ct_smem_raw[];
  CtShared &S = *reinterpret_cast<CtShared *>(ct_smem_raw);
  if (threadIdx.x == 0) {
    for (int k = 0; k < CT_NST; k++) ct_mbar_init(&S.full[k]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned seq = 0;
  int item = blockIdx.x;
  if (B.counter) {
    if (threadIdx.x == 0) S.next_item = atomicAdd(B.counter, 1);
    __syncthreads();
    item = S.next_item;
    __syncthreads();
  }
  while (item < B.total_items) {
    if (!coh_tma_item<WAZ, WRG, COMP>(S, B, item, seq)) break;
    if (!B.counter) break;
    if (threadIdx.x == 0) S.next_item = atomicAdd(B.counter, 1);
    __syncthreads();
    item = S.next_item;
    __syncthreads();
  }
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on it).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    (void)cudaGetLastError();
  });
  return fn;
}

// The TMA variant takes a job when both images start on a 16-byte boundary
// and their row pitches are multiples of 16 bytes (a tensor map's rules).
static bool tma_eligible(const CohJob &J) {
  const uintptr_t m = reinterpret_cast<uintptr_t>(J.master);
  const uintptr_t s = reinterpret_cast<uintptr_t>(J.slave);
  return (m % 16 == 0) && (s % 16 == 0) && ((J.master_pitch * 4) % 16 == 0) &&
         ((J.slave_pitch * 8) % 16 == 0) && J.pixels >= 1 && J.lines >= 1;
}

static int encode_maps(const CohJob &J, CUtensorMap *tm_m, CUtensorMap *tm_s) {
  auto fn = tensor_map_encoder();
  if (!fn) return TOPS_E_CUDA;
  const cuuint64_t dims[2] = {(cuuint64_t)J.pixels, (cuuint64_t)J.lines};
  const cuuint32_t box[2] = {(cuuint32_t)CT_LW, (cuuint32_t)CT_CH};
  const cuuint32_t estr[2] = {1, 1};
  const cuuint64_t sm[1] = {(cuuint64_t)J.master_pitch * 4};
  const cuuint64_t ss[1] = {(cuuint64_t)J.slave_pitch * 8};
  CUresult r = fn(tm_m, CU_TENSOR_MAP_DATA_TYPE_INT32, 2, const_cast<short2 *>(J.master), dims,
                  sm, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return TOPS_E_INVALID;
  r = fn(tm_s, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<float2 *>(J.slave), dims, ss, box,
         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? TOPS_OK : TOPS_E_INVALID;
}

template <int WAZ, int WRG>
static int launch_coh_tma(const CohJob *jobs, int njobs, const TileCfg &cfg, int dev,
                          cudaStream_t st) {
  static PerDeviceOnce setup;
  int resident = 0;
  const int s0 = once_per_device(
      setup, dev,
      [&](int &v) -> int {
        for (auto fn : {coh_tma_kernel<WAZ, WRG, false>, coh_tma_kernel<WAZ, WRG, true>})
          TOPS_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(CtShared)));
        int per_sm = 0, sms = 0;
        TOPS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, coh_tma_kernel<WAZ, WRG, false>, CT_NT, sizeof(CtShared)));
        TOPS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        v = per_sm * sms;
        return TOPS_OK;
      },
      &resident);
  if (s0 != TOPS_OK) return s0;
  for (int j0 = 0, k = 0; j0 < njobs; j0 += CT_MAXJOBS, k++) {
    CtBatch B;
    B.njobs = 0;
    B.compensated = cfg.compensated;
    B.counter = cfg.counters ? cfg.counters + k : nullptr;
    int items = 0;
    for (int j = j0; j < njobs && j < j0 + CT_MAXJOBS; j++) {
      CohJob &J = B.jobs[B.njobs];
      J = jobs[j];
      J.seg_rows = cfg.seg_rows ? cfg.seg_rows : CT_SEG;
      J.segs = (J.lines + J.seg_rows - 1) / J.seg_rows;
      J.strips = (J.pixels + CtWin<WRG>::TW - 1) / CtWin<WRG>::TW;
      J.item_begin = items;
      items += J.strips * J.segs;
      const int s = encode_maps(J, &B.tm_m[B.njobs], &B.tm_s[B.njobs]);
      if (s != TOPS_OK) return s;
      B.njobs++;
    }
    B.total_items = items;
    if (!items) continue;
    int grid = items;
    if (B.counter) {
      TOPS_CUDA_TRY(cudaMemsetAsync(B.counter, 0, sizeof(int), st));
      grid = min(items, cfg.grid > 0 ? cfg.grid : resident);
    }
    if (B.compensated)
      coh_tma_kernel<WAZ, WRG, true><<<grid, CT_NT, sizeof(CtShared), st>>>(B);
    else
      coh_tma_kernel<WAZ, WRG, false><<<grid, CT_NT, sizeof(CtShared), st>>>(B);
    TOPS_CUDA_TRY(cudaGetLastError());
  }
  return TOPS_OK;
}

template <int WAZ, int WRG>
static int launch_coh_t(const CoBatch &B, int grid, cudaStream_t st) {
  if (B.compensated)
    coherence_kernel<WAZ, WRG, true><<<grid, CO_NT, 0, st>>>(B);
  else
    coherence_kernel<WAZ, WRG, false><<<grid, CO_NT, 0, st>>>(B);
  TOPS_CUDA_TRY(cudaGetLastError());
  return TOPS_OK;
}

template <int WAZ, int WRG>
static int coh_resident(int dev) {
  static PerDeviceOnce setup;
  int resident = 0;
  const int s = once_per_device(
      setup, dev,
      [&](int &v) -> int {
        int per_sm = 0, sms = 0;
        TOPS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, coherence_kernel<WAZ, WRG, false>, CO_NT, 0));
        TOPS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        v = per_sm * sms;
        return TOPS_OK;
      },
      &resident);
  return s == TOPS_OK ? resident : 0;
}

// The compiled (azimuth, range) windows: the config's 3 x 10 and the
// reference driver's 6 x 24 (Func.cpp:2583-2584); others run generic code.
template <int WAZ>
static int launch_coh_rg(const CoBatch &B, int grid, int resident_only, int dev,
                         cudaStream_t st) {
  if (B.win_rg == 10)
    return resident_only ? coh_resident<WAZ, 10>(dev) : launch_coh_t<WAZ, 10>(B, grid, st);
  if (B.win_rg == 24)
    return resident_only ? coh_resident<WAZ, 24>(dev) : launch_coh_t<WAZ, 24>(B, grid, st);
  return resident_only ? coh_resident<WAZ, 0>(dev) : launch_coh_t<WAZ, 0>(B, grid, st);
}

static int coh_dispatch(const CoBatch &B, int grid, int resident_only, int dev, cudaStream_t st) {
  if (B.win_az == 3) return launch_coh_rg<3>(B, grid, resident_only, dev, st);
  if (B.win_az == 6) return launch_coh_rg<6>(B, grid, resident_only, dev, st);
  return launch_coh_rg<0>(B, grid, resident_only, dev, st);
}

int launch_coherence(const CohJob *jobs, int njobs, int win_rg, int win_az, const TileCfg &cfg,
                     cudaStream_t st) {
  if (win_rg < 1 || win_az < 1 || win_rg > CO_MAX_WIN_RG) return TOPS_E_INVALID;
  if (cfg.seg_rows < 0 || cfg.seg_rows > 512 || (cfg.seg_rows && cfg.seg_rows < CO_GR))
    return TOPS_E_INVALID;
  int dev = 0;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return TOPS_E_INVALID;
  // the TMA-staged kernel for the pipeline's 10 x 3 and the reference
  // driver's 24 x 6 windows (and 10 x 6, 24 x 3)
  if ((win_rg == 10 || win_rg == 24) && (win_az == 3 || win_az == 6) && tensor_map_encoder()) {
    bool all = true;
    for (int j = 0; j < njobs; j++) all = all && tma_eligible(jobs[j]);
    if (all) {
      if (win_rg == 10)
        return win_az == 3 ? launch_coh_tma<3, 10>(jobs, njobs, cfg, dev, st)
                           : launch_coh_tma<6, 10>(jobs, njobs, cfg, dev, st);
      return win_az == 3 ? launch_coh_tma<3, 24>(jobs, njobs, cfg, dev, st)
                         : launch_coh_tma<6, 24>(jobs, njobs, cfg, dev, st);
    }
  }
  for (int j0 = 0, k = 0; j0 < njobs; j0 += CO_MAXJOBS, k++) {
    CoBatch B;
    B.njobs = 0;
    B.compensated = cfg.compensated;
    B.win_rg = win_rg;
    B.win_az = win_az;
    B.counter = cfg.counters ? cfg.counters + k : nullptr;
    int items = 0;
    for (int j = j0; j < njobs && j < j0 + CO_MAXJOBS; j++) {
      CohJob &J = B.jobs[B.njobs];
      J = jobs[j];
      if (cfg.seg_rows) {
        J.seg_rows = cfg.seg_rows;
        J.segs = (J.lines + cfg.seg_rows - 1) / cfg.seg_rows;
      }
      J.item_begin = items;
      items += J.strips * J.segs;
      B.njobs++;
    }
    B.total_items = items;
    if (!items) continue;
    int grid = items;
    if (B.counter) {
      TOPS_CUDA_TRY(cudaMemsetAsync(B.counter, 0, sizeof(int), st));
      const int res = coh_dispatch(B, 0, 1, dev, st);
      if (res <= 0) return TOPS_E_CUDA;
      grid = min(items, cfg.grid > 0 ? cfg.grid : res);
    }
    const int s = coh_dispatch(B, grid, 0, dev, st);
    if (s != TOPS_OK) return s;
  }
  return TOPS_OK;
}

int fill_coh_job(const tops_coh_job &u, CohJob &J) {
  if (!u.master || !u.slave || !u.coh || u.lines <= 0 || u.pixels <= 0) return TOPS_E_INVALID;
  if ((u.master_pitch % sizeof(short2)) || (u.slave_pitch % sizeof(float2)) ||
      (u.coh_pitch % sizeof(float)))
    return TOPS_E_INVALID;
  J.master = static_cast<const short2 *>(u.master);
  J.master_pitch = (long)(u.master_pitch / sizeof(short2));
  J.slave = static_cast<const float2 *>(u.slave);
  J.slave_pitch = (long)(u.slave_pitch / sizeof(float2));
  J.coh = u.coh;
  J.coh_pitch = (long)(u.coh_pitch / sizeof(float));
  if (J.master_pitch < u.pixels || J.slave_pitch < u.pixels || J.coh_pitch < u.pixels)
    return TOPS_E_INVALID;
  J.lines = u.lines;
  J.pixels = u.pixels;
  J.strips = (u.pixels + CO_TW - 1) / CO_TW;
  J.seg_rows = CO_SEG;
  J.segs = (u.lines + CO_SEG - 1) / CO_SEG;
  return TOPS_OK;
}

}  // namespace tops

using namespace tops;

extern "C" int tops_coherence(const tops_coh_job *jobs, int njobs, int win_rg, int win_az,
                              void *stream) {
  if ((!jobs && njobs > 0) || njobs < 0) return TOPS_E_INVALID;
  std::vector<CohJob> J(njobs);
  for (int j = 0; j < njobs; j++) {
    int s = fill_coh_job(jobs[j], J[j]);
    if (s != TOPS_OK) return s;
  }
  return launch_coherence(J.data(), njobs, win_rg, win_az, TileCfg(),
                          static_cast<cudaStream_t>(stream));
}

namespace tops {

int coherence_launch(const tops_coh_job *jobs, int njobs, int win_rg, int win_az,
                     const TileCfg &cfg, cudaStream_t st) {
  if ((!jobs && njobs > 0) || njobs < 0) return TOPS_E_INVALID;
  std::vector<CohJob> J(njobs);
  for (int j = 0; j < njobs; j++) {
    int s = fill_coh_job(jobs[j], J[j]);
    if (s != TOPS_OK) return s;
  }
  return launch_coherence(J.data(), njobs, win_rg, win_az, cfg, st);
}

}  // namespace tops

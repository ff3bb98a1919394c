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
#include <cuda_runtime.h>

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

// Horizontal pass of one group: CO_CPI consecutive outputs per item.  The
// amplitude mask |s| < 0.001 of the reference (EstCoh.cu:393, 446) is
// evaluated as |s|^2 < 1e-6.  WRG > 0: range window known at compile time;
// an item starts at a multiple of 8 columns, so pad8(cg + i) = pad8(cg) +
// pad8(i) and every shared-memory offset below is a constant.
template <int WRG>
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
      if (u > 0) {
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
template <int WAZ, int WRG>
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
      coh_horizontal<WRG>(S, J, tid, rg, gr, c0, cN, win_rg, dx);
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
      coh_horizontal<WRG>(S, J, tid, rg, gr, c0, cN, win_rg, dx);
      __syncthreads();
    }
  }
}

template <int WAZ, int WRG>
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
    coherence_item<WAZ, WRG>(S, B, item);
    if (!B.counter) break;
    if (threadIdx.x == 0) S.next_item = atomicAdd(B.counter, 1);
    __syncthreads();
    item = S.next_item;
    __syncthreads();
  }
}

template <int WAZ, int WRG>
static int launch_coh_t(const CoBatch &B, int grid, cudaStream_t st) {
  coherence_kernel<WAZ, WRG><<<grid, CO_NT, 0, st>>>(B);
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
            &per_sm, coherence_kernel<WAZ, WRG>, CO_NT, 0));
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
  for (int j0 = 0, k = 0; j0 < njobs; j0 += CO_MAXJOBS, k++) {
    CoBatch B;
    B.njobs = 0;
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

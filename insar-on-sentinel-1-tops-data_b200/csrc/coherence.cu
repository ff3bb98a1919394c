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
// rows: it reads master (CInt16) and slave (complex64) once per row with
// coalesced loads, forms the four products and accumulates the vertical box
// sums for the group's rows in registers.  The vertical sums go to shared
// memory; the horizontal box is a sliding sum over 8 consecutive outputs per
// thread, written with 16-byte stores.  The azimuth window is a template
// parameter for the common sizes (3 and the reference's 6).  HBM traffic is the algorithmic
// 4 + 8 + 4 bytes per pixel plus the column halo.
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace tops {

constexpr int CO_NT = 256;
constexpr int CO_TW = 224;   // output columns per strip (win_rg <= 33)
constexpr int CO_GR = 8;     // rows per group
constexpr int CO_SEG = 64;   // rows per work item
constexpr int CO_CPI = 8;    // output columns per horizontal item
constexpr int CO_MAXJOBS = 32;
constexpr int CO_MAX_WIN_RG = CO_NT - CO_TW + 1;

struct CoBatch {
  int njobs, total_items, win_rg, win_az;
  CohJob jobs[CO_MAXJOBS];
};

struct CoShared {
  float4 V[CO_GR][pad8(CO_NT)];      // vertical sums (re, im, |s|^2, |m|^2), pad8(x)
  float judge[CO_GR][pad8(CO_NT)];   // |s|^2 of the centre pixel, pad8(x)
};

// WAZ > 0: azimuth window known at compile time (the vertical box is fully
// unrolled); WAZ == 0: runtime window.  The amplitude mask |s| < 0.001 of
// the reference (EstCoh.cu:393, 446) is evaluated as |s|^2 < 1e-6.
template <int WAZ>
__global__ void __launch_bounds__(CO_NT) coherence_kernel(const __grid_constant__ CoBatch B) {
  __shared__ CoShared S;
  const int tid = threadIdx.x;
  const int item = blockIdx.x;
  if (item >= B.total_items) return;
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

  for (int rg = r_begin; rg < r_end; rg += CO_GR) {
    const int gr = min(CO_GR, r_end - rg);
    // ---- vertical pass: input rows rg-dy .. rg-dy+gr+win_az-2
    float4 acc[CO_GR];
    float judge[CO_GR];
#pragma unroll
    for (int k = 0; k < CO_GR; k++) {
      acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      judge[k] = 0.f;
    }
    const int nin = gr + win_az - 1;
    auto product = [&](short2 m, float2 s) {
      const float mr = m.x, mi = m.y;
      return make_float4(mr * s.x + mi * s.y,   // m * conj(s)
                         mi * s.x - mr * s.y, s.x * s.x + s.y * s.y, mr * mr + mi * mi);
    };
    auto load = [&](int q, short2 &m, float2 &s) {
      const int y = rg - dy + q;
      m = make_short2(0, 0);
      s = make_float2(0.f, 0.f);
      if (xin && q < nin && y >= 0 && y < J.lines) {
        m = J.master[(long)y * J.master_pitch + x];
        s = J.slave[(long)y * J.slave_pitch + x];
      }
    };
    if (WAZ > 0) {
      // all loads of the group first (memory-level parallelism), then math
      constexpr int NQ = CO_GR + (WAZ > 0 ? WAZ : 1) - 1;
      short2 mv[NQ];
      float2 sv[NQ];
#pragma unroll
      for (int q = 0; q < NQ; q++) load(q, mv[q], sv[q]);
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        const float4 p = product(mv[q], sv[q]);
#pragma unroll
        for (int k = 0; k < CO_GR; k++) {
          if (q - k >= 0 && q - k < WAZ) {
            acc[k].x += p.x;
            acc[k].y += p.y;
            acc[k].z += p.z;
            acc[k].w += p.w;
          }
          if (q == k + (WAZ - 1) / 2) judge[k] = p.z;
        }
      }
    } else {
      for (int q = 0; q < nin; q++) {
        short2 m;
        float2 sl;
        load(q, m, sl);
        const float4 p = product(m, sl);
#pragma unroll
        for (int k = 0; k < CO_GR; k++) {
          const int j = q - k;
          if (j >= 0 && j < win_az) {
            acc[k].x += p.x;
            acc[k].y += p.y;
            acc[k].z += p.z;
            acc[k].w += p.w;
          }
          if (q == k + dy) judge[k] = p.z;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < CO_GR; k++) {
      S.V[k][pad8(tid)] = acc[k];
      S.judge[k][pad8(tid)] = judge[k];
    }
    __syncthreads();
    // ---- horizontal pass: CO_CPI consecutive outputs per item
    constexpr int NG = CO_TW / CO_CPI;
    for (int it = tid; it < gr * NG; it += CO_NT) {
      const int k = it / NG;
      const int cg = (it - k * NG) * CO_CPI;
      if (cg >= cN) continue;
      float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int i = 0; i < win_rg; i++) {
        const float4 v = S.V[k][pad8(cg + i)];
        w.x += v.x;
        w.y += v.y;
        w.z += v.z;
        w.w += v.w;
      }
      float out[CO_CPI];
#pragma unroll
      for (int u = 0; u < CO_CPI; u++) {
        if (u > 0) {
          const float4 a = S.V[k][pad8(cg + u - 1 + win_rg)];
          const float4 b = S.V[k][pad8(cg + u - 1)];
          w.x += a.x - b.x;
          w.y += a.y - b.y;
          w.z += a.z - b.z;
          w.w += a.w - b.w;
        }
        const float p = w.z * w.w;
        float g = (p > 0.f) ? sqrtf(w.x * w.x + w.y * w.y) * rsqrtf(p) : 0.f;
        if (S.judge[k][pad8(cg + u + dx)] < 1e-6f) g = 0.f;
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
    __syncthreads();
  }
}

int launch_coherence(const CohJob *jobs, int njobs, int win_rg, int win_az, cudaStream_t st) {
  if (win_rg < 1 || win_az < 1 || win_rg > CO_MAX_WIN_RG) return TOPS_E_INVALID;
  for (int j0 = 0; j0 < njobs; j0 += CO_MAXJOBS) {
    CoBatch B;
    B.njobs = 0;
    B.win_rg = win_rg;
    B.win_az = win_az;
    int items = 0;
    for (int j = j0; j < njobs && j < j0 + CO_MAXJOBS; j++) {
      B.jobs[B.njobs] = jobs[j];
      B.jobs[B.njobs].item_begin = items;
      items += jobs[j].strips * jobs[j].segs;
      B.njobs++;
    }
    B.total_items = items;
    if (!items) continue;
    if (win_az == 3)
      coherence_kernel<3><<<items, CO_NT, 0, st>>>(B);
    else if (win_az == 6)
      coherence_kernel<6><<<items, CO_NT, 0, st>>>(B);
    else
      coherence_kernel<0><<<items, CO_NT, 0, st>>>(B);
    TOPS_CUDA_TRY(cudaGetLastError());
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
  return launch_coherence(J.data(), njobs, win_rg, win_az, static_cast<cudaStream_t>(stream));
}

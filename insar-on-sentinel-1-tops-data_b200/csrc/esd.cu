// esd.cu -- Enhanced Spectral Diversity azimuth-shift estimation (sm_100a).
//
// Reference chain per overlap (EstESDShifts_NonOverlap, EstESD.cu:914-1252):
//   CohMatrixSet (:94-128) + CohFirstLineSet_ESD/CohDiffer_vertical_ESD/
//   shfl_vertical_ESD/CpCoh2_ESD (:297-546)   -> gamma of the forward and of
//                                                the backward band (zero-
//                                                padded winAz x winRg box)
//   Divide2 (:243-259)                        -> gamma = (gF + gB) / 2
//   DoubleDifference4OneD (:62-91)            -> dd = (mF sF*) conj(mB sB*)
//   MaskOut (:130-161)                        -> 0 if gamma < thr or >= 1,
//                                                else exp(i arg dd)
//   reduce0 x3 (:262-295)                     -> S = sum over the band
//   host (:1213-1217)                         -> shift = atan2(S)/(2 pi df dt)
//
// B200 design: ONE kernel for all overlaps and both bands.  A CTA owns a
// (strip, row segment) of one overlap; each thread owns a loaded column,
// reads the four bands once per row (coalesced), keeps the vertical box sums
// of both bands in registers and the centre-pixel interferograms in shared
// memory; the horizontal box, the mask and the unit phasor are evaluated per
// output pixel and accumulated in registers.  Per-CTA partial sums go to a
// scratch array; a second tiny kernel reduces them per overlap in a fixed
// order (deterministic) and evaluates the shift on the device, so the
// shifts can feed the corrected resample without a host round trip.
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>
#include <vector>

#include "common.cuh"

namespace tops {

constexpr int ES_NT = 256;
constexpr int ES_TW = 224;
constexpr int ES_GR = 4;
constexpr int ES_SEG = 32;
constexpr int ES_MAXOV = 32;

struct EsBatch {
  int n_ov, total_items, win_rg, win_az;
  float thr;
  int compensated;   // 1: per-thread phasor sums with Kahan compensation
  EsdOverlap ov[ES_MAXOV];
};

// Shared rows are padded by one slot every 4 (pad4): a horizontal item
// starts at a multiple of 4 columns, so its 16-byte sum loads and 8-byte
// centre loads fall in distinct banks across the warp, and the padded
// offsets of an item are constants when the window width is.
__host__ __device__ constexpr int es_pad(int x) { return x + (x >> 2); }

struct EsShared {
  float4 VF[ES_GR][es_pad(ES_NT)];
  float4 VB[ES_GR][es_pad(ES_NT)];
  float2 IF[ES_GR][es_pad(ES_NT)];   // centre mF * conj(sF)
  float2 IB[ES_GR][es_pad(ES_NT)];   // centre mB * conj(sB)
  float2 red[ES_NT / 32];
};

__device__ __forceinline__ float4 prod4(short2 m, float2 s) {
  const float mr = m.x, mi = m.y;
  return make_float4(mr * s.x + mi * s.y, mi * s.x - mr * s.y, s.x * s.x + s.y * s.y,
                     mr * mr + mi * mi);
}

// |sum m s*| / sqrt(sum |s|^2 sum |m|^2) as num rsqrt(num) rsqrt(p): two
// MUFU reciprocal square roots instead of two IEEE square roots and a
// division (relative error a few 1e-7)
__device__ __forceinline__ float gamma_of(float4 w) {
  const float p = w.z * w.w;
  const float num = fmaf(w.x, w.x, w.y * w.y);
  return (p > 0.f && num > 0.f) ? num * rsqrtf(num) * rsqrtf(p) : 0.f;
}

// WAZ > 0: the azimuth window height at compile time, so the input rows of a
// group are loaded together (their latencies overlap); 0: any height.  WRG >
// 0: the range window width at compile time (the horizontal box unrolls).
template <int WAZ, int WRG>
__global__ void __launch_bounds__(ES_NT, 2) esd_kernel(const __grid_constant__ EsBatch B,
                                                        double2 *partials) {
  extern __shared__ __align__(16) unsigned char es_smem[];
  EsShared &S = *reinterpret_cast<EsShared *>(es_smem);
  const int tid = threadIdx.x;
  const int item = blockIdx.x;
  if (item >= B.total_items) return;
  int ob = 0;
  while (ob + 1 < B.n_ov && B.ov[ob + 1].item_begin <= item) ob++;
  const EsdOverlap &O = B.ov[ob];
  const int local = item - O.item_begin;
  const int strip = local % O.strips, seg = local / O.strips;
  const int win_rg = WRG > 0 ? WRG : B.win_rg, win_az = WAZ > 0 ? WAZ : B.win_az;
  const int dw = (win_rg - 1) / 2, dh = (win_az - 1) / 2;
  const int c0 = strip * ES_TW;
  const int cN = min(ES_TW, O.pixels - c0);
  const int nload = cN + win_rg - 1;
  const int r_begin = seg * O.seg_rows;
  const int r_end = min(r_begin + O.seg_rows, O.lines);
  const int x = c0 - dw + tid;
  const bool xin = tid < nload && x >= 0 && x < O.pixels;
  float accr = 0.f, acci = 0.f;
  float cr = 0.f, ci = 0.f;   // Kahan compensation terms (compensated mode)
  const bool comp = B.compensated != 0;
  // adds one unit phasor to the thread's sums
  auto accumulate = [&](float re, float im) {
    if (comp) {
      const float yr = re - cr, yi = im - ci;
      const float tr = accr + yr, ti = acci + yi;
      cr = (tr - accr) - yr;
      ci = (ti - acci) - yi;
      accr = tr;
      acci = ti;
    } else {
      accr += re;
      acci += im;
    }
  };

  // horizontal box, mask and unit phasor of the group's rows (shared-memory
  // vertical sums and centre interferograms), accumulated into accr / acci
  auto horizontal = [&](int gr) {
    const int ngrp = (cN + 3) >> 2;
    for (int it = tid; it < gr * ngrp; it += ES_NT) {
      const int k = it / ngrp;
      const int cg = (it - k * ngrp) << 2;
      float4 wF = make_float4(0.f, 0.f, 0.f, 0.f), wB = wF;
      const float4 *VF = &S.VF[k][es_pad(cg)], *VB = &S.VB[k][es_pad(cg)];
#pragma unroll
      for (int i = 0; i < win_rg; i++) {
        const float4 a = VF[es_pad(i)], b = VB[es_pad(i)];
        wF.x += a.x; wF.y += a.y; wF.z += a.z; wF.w += a.w;
        wB.x += b.x; wB.y += b.y; wB.z += b.z; wB.w += b.w;
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (u > 0) {
          const int ia = es_pad(u - 1 + win_rg), ib = es_pad(u - 1);
          const float4 a = VF[ia], b = VF[ib];
          wF.x += a.x - b.x; wF.y += a.y - b.y; wF.z += a.z - b.z; wF.w += a.w - b.w;
          const float4 c = VB[ia], d = VB[ib];
          wB.x += c.x - d.x; wB.y += c.y - d.y; wB.z += c.z - d.z; wB.w += c.w - d.w;
        }
        if (cg + u >= cN) continue;
        const float g = (gamma_of(wF) + gamma_of(wB)) * 0.5f;
        if (g < B.thr || g >= 1.f) continue;
        const float2 f = S.IF[k][es_pad(cg) + es_pad(u + dw)];
        const float2 b = S.IB[k][es_pad(cg) + es_pad(u + dw)];
        // (mF sF*) * conj(mB sB*)
        const float dre = f.x * b.x + f.y * b.y;
        const float dim = f.y * b.x - f.x * b.y;
        const float n2 = dre * dre + dim * dim;
        if (n2 > 0.f) {
          const float inv = rsqrtf(n2);
          accumulate(dre * inv, dim * inv);
        } else {
          // An exactly-zero double difference (a slave sample outside its
          // box) has the phase atan2 gives its signed zeros: 0, -0, pi or
          // -pi, as in MaskOut (EstESD.cu:149-155).  dre and dim carry the
          // same signs of zero as the reference's cuCmulf products.
          float sn, cs;
          sincosf(atan2f(dim, dre), &sn, &cs);
          accumulate(cs, sn);
        }
      }
    }
  };

  if constexpr (WAZ > 0 && WAZ <= 4) {
    // Short windows: the products of the last WAZ - 1 input rows stay in
    // registers from one group to the next, so every input row is read
    // once, and the next group's rows are loaded before the current group's
    // horizontal pass, so their latency overlaps it.
    constexpr int NQ = WAZ - 1 > 0 ? WAZ - 1 : 1;
    auto load = [&](int y, short2 &mf, float2 &sf, short2 &mb, float2 &sb) {
      mf = mb = make_short2(0, 0);
      sf = sb = make_float2(0.f, 0.f);
      if (xin && y >= 0 && y < O.lines) {
        const long mo = (long)y * O.m_pitch + x, so = (long)y * O.s_pitch + x;
        mf = O.mF[mo];
        sf = O.sF[so];
        mb = O.mB[mo];
        sb = O.sB[so];
      }
    };
    float4 qF[NQ], qB[NQ];
#pragma unroll
    for (int j = 0; j < WAZ - 1; j++) {
      short2 mf, mb;
      float2 sf, sb;
      load(r_begin - dh + j, mf, sf, mb, sb);
      qF[j] = prod4(mf, sf);
      qB[j] = prod4(mb, sb);
    }
    short2 vmf[ES_GR], vmb[ES_GR];
    float2 vsf[ES_GR], vsb[ES_GR];
#pragma unroll
    for (int k = 0; k < ES_GR; k++)
      load(r_begin - dh + WAZ - 1 + k, vmf[k], vsf[k], vmb[k], vsb[k]);
    for (int rg = r_begin; rg < r_end; rg += ES_GR) {
      const int gr = min(ES_GR, r_end - rg);
      float4 pF[WAZ - 1 + ES_GR], pB[WAZ - 1 + ES_GR];
#pragma unroll
      for (int j = 0; j < WAZ - 1; j++) {
        pF[j] = qF[j];
        pB[j] = qB[j];
      }
#pragma unroll
      for (int k = 0; k < ES_GR; k++) {
        pF[WAZ - 1 + k] = prod4(vmf[k], vsf[k]);
        pB[WAZ - 1 + k] = prod4(vmb[k], vsb[k]);
      }
      const int rn = rg + ES_GR;
      if (rn < r_end) {
#pragma unroll
        for (int k = 0; k < ES_GR; k++)
          load(rn - dh + WAZ - 1 + k, vmf[k], vsf[k], vmb[k], vsb[k]);
      }
#pragma unroll
      for (int k = 0; k < ES_GR; k++) {
        float4 aF = pF[k], aB = pB[k];
#pragma unroll
        for (int j = 1; j < WAZ; j++) {
          aF.x += pF[k + j].x; aF.y += pF[k + j].y; aF.z += pF[k + j].z; aF.w += pF[k + j].w;
          aB.x += pB[k + j].x; aB.y += pB[k + j].y; aB.z += pB[k + j].z; aB.w += pB[k + j].w;
        }
        S.VF[k][es_pad(tid)] = aF;
        S.VB[k][es_pad(tid)] = aB;
        S.IF[k][es_pad(tid)] = make_float2(pF[k + dh].x, pF[k + dh].y);
        S.IB[k][es_pad(tid)] = make_float2(pB[k + dh].x, pB[k + dh].y);
      }
#pragma unroll
      for (int j = 0; j < WAZ - 1; j++) {
        qF[j] = pF[ES_GR + j];
        qB[j] = pB[ES_GR + j];
      }
      __syncthreads();
      horizontal(gr);
      __syncthreads();
    }
  } else {
  for (int rg = r_begin; rg < r_end; rg += ES_GR) {
    const int gr = min(ES_GR, r_end - rg);
    float4 aF[ES_GR], aB[ES_GR];
    float2 cF[ES_GR], cB[ES_GR];
#pragma unroll
    for (int k = 0; k < ES_GR; k++) {
      aF[k] = aB[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      cF[k] = cB[k] = make_float2(0.f, 0.f);
    }
    // input rows rg - dh .. rg - dh + nin - 1 (all of them for a full group:
    // rows past the overlap's end load as zero)
    const int nin = WAZ > 0 ? ES_GR + WAZ - 1 : gr + win_az - 1;
#pragma unroll
    for (int q = 0; q < (WAZ > 0 ? ES_GR + WAZ - 1 : 1 << 20); q++) {
      if (WAZ == 0 && q >= nin) break;
      const int y = rg - dh + q;
      float4 pF = make_float4(0.f, 0.f, 0.f, 0.f), pB = pF;
      if (xin && y >= 0 && y < O.lines) {
        const long mo = (long)y * O.m_pitch + x, so = (long)y * O.s_pitch + x;
        pF = prod4(O.mF[mo], O.sF[so]);
        pB = prod4(O.mB[mo], O.sB[so]);
      }
#pragma unroll
      for (int k = 0; k < ES_GR; k++) {
        const int j = q - k;
        if (j >= 0 && j < win_az) {
          aF[k].x += pF.x; aF[k].y += pF.y; aF[k].z += pF.z; aF[k].w += pF.w;
          aB[k].x += pB.x; aB[k].y += pB.y; aB[k].z += pB.z; aB[k].w += pB.w;
        }
        if (q == k + dh) {
          cF[k] = make_float2(pF.x, pF.y);
          cB[k] = make_float2(pB.x, pB.y);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < ES_GR; k++) {
      S.VF[k][es_pad(tid)] = aF[k];
      S.VB[k][es_pad(tid)] = aB[k];
      S.IF[k][es_pad(tid)] = cF[k];
      S.IB[k][es_pad(tid)] = cB[k];
    }
    __syncthreads();
    horizontal(gr);
    __syncthreads();
  }
  }
  // ---- block reduction (fixed order); Kahan's best estimate is the sum
  // less its compensation term
  if (comp) {
    accr -= cr;
    acci -= ci;
  }
  for (int o = 16; o > 0; o >>= 1) {
    accr += __shfl_xor_sync(0xffffffffu, accr, o);
    acci += __shfl_xor_sync(0xffffffffu, acci, o);
  }
  if ((tid & 31) == 0) S.red[tid >> 5] = make_float2(accr, acci);
  __syncthreads();
  if (tid == 0) {
    double r = 0.0, i = 0.0;
    for (int w = 0; w < ES_NT / 32; w++) {
      r += S.red[w].x;
      i += S.red[w].y;
    }
    partials[item] = make_double2(r, i);
  }
}

__global__ void esd_finalize_kernel(const __grid_constant__ EsBatch B, const double2 *partials,
                                    double *shifts, double *sums, int ov_offset) {
  __shared__ double sr[256], si[256];
  const int o = blockIdx.x;
  const EsdOverlap &O = B.ov[o];
  const int n = O.strips * O.segs;
  double r = 0.0, i = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    r += partials[O.item_begin + k].x;
    i += partials[O.item_begin + k].y;
  }
  sr[threadIdx.x] = r;
  si[threadIdx.x] = i;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sr[threadIdx.x] += sr[threadIdx.x + s];
      si[threadIdx.x] += si[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double R = sr[0], I = si[0];
    shifts[ov_offset + o] = atan2(I, R) / (2 * kPi * O.spec_sep * O.dt);
    if (sums) {
      sums[2 * (ov_offset + o)] = R;
      sums[2 * (ov_offset + o) + 1] = I;
    }
  }
}

static int esd_items(const EsdOverlap &o) { return o.strips * o.segs; }

int fill_esd_overlap(const tops_esd_overlap &u, EsdOverlap &O) {
  if (!u.mF || !u.mB || !u.sF || !u.sB || u.lines < 0 || u.pixels <= 0) return TOPS_E_INVALID;
  if ((u.m_pitch % sizeof(short2)) || (u.s_pitch % sizeof(float2))) return TOPS_E_INVALID;
  O.mF = static_cast<const short2 *>(u.mF);
  O.mB = static_cast<const short2 *>(u.mB);
  O.m_pitch = (long)(u.m_pitch / sizeof(short2));
  O.sF = static_cast<const float2 *>(u.sF);
  O.sB = static_cast<const float2 *>(u.sB);
  O.s_pitch = (long)(u.s_pitch / sizeof(float2));
  if (O.m_pitch < u.pixels || O.s_pitch < u.pixels) return TOPS_E_INVALID;
  O.lines = u.lines;
  O.pixels = u.pixels;
  O.spec_sep = u.spec_sep;
  O.dt = u.dt;
  O.strips = (u.pixels + ES_TW - 1) / ES_TW;
  O.seg_rows = ES_SEG;
  O.segs = u.lines > 0 ? (u.lines + ES_SEG - 1) / ES_SEG : 1;
  return TOPS_OK;
}

size_t esd_scratch_bytes(const EsdOverlap *ov, int n) {
  size_t items = 0;
  for (int i = 0; i < n; i++) items += esd_items(ov[i]);
  return items * sizeof(double2);
}

int launch_esd(const EsdOverlap *ovs, int n_ov, int win_az, int win_rg, float thr,
               double *shifts, double *sums, void *scratch, size_t scratch_bytes,
               cudaStream_t st, int compensated) {
  if (win_rg < 1 || win_az < 1 || win_rg > ES_NT - ES_TW + 1) return TOPS_E_INVALID;
  if (esd_scratch_bytes(ovs, n_ov) > scratch_bytes || (!scratch && n_ov > 0) || !shifts)
    return TOPS_E_INVALID;
  // the shared-memory opt-in is a per-device function attribute
  static PerDeviceOnce setup;
  int dev = 0;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  const int s0 = once_per_device(
      setup, dev,
      [&](int &) -> int {
        for (auto fn : {esd_kernel<3, 10>, esd_kernel<3, 0>, esd_kernel<6, 24>, esd_kernel<6, 0>,
                        esd_kernel<0, 0>})
          TOPS_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(EsShared)));
        return TOPS_OK;
      },
      nullptr);
  if (s0 != TOPS_OK) return s0;
  double2 *part = static_cast<double2 *>(scratch);
  for (int o0 = 0; o0 < n_ov; o0 += ES_MAXOV) {
    EsBatch B;
    B.n_ov = 0;
    B.win_rg = win_rg;
    B.win_az = win_az;
    B.thr = thr;
    B.compensated = compensated;
    int items = 0;
    for (int o = o0; o < n_ov && o < o0 + ES_MAXOV; o++) {
      B.ov[B.n_ov] = ovs[o];
      B.ov[B.n_ov].item_begin = items;
      items += esd_items(ovs[o]);
      B.n_ov++;
    }
    B.total_items = items;
    if (win_az == 3 && win_rg == 10)
      esd_kernel<3, 10><<<items, ES_NT, sizeof(EsShared), st>>>(B, part);
    else if (win_az == 3)
      esd_kernel<3, 0><<<items, ES_NT, sizeof(EsShared), st>>>(B, part);
    else if (win_az == 6 && win_rg == 24)
      esd_kernel<6, 24><<<items, ES_NT, sizeof(EsShared), st>>>(B, part);
    else if (win_az == 6)
      esd_kernel<6, 0><<<items, ES_NT, sizeof(EsShared), st>>>(B, part);
    else
      esd_kernel<0, 0><<<items, ES_NT, sizeof(EsShared), st>>>(B, part);
    TOPS_CUDA_TRY(cudaGetLastError());
    esd_finalize_kernel<<<B.n_ov, 256, 0, st>>>(B, part, shifts, sums, o0);
    TOPS_CUDA_TRY(cudaGetLastError());
    part += items;
  }
  return TOPS_OK;
}

}  // namespace tops

using namespace tops;

extern "C" size_t tops_esd_scratch_bytes(const tops_esd_overlap *ovs, int n_ov) {
  std::vector<EsdOverlap> O(n_ov > 0 ? n_ov : 0);
  for (int i = 0; i < n_ov; i++)
    if (fill_esd_overlap(ovs[i], O[i]) != TOPS_OK) return 0;
  return esd_scratch_bytes(O.data(), n_ov);
}

extern "C" int tops_esd(const tops_esd_overlap *ovs, int n_ov, int win_az, int win_rg,
                        float coh_thr, double *shifts_dev, double *sums_dev, void *scratch_dev,
                        size_t scratch_bytes, void *stream) {
  if ((!ovs && n_ov > 0) || n_ov < 0) return TOPS_E_INVALID;
  std::vector<EsdOverlap> O(n_ov);
  for (int i = 0; i < n_ov; i++) {
    int s = fill_esd_overlap(ovs[i], O[i]);
    if (s != TOPS_OK) return s;
  }
  return launch_esd(O.data(), n_ov, win_az, win_rg, coh_thr, shifts_dev, sums_dev, scratch_dev,
                    scratch_bytes, static_cast<cudaStream_t>(stream), 0);
}

// --------------------------------------------------- allocation-free ESD
// tops_esd() needs a caller-allocated scratch buffer for the per-CTA partial
// sums.  Callers that must not allocate device memory use
// tops_esd_static(), whose scratch is this file-scope array.  Every GPU
// that loads the library holds it (256 KB) until the process exits.
namespace tops {

constexpr int ESD_STATIC_PARTIALS = 16384;
static __device__ __align__(256) double2 g_esd_static_partials[ESD_STATIC_PARTIALS];
constexpr int ESD_STATIC_MAX_DEVICES = 64;

// Device address of the array on the current device.  Host code cannot use
// the symbol itself (it names a host-side stand-in), so the address is
// fetched once per device with cudaGetSymbolAddress and cached.
static int esd_static_scratch(double2 **out) {
  static std::mutex mu;
  static double2 *addr[ESD_STATIC_MAX_DEVICES] = {};
  int dev = -1;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= ESD_STATIC_MAX_DEVICES) return TOPS_E_INVALID;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    TOPS_CUDA_TRY(cudaGetSymbolAddress(&p, g_esd_static_partials));
    addr[dev] = static_cast<double2 *>(p);
  }
  *out = addr[dev];
  return TOPS_OK;
}

}  // namespace tops

extern "C" int tops_esd_static(const tops_esd_overlap *ovs, int n_ov, int win_az, int win_rg,
                               float coh_thr, double *shifts_dev, double *sums_dev,
                               void *stream) {
  if (!ovs || n_ov < 1 || n_ov > ES_MAXOV) return TOPS_E_INVALID;
  EsdOverlap O[ES_MAXOV];  // host stack: no heap allocation either
  size_t items = 0;
  for (int i = 0; i < n_ov; i++) {
    int s = fill_esd_overlap(ovs[i], O[i]);
    if (s != TOPS_OK) return s;
    items += (size_t)esd_items(O[i]);
  }
  if (items > (size_t)ESD_STATIC_PARTIALS) {
    fprintf(stderr,
            "tops_esd_static: %zu partial sums needed, the static scratch holds %d "
            "(use tops_esd with a caller-provided scratch buffer)\n",
            items, ESD_STATIC_PARTIALS);
    return TOPS_E_INVALID;
  }
  double2 *scratch = nullptr;
  int s = esd_static_scratch(&scratch);
  if (s != TOPS_OK) return s;
  // every partial this call reads is written by this call's own launch, so
  // nothing in the shared array has to be cleared first
  return launch_esd(O, n_ov, win_az, win_rg, coh_thr, shifts_dev, sums_dev, scratch,
                    (size_t)ESD_STATIC_PARTIALS * sizeof(double2),
                    static_cast<cudaStream_t>(stream), 0);
}

namespace tops {

int esd_launch(const tops_esd_overlap *ovs, int n_ov, int win_az, int win_rg, float coh_thr,
               double *shifts_dev, double *sums_dev, void *scratch_dev, size_t scratch_bytes,
               int compensated, cudaStream_t st) {
  if ((!ovs && n_ov > 0) || n_ov < 0) return TOPS_E_INVALID;
  std::vector<EsdOverlap> O(n_ov);
  for (int i = 0; i < n_ov; i++) {
    int s = fill_esd_overlap(ovs[i], O[i]);
    if (s != TOPS_OK) return s;
  }
  return launch_esd(O.data(), n_ov, win_az, win_rg, coh_thr, shifts_dev, sums_dev, scratch_dev,
                    scratch_bytes, st, compensated);
}

}  // namespace tops

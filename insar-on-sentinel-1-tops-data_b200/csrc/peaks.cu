// peaks.cu -- measured FP64 throughput of the device (sm_100a), the
// denominator of the geometric coregistration's roofline: that stage is
// bound by FP64 arithmetic (zero-Doppler Newton solves), not by HBM.
//
// Every thread runs 8 independent FP64 fused-multiply-add chains (enough
// to cover the FMA latency with the resident warps), so the kernel time
// is the FP64 pipes' throughput.  Clocks and power limits are left as they
// are; the number is the one a kernel sees under the current conditions.
#include <cuda_runtime.h>

#include "common.cuh"

namespace tops {

constexpr int PK_NT = 256;
constexpr int PK_CHAINS = 8;

__device__ double g_fp64_sink;   // written only if the chains end at -1 (never)

__global__ void __launch_bounds__(PK_NT) fp64_fma_kernel(int iters) {
  double a[PK_CHAINS];
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) a[k] = 1e-3 * (threadIdx.x + k);
  const double b = 0.9999999, c = 1e-9;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < PK_CHAINS; k++) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) s += a[k];
  if (s == -1.0) g_fp64_sink = s;   // keeps the chains live
}

}  // namespace tops

using namespace tops;

extern "C" int tops_fp64_peak(double *tflops, void *stream) {
  if (!tflops) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0, per_sm = 0;
  TOPS_CUDA_TRY(cudaGetDevice(&dev));
  TOPS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  TOPS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp64_fma_kernel, PK_NT, 0));
  const int blocks = sms * (per_sm > 0 ? per_sm : 1);
  const int iters = 1 << 14;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TOPS_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    TOPS_CUDA_TRY(cudaErrorMemoryAllocation);
  }
  double best = 0.0;
  int r = TOPS_OK;
  for (int rep = 0; rep < 4 && r == TOPS_OK; rep++) {   // first launch is a warm-up
    cudaEventRecord(e0, st);
    fp64_fma_kernel<<<blocks, PK_NT, 0, st>>>(iters);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      set_cuda_error(e);
      (void)cudaGetLastError();
      r = TOPS_E_CUDA;
      break;
    }
    const double flops = 2.0 * PK_CHAINS * (double)iters * blocks * PK_NT;
    if (rep > 0 && ms > 0.f) best = fmax(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r == TOPS_OK) *tflops = best;
  return r;
}

// stitch.cu -- debursting row gather (sm_100a): dst row i = src row
// line_map[i] for CInt16, float or complex64 images (Stitch_OneSubswath,
// Func.cpp:2822-2933, which copies the rows line by line through GDAL).
//
// HBM-bound copy: one CTA per few output rows; threads move 16-byte vectors
// when both images' bases and pitches allow it, else 4-byte words.  The map
// comes from tops_stitch_line_map.  tops::row_copy runs the same loop
// without a map (row i copies row i) over several images in one launch.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "launch.h"

namespace tops {

constexpr int ST_NT = 256;
constexpr int ST_ROWS = 4;   // output rows per CTA

template <typename V>
__global__ void __launch_bounds__(ST_NT) stitch_kernel(const char *__restrict__ src, size_t sp,
                                                      char *__restrict__ dst, size_t dp,
                                                      const int *__restrict__ map, int height,
                                                      int nvec) {
  const int r0 = blockIdx.x * ST_ROWS;
  for (int r = r0; r < r0 + ST_ROWS && r < height; r++) {
    const V *s = reinterpret_cast<const V *>(src + (size_t)__ldg(map + r) * sp);
    V *d = reinterpret_cast<V *>(dst + (size_t)r * dp);
    for (int i = threadIdx.x; i < nvec; i += ST_NT) d[i] = __ldg(s + i);
  }
}

constexpr int RC_MAX = 16;   // copies per row_copy launch
struct RowCopies {
  RowCopy c[RC_MAX];
};

template <typename V>
__global__ void __launch_bounds__(ST_NT) row_copy_kernel(const RowCopies cs) {
  const RowCopy &c = cs.c[blockIdx.y];
  const int nvec = (int)(c.row_bytes / sizeof(V));
  const int r0 = blockIdx.x * ST_ROWS;
  for (int r = r0; r < r0 + ST_ROWS && r < c.height; r++) {
    const V *s = reinterpret_cast<const V *>(static_cast<const char *>(c.src) + (size_t)r * c.src_pitch);
    V *d = reinterpret_cast<V *>(static_cast<char *>(c.dst) + (size_t)r * c.dst_pitch);
    for (int i = threadIdx.x; i < nvec; i += ST_NT) d[i] = __ldg(s + i);
  }
}

int row_copy(const RowCopy *copies, int n, cudaStream_t st, int *launches) {
  if (n < 0 || (n > 0 && !copies)) return TOPS_E_INVALID;
  for (int k = 0; k < n; k++) {
    const RowCopy &c = copies[k];
    if (!c.src || !c.dst || c.height < 0 || c.row_bytes == 0 || (c.row_bytes & 3) ||
        c.src_pitch < c.row_bytes || c.dst_pitch < c.row_bytes || ((c.src_pitch | c.dst_pitch) & 3))
      return TOPS_E_INVALID;
  }
  for (int k0 = 0; k0 < n; k0 += RC_MAX) {
    RowCopies cs = {};
    int rows = 0, m = 0;
    uintptr_t bits = 0;
    for (int k = k0; k < n && k < k0 + RC_MAX; k++) {
      const RowCopy &c = copies[k];
      if (c.height == 0) continue;
      cs.c[m++] = c;
      rows = c.height > rows ? c.height : rows;
      bits |= reinterpret_cast<uintptr_t>(c.src) | reinterpret_cast<uintptr_t>(c.dst) |
              c.src_pitch | c.dst_pitch | c.row_bytes;
    }
    if (m == 0) continue;
    const dim3 grid((rows + ST_ROWS - 1) / ST_ROWS, m);
    if (!(bits & 15))
      row_copy_kernel<int4><<<grid, ST_NT, 0, st>>>(cs);
    else
      row_copy_kernel<int><<<grid, ST_NT, 0, st>>>(cs);
    TOPS_CUDA_TRY(cudaGetLastError());
    if (launches) *launches += 1;
  }
  return TOPS_OK;
}

}  // namespace tops

using namespace tops;

extern "C" int tops_stitch(const void *src, size_t src_pitch, void *dst, size_t dst_pitch,
                           const int *line_map_dev, int height, size_t row_bytes, void *stream) {
  if (!src || !dst || !line_map_dev || height < 0 || row_bytes == 0 || (row_bytes & 3) ||
      src_pitch < row_bytes || dst_pitch < row_bytes || (src_pitch & 3) || (dst_pitch & 3))
    return TOPS_E_INVALID;
  if (height == 0) return TOPS_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = (height + ST_ROWS - 1) / ST_ROWS;
  const bool v16 = !((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst) |
                      src_pitch | dst_pitch | row_bytes) & 15);
  if (v16)
    stitch_kernel<int4><<<blocks, ST_NT, 0, st>>>(static_cast<const char *>(src), src_pitch,
                                                 static_cast<char *>(dst), dst_pitch, line_map_dev,
                                                 height, (int)(row_bytes / 16));
  else
    stitch_kernel<int><<<blocks, ST_NT, 0, st>>>(static_cast<const char *>(src), src_pitch,
                                                static_cast<char *>(dst), dst_pitch, line_map_dev,
                                                height, (int)(row_bytes / 4));
  TOPS_CUDA_TRY(cudaGetLastError());
  return TOPS_OK;
}

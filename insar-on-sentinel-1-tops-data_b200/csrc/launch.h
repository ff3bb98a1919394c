// launch.h -- library-internal launch controls of the resample and coherence
// kernels, used by the batched plans (host/pipeline.cpp): the work-item tile
// (rows per item) and the scheduling mode.
//
//   seg_rows  output rows per work item; the resample kernel takes 12..252
//             (0: the longest of 252, 168, 120, 84 that gives two waves of
//             items), the coherence kernel 8..512 (0: its default)
//   counters  if non-null: persistent launch.  `grid` CTAs (0: as many as
//             fit on the device at once) pull work items from a queue -- the
//             device int counters[k], set to 0 on the stream before the k-th
//             launch of the call (a call launches once per 32 jobs).  The
//             caller provides at least (njobs + 31) / 32 ints.
#pragma once
#include <cuda_runtime.h>

#include "tops_b200.h"

namespace tops {

struct TileCfg {
  int seg_rows = 0;
  int *counters = nullptr;
  int grid = 0;
  int compensated = 0;   // coherence: window sums without the sliding update
};

int resample_launch(const tops_lut_dev *lut, const tops_resample_job *jobs, int njobs,
                    int precision, const TileCfg &cfg, cudaStream_t st);
// As resample_launch with one LUT per job (sub-swaths of one batch differ in
// PRF and bandwidth).
int resample_launch_multi(const tops_lut_dev *const *luts, const tops_resample_job *jobs,
                          int njobs, int precision, const TileCfg &cfg, cudaStream_t st);
int coherence_launch(const tops_coh_job *jobs, int njobs, int win_rg, int win_az,
                     const TileCfg &cfg, cudaStream_t st);
// tops_esd with the accumulation mode: compensated = 1 sums each thread's
// unit phasors with Kahan compensation.
int esd_launch(const tops_esd_overlap *ovs, int n_ov, int win_az, int win_rg, float coh_thr,
               double *shifts_dev, double *sums_dev, void *scratch_dev, size_t scratch_bytes,
               int compensated, cudaStream_t st);
// Same-device 2-D copies (dst row i = src row i) with the debursting gather
// kernel, several in one launch (blockIdx.y picks the copy): HBM speed,
// where the copy engine reaches about a third of it.  Pitches and row_bytes
// as tops_stitch takes them.
struct RowCopy {
  const void *src;
  size_t src_pitch;
  void *dst;
  size_t dst_pitch;
  size_t row_bytes;
  int height;
};
// One launch per 16 copies; *launches (if non-null) counts them.
int row_copy(const RowCopy *copies, int n, cudaStream_t st, int *launches);

}  // namespace tops

// batch.cpp -- several burst-pair plans (sub-swaths of different burst
// sizes) processed together: one launch per stage for all their bursts,
// optionally persistent kernels over a work queue, captured as one CUDA
// graph, with the work-item tile picked by a measurement-driven autotuner.
#include <cuda_runtime.h>
#include <string.h>

#include <vector>

#include "launch.h"
#include "pair_impl.h"

namespace {

#define B_TRY(expr)               \
  do {                            \
    int _s = (expr);              \
    if (_s != TOPS_OK) return _s; \
  } while (0)

#define B_CUDA(expr)                                                             \
  do {                                                                           \
    cudaError_t _e = (expr);                                                     \
    if (_e != cudaSuccess) {                                                     \
      (void)cudaGetLastError();                                                  \
      return _e == cudaErrorMemoryAllocation ? TOPS_E_NOMEM : TOPS_E_CUDA;       \
    }                                                                            \
  } while (0)

constexpr int kCounters = 64;   // queue counters: one per launch of a stage

}  // namespace

struct tops_batch {
  std::vector<tops_pair *> pairs;
  tops_pair_opts o;
  tops_tune tune;
  int n_ov = 0;                   // overlaps of all pairs
  std::vector<int> ov_begin;      // first overlap of each pair
  double *d_shift = nullptr, *d_sums = nullptr;
  int *d_counters = nullptr;
  void *d_geo_scratch = nullptr, *d_esd_scratch = nullptr;
  size_t geo_scratch = 0, esd_scratch = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t capture_stream = nullptr;
  int n_launches = 0;
  std::vector<void *> allocs;

  int alloc(void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? TOPS_E_NOMEM : TOPS_E_CUDA;
    allocs.push_back(*p);
    return TOPS_OK;
  }
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
  }
  ~tops_batch() {
    drop_graph();
    if (capture_stream) cudaStreamDestroy(capture_stream);
    for (void *p : allocs) cudaFree(p);
  }
};

namespace {

tops::TileCfg tile(int seg_rows, int persistent, int *counters) {
  tops::TileCfg c;
  c.seg_rows = seg_rows;
  c.counters = persistent ? counters : nullptr;
  return c;
}

int chunks(size_t n, int per) { return (int)((n + per - 1) / per); }

// The resample stage of all pairs as one launch (chunked per 32 jobs).
int batch_resample(tops_batch *B, bool esd_pass, int *counters, cudaStream_t st, int *launches) {
  std::vector<tops_resample_job> jobs;
  std::vector<const tops_lut_dev *> luts;
  std::vector<tops::RowCopy> copies;
  for (size_t p = 0; p < B->pairs.size(); p++) {
    const tops_pair *P = B->pairs[p];
    const size_t n0 = jobs.size();
    if (esd_pass) {
      pair_rs2_jobs(P, B->d_shift + B->ov_begin[p], jobs);
      // the first burst's ReSlaveESD copied from its ReSlave (or resampled
      // as it, without the full ReSlave): one copy launch for all pairs
      tops::RowCopy c;
      if (pair_first_burst_copy(P, &c)) {
        copies.push_back(c);
        jobs.erase(jobs.begin() + (long)n0);
      }
    } else {
      pair_rs1_jobs(P, jobs);
    }
    luts.resize(jobs.size(), P->lut);
  }
  if (!copies.empty()) {
    const int r = tops::row_copy(copies.data(), (int)copies.size(), st, launches);
    if (r != TOPS_OK) return r;
  }
  *launches += chunks(jobs.size(), 32);
  if (jobs.empty()) return TOPS_OK;
  return tops::resample_launch_multi(luts.data(), jobs.data(), (int)jobs.size(), B->o.precision,
                                     tile(B->tune.rs_seg_rows, B->tune.rs_persistent, counters),
                                     st);
}

int batch_coherence(tops_batch *B, int *counters, cudaStream_t st) {
  std::vector<tops_coh_job> cj;
  for (tops_pair *P : B->pairs) pair_coh_jobs(P, cj);
  tops::TileCfg cfg = tile(B->tune.coh_seg_rows, B->tune.coh_persistent, counters);
  cfg.compensated = B->o.compensated;
  return tops::coherence_launch(cj.data(), (int)cj.size(), B->o.win_rg, B->o.win_az, cfg, st);
}


}  // namespace

extern "C" {

int tops_batch_create(tops_pair *const *pairs, int n, tops_batch **out) {
  if (!pairs || n < 1 || !out) return TOPS_E_INVALID;
  for (int i = 0; i < n; i++) {
    const tops_pair *P = pairs[i];
    if (!P || !P->dem_set) return TOPS_E_INVALID;
    const tops_pair_opts &a = P->o, &b = pairs[0]->o;
    if (a.win_rg != b.win_rg || a.win_az != b.win_az || a.esd_threshold != b.esd_threshold ||
        a.precision != b.precision || a.compensated != b.compensated)
      return TOPS_E_INVALID;
    for (int k = 0; k < i; k++)
      if (pairs[k] == P) return TOPS_E_INVALID;
  }
  tops_batch *B = new tops_batch();
  auto fail = [&](int e) {
    delete B;
    return e;
  };
  B->pairs.assign(pairs, pairs + n);
  B->o = pairs[0]->o;
  memset(&B->tune, 0, sizeof(B->tune));
  std::vector<tops_geo_job> geo;
  std::vector<tops_esd_overlap> ovs;
  for (tops_pair *P : B->pairs) {
    geo.insert(geo.end(), P->geo.begin(), P->geo.end());
    B->ov_begin.push_back((int)ovs.size());
    pair_esd_overlaps(P, ovs);
  }
  B->n_ov = (int)ovs.size();
  void *v;
  int st;
  B->geo_scratch = tops_geocoreg_scratch_bytes(geo.data(), (int)geo.size());
  if ((st = B->alloc(&v, B->geo_scratch))) return fail(st);
  B->d_geo_scratch = v;
  if (B->n_ov > 0) {
    B->esd_scratch = tops_esd_scratch_bytes(ovs.data(), B->n_ov);
    if (B->esd_scratch == 0) return fail(TOPS_E_INVALID);
    if ((st = B->alloc(&v, B->esd_scratch))) return fail(st);
    B->d_esd_scratch = v;
  }
  if ((st = B->alloc(&v, sizeof(double) * (B->n_ov > 0 ? B->n_ov : 1)))) return fail(st);
  B->d_shift = static_cast<double *>(v);
  if ((st = B->alloc(&v, 2 * sizeof(double) * (B->n_ov > 0 ? B->n_ov : 1)))) return fail(st);
  B->d_sums = static_cast<double *>(v);
  if ((st = B->alloc(&v, sizeof(int) * kCounters))) return fail(st);
  B->d_counters = static_cast<int *>(v);
  *out = B;
  return TOPS_OK;
}

int tops_batch_destroy(tops_batch *B) {
  delete B;
  return TOPS_OK;
}

int tops_batch_set_tune(tops_batch *B, const tops_tune *t) {
  if (!B || !t) return TOPS_E_INVALID;
  if (t->rs_seg_rows < 0 || t->rs_seg_rows > 252 || (t->rs_seg_rows && t->rs_seg_rows < 12) ||
      t->coh_seg_rows < 0 || t->coh_seg_rows > 512 || (t->coh_seg_rows && t->coh_seg_rows < 8))
    return TOPS_E_INVALID;
  B->tune = *t;
  B->drop_graph();   // the graph holds the previous launch shapes
  return TOPS_OK;
}

int tops_batch_get_tune(const tops_batch *B, tops_tune *t) {
  if (!B || !t) return TOPS_E_INVALID;
  *t = B->tune;
  return TOPS_OK;
}

int tops_batch_run(tops_batch *B, void *stream) {
  if (!B) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int launches = 0;
  // 1. geometric coregistration of every burst of every pair
  std::vector<tops_geo_job> geo;
  for (tops_pair *P : B->pairs) geo.insert(geo.end(), P->geo.begin(), P->geo.end());
  B_TRY(tops_geocoreg(geo.data(), (int)geo.size(), B->d_geo_scratch, B->geo_scratch, stream));
  launches += 2 * chunks(geo.size(), 16);
  // 2. resample without shift
  size_t n_rs1 = 0;
  {
    std::vector<tops_resample_job> tmp;
    for (tops_pair *P : B->pairs) pair_rs1_jobs(P, tmp);
    n_rs1 = tmp.size();
  }
  int *ctr = B->d_counters;
  B_TRY(batch_resample(B, false, ctr, st, &launches));
  ctr += chunks(n_rs1, 32);
  // 3. ESD over all overlaps; every pair's shifts are also copied into its
  //    own plan (tops_pair_download reads them there)
  if (B->n_ov > 0) {
    std::vector<tops_esd_overlap> ovs;
    for (tops_pair *P : B->pairs) pair_esd_overlaps(P, ovs);
    B_TRY(tops::esd_launch(ovs.data(), B->n_ov, B->o.win_az, B->o.win_rg, B->o.esd_threshold, B->d_shift,
                   B->d_sums, B->d_esd_scratch, B->esd_scratch, B->o.compensated, static_cast<cudaStream_t>(stream)));
    launches += 2 * chunks(ovs.size(), 32);
    for (size_t p = 0; p < B->pairs.size(); p++) {
      tops_pair *P = B->pairs[p];
      if (P->nb > 1)
        B_CUDA(cudaMemcpyAsync(P->d_shift, B->d_shift + B->ov_begin[p],
                               sizeof(double) * (P->nb - 1), cudaMemcpyDeviceToDevice, st));
    }
  }
  // 4. resample with the ESD shifts
  size_t n_rs2 = 0;
  for (tops_pair *P : B->pairs) n_rs2 += P->nb;
  B_TRY(batch_resample(B, true, ctr, st, &launches));
  ctr += chunks(n_rs2, 32);
  // 5. coherence
  B_TRY(batch_coherence(B, ctr, st));
  launches += chunks(n_rs2, 32);
  ctr += chunks(n_rs2, 32);
  if (ctr - B->d_counters > kCounters) return TOPS_E_INVALID;
  B->n_launches = launches;
  return TOPS_OK;
}

int tops_batch_run_graph(tops_batch *B, void *stream) {
  if (!B) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!B->graph_exec) {
    // one eager run first: it sets per-kernel attributes outside the capture
    B_TRY(tops_batch_run(B, stream));
    if (!B->capture_stream)
      B_CUDA(cudaStreamCreateWithFlags(&B->capture_stream, cudaStreamNonBlocking));
    cudaStream_t cs = B->capture_stream;
    B_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int s = tops_batch_run(B, cs);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    if (s != TOPS_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    B_CUDA(e);
    B->graph = g;
    B_CUDA(cudaGraphInstantiate(&B->graph_exec, g, 0));
  }
  B_CUDA(cudaGraphLaunch(B->graph_exec, st));
  return TOPS_OK;
}

int tops_batch_launches(const tops_batch *B) { return B ? B->n_launches : -1; }

// Autotuner: times the resample (ESD pass) and coherence stages of this
// batch for every candidate tile -- rows per work item and grid-sized versus
// persistent work-queue scheduling -- with CUDA events on `stream`, and keeps
// the fastest of each.  Runs the whole batch once first so the stage inputs
// (offsets, ESD shifts) are valid.
int tops_batch_autotune(tops_batch *B, void *stream, tops_tune *best, double *best_ms) {
  if (!B) return TOPS_E_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  B->drop_graph();
  memset(&B->tune, 0, sizeof(B->tune));
  B_TRY(tops_batch_run(B, stream));
  cudaEvent_t e0, e1;
  B_CUDA(cudaEventCreate(&e0));
  B_CUDA(cudaEventCreate(&e1));
  auto time_stage = [&](bool resample, int seg, int pers, float &ms) -> int {
    tops_tune t = B->tune;
    if (resample) {
      t.rs_seg_rows = seg;
      t.rs_persistent = pers;
    } else {
      t.coh_seg_rows = seg;
      t.coh_persistent = pers;
    }
    const tops_tune keep = B->tune;
    B->tune = t;
    float acc = 0.f;
    int s = TOPS_OK, launches = 0;
    for (int rep = 0; rep < 3 && s == TOPS_OK; rep++) {   // rep 0 warms up
      if (cudaEventRecord(e0, st) != cudaSuccess) s = TOPS_E_CUDA;
      if (s == TOPS_OK)
        s = resample ? batch_resample(B, true, B->d_counters, st, &launches)
                     : batch_coherence(B, B->d_counters, st);
      if (s == TOPS_OK && cudaEventRecord(e1, st) != cudaSuccess) s = TOPS_E_CUDA;
      if (s == TOPS_OK && cudaEventSynchronize(e1) != cudaSuccess) s = TOPS_E_CUDA;
      float m = 0.f;
      if (s == TOPS_OK && cudaEventElapsedTime(&m, e0, e1) != cudaSuccess) s = TOPS_E_CUDA;
      if (rep > 0) acc += m;
    }
    B->tune = keep;
    ms = acc / 2.f;
    return s;
  };
  const int rs_seg[] = {84, 168, 252};
  const int coh_seg[] = {64, 128, 256, 512};
  float best_rs = 1e30f, best_coh = 1e30f;
  tops_tune bt;
  memset(&bt, 0, sizeof(bt));
  int s = TOPS_OK;
  for (int seg : rs_seg)
    for (int pers = 0; pers < 2 && s == TOPS_OK; pers++) {
      float ms = 0.f;
      s = time_stage(true, seg, pers, ms);
      if (s == TOPS_OK && ms < best_rs) {
        best_rs = ms;
        bt.rs_seg_rows = seg;
        bt.rs_persistent = pers;
      }
    }
  for (int seg : coh_seg)
    for (int pers = 0; pers < 2 && s == TOPS_OK; pers++) {
      float ms = 0.f;
      s = time_stage(false, seg, pers, ms);
      if (s == TOPS_OK && ms < best_coh) {
        best_coh = ms;
        bt.coh_seg_rows = seg;
        bt.coh_persistent = pers;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != TOPS_OK) return s;
  B->tune = bt;
  // restore every output with the chosen tiles
  B_TRY(tops_batch_run(B, stream));
  if (best) *best = bt;
  if (best_ms) {
    best_ms[0] = best_rs;
    best_ms[1] = best_coh;
  }
  return TOPS_OK;
}

}  // extern "C"

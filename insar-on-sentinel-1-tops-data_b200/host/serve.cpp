// serve.cpp -- the serving loop of tops_serve.h: HBM-budget admission over a
// device arena, one stream per slot, device-resident DEM tiles, shared LUTs.
#include <cuda_runtime.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <deque>
#include <map>
#include <tuple>
#include <vector>

#include "pair_impl.h"
#include "tops_serve.h"

namespace {

using Clock = std::chrono::steady_clock;

struct DemTile {
  float *d = nullptr;
  size_t pitch = 0;
  int lines = 0, pixels = 0;
  double lat0 = 0, lon0 = 0, dlat = 0, dlon = 0;
};

struct Job {
  long id = 0;
  tops_job_desc desc;
  size_t footprint = 0;
  int status = TOPS_OK;
  double arrival = 0, admit = -1;
  std::atomic<double> done{-1.0};   // written by the stream callback
  tops_pair *P = nullptr;
  Clock::time_point t0;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  Job *job = nullptr;
  // pinned staging of the small outputs: a copy into pageable memory would
  // make the enqueue wait for the whole job
  double *h_cpm = nullptr, *h_shift = nullptr;
};

using LutKey = std::tuple<double, double, double>;

// Stream callback after a job's last download: its completion time.
void CUDART_CB mark_done(void *p) {
  Job *j = static_cast<Job *>(p);
  j->done.store(std::chrono::duration<double>(Clock::now() - j->t0).count());
}

}  // namespace

struct tops_server {
  tops_server_cfg cfg{};
  void *d_base = nullptr;
  Arena *arena = nullptr;
  std::vector<Slot> slots;
  std::deque<Job *> queue;
  std::vector<tops_job_done> finished;
  std::vector<DemTile> dems;
  std::map<LutKey, tops_lut_dev *> luts;
  Clock::time_point t0 = Clock::now();
  long next_id = 1;
  tops_server_stats st{};

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  void finish(Job *j, int status, double done_s) {
    tops_job_done d;
    d.job_id = j->id;
    d.status = status;
    d.arrival_s = j->arrival;
    d.admit_s = j->admit;
    d.done_s = done_s;
    d.footprint = j->footprint;
    finished.push_back(d);
    if (status == TOPS_OK)
      st.completed++;
    else
      st.rejected++;
    delete j;
  }

  int lut_for(const tops_swath_info &m, tops_lut_dev **out) {
    const LutKey k(m.prf, m.az_bandwidth, m.rsr);
    auto it = luts.find(k);
    if (it != luts.end()) {
      *out = it->second;
      return TOPS_OK;
    }
    std::vector<float> kaz(2048 * 12), krg(2048 * 12);
    int s = tops_lut(12, m.prf, m.az_bandwidth, 2 * m.rsr, kaz.data(), krg.data());
    if (s != TOPS_OK) return s;
    tops_lut_dev *L = nullptr;
    if ((s = tops_lut_create(kaz.data(), krg.data(), &L)) != TOPS_OK) return s;
    luts[k] = L;
    *out = L;
    return TOPS_OK;
  }

  // Enqueues the whole job on the slot's stream; TOPS_E_NOMEM: does not fit
  // the free arena now (nothing is left allocated).
  int launch(Job *j, Slot &s) {
    const tops_job_desc &d = j->desc;
    if (d.dem_id < 0 || d.dem_id >= (int)dems.size()) return TOPS_E_INVALID;
    tops_lut_dev *lut = nullptr;
    int r = lut_for(d.master, &lut);
    if (r != TOPS_OK) return r;
    tops_pair *P = nullptr;
    r = pair_create(&d.master, &d.slave, &d.opts, 0, 0, arena, lut, s.stream, true, &P);
    if (r != TOPS_OK) return r;
    const DemTile &t = dems[d.dem_id];
    if ((r = pair_bind_dem(P, t.d, t.pitch, t.lines, t.pixels, t.lat0, t.lon0, t.dlat, t.dlon,
                           d.windows)) != TOPS_OK ||
        (r = tops_pair_upload(P, d.master_slc, d.slave_slc, s.stream)) != TOPS_OK ||
        (r = tops_pair_run(P, s.stream)) != TOPS_OK ||
        (r = tops_pair_download(P, d.reslave, d.reslave_esd, d.coh, s.h_cpm, s.h_shift,
                                s.stream)) != TOPS_OK) {
      // nothing may still read the plan's memory before it is released
      cudaStreamSynchronize(s.stream);
      delete P;
      return r;
    }
    j->t0 = t0;
    if (cudaLaunchHostFunc(s.stream, mark_done, j) != cudaSuccess ||
        cudaEventRecord(s.ev, s.stream) != cudaSuccess) {
      cudaStreamSynchronize(s.stream);
      delete P;
      return TOPS_E_CUDA;
    }
    j->P = P;
    return TOPS_OK;
  }

  int progress() {
    // retire finished jobs; their plans' blocks go back to the arena
    for (Slot &s : slots) {
      if (!s.job) continue;
      const cudaError_t e = cudaEventQuery(s.ev);
      if (e == cudaErrorNotReady) continue;
      Job *j = s.job;
      s.job = nullptr;
      st.running--;
      if (e != cudaSuccess) {
        (void)cudaGetLastError();
        cudaStreamSynchronize(s.stream);
      }
      double done = j->done.load();
      if (done < 0) done = now();
      const int nb = j->desc.master.n_bursts;
      if (e == cudaSuccess && j->desc.cpm)
        memcpy(j->desc.cpm, s.h_cpm, sizeof(double) * 12 * nb);
      if (e == cudaSuccess && j->desc.shifts && nb > 1)
        memcpy(j->desc.shifts, s.h_shift, sizeof(double) * (nb - 1));
      delete j->P;
      j->P = nullptr;
      finish(j, e == cudaSuccess ? TOPS_OK : TOPS_E_CUDA, done);
    }
    // admit queued jobs in arrival order while a slot is free and they fit
    while (!queue.empty()) {
      Job *j = queue.front();
      if (j->footprint > arena->capacity()) {
        queue.pop_front();
        st.queued--;
        finish(j, TOPS_E_BUDGET, now());
        continue;
      }
      Slot *free_slot = nullptr;
      for (Slot &s : slots)
        if (!s.job) {
          free_slot = &s;
          break;
        }
      if (!free_slot) break;
      j->admit = now();
      const int r = launch(j, *free_slot);
      if (r == TOPS_E_NOMEM) {
        bool running = false;
        for (Slot &s : slots) running = running || s.job != nullptr;
        if (running) {   // wait until running jobs release memory
          j->admit = -1;
          break;
        }
        // nothing runs, yet the job does not fit: its buffers do not fit
        // even the empty arena, so it never will -- end it now rather than
        // leave the queue stalled behind it
        queue.pop_front();
        st.queued--;
        finish(j, TOPS_E_NOMEM, now());
        continue;
      }
      queue.pop_front();
      st.queued--;
      if (r != TOPS_OK) {
        finish(j, r, now());
        continue;
      }
      free_slot->job = j;
      st.admitted++;
      st.running++;
      const size_t used = arena->in_use();
      if (used > st.hbm_peak) st.hbm_peak = used;
    }
    st.hbm_in_use = arena->in_use();
    return TOPS_OK;
  }
};

extern "C" {

size_t tops_server_job_footprint(const tops_job_desc *job) {
  if (!job) return 0;
  return tops_pair_footprint(&job->master, &job->opts, 0, 0);
}

int tops_server_create(const tops_server_cfg *cfg, tops_server **out) {
  if (!cfg || !out || cfg->slots < 1 || cfg->slots > 64 || cfg->hbm_budget < Arena::kAlign)
    return TOPS_E_INVALID;
  tops_server *S = new tops_server();
  S->cfg = *cfg;
  if (cudaMalloc(&S->d_base, cfg->hbm_budget) != cudaSuccess) {
    (void)cudaGetLastError();
    delete S;
    return TOPS_E_NOMEM;
  }
  S->arena = new Arena(reinterpret_cast<uintptr_t>(S->d_base), cfg->hbm_budget);
  S->slots.resize(cfg->slots);
  for (Slot &s : S->slots) {
    if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&s.h_cpm, sizeof(double) * 12 * TOPS_MAX_BURSTS) != cudaSuccess ||
        cudaMallocHost(&s.h_shift, sizeof(double) * TOPS_MAX_BURSTS) != cudaSuccess) {
      (void)cudaGetLastError();
      tops_server_destroy(S);
      return TOPS_E_CUDA;
    }
  }
  *out = S;
  return TOPS_OK;
}

int tops_server_destroy(tops_server *S) {
  if (!S) return TOPS_OK;
  if (S->arena) tops_server_drain(S);
  for (Job *j : S->queue) delete j;
  for (Slot &s : S->slots) {
    if (s.stream) cudaStreamDestroy(s.stream);
    if (s.ev) cudaEventDestroy(s.ev);
    if (s.h_cpm) cudaFreeHost(s.h_cpm);
    if (s.h_shift) cudaFreeHost(s.h_shift);
  }
  for (auto &kv : S->luts) tops_lut_destroy(kv.second);
  for (DemTile &t : S->dems) cudaFree(t.d);
  delete S->arena;
  if (S->d_base) cudaFree(S->d_base);
  delete S;
  return TOPS_OK;
}

int tops_server_add_dem(tops_server *S, const float *dem, int lines, int pixels, double lat0,
                        double lon0, double dlat, double dlon, int *dem_id) {
  if (!S || !dem || lines < 1 || pixels < 1 || !dem_id) return TOPS_E_INVALID;
  DemTile t;
  t.lines = lines;
  t.pixels = pixels;
  t.lat0 = lat0;
  t.lon0 = lon0;
  t.dlat = dlat;
  t.dlon = dlon;
  if (cudaMallocPitch(&t.d, &t.pitch, (size_t)pixels * sizeof(float), lines) != cudaSuccess) {
    (void)cudaGetLastError();
    return TOPS_E_NOMEM;
  }
  if (cudaMemcpy2D(t.d, t.pitch, dem, (size_t)pixels * sizeof(float), (size_t)pixels * 4, lines,
                   cudaMemcpyHostToDevice) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(t.d);
    return TOPS_E_CUDA;
  }
  S->dems.push_back(t);
  *dem_id = (int)S->dems.size() - 1;
  return TOPS_OK;
}

int tops_server_submit(tops_server *S, const tops_job_desc *job, long *job_id) {
  if (!S || !job || !job->master_slc || !job->slave_slc || !job->reslave_esd || !job->coh)
    return TOPS_E_INVALID;
  Job *j = new Job();
  j->id = S->next_id++;
  j->desc = *job;
  j->arrival = S->now();
  j->footprint = tops_server_job_footprint(job);
  if (j->footprint == 0) {
    delete j;
    return TOPS_E_INVALID;
  }
  S->queue.push_back(j);
  S->st.submitted++;
  S->st.queued++;
  if (job_id) *job_id = j->id;
  return S->progress();
}

int tops_server_progress(tops_server *S) { return S ? S->progress() : TOPS_E_INVALID; }

int tops_server_poll(tops_server *S, tops_job_done *done, int max, int *n_done) {
  if (!S || (!done && max > 0) || max < 0 || !n_done) return TOPS_E_INVALID;
  S->progress();
  const int n = (int)S->finished.size() < max ? (int)S->finished.size() : max;
  for (int i = 0; i < n; i++) done[i] = S->finished[i];
  S->finished.erase(S->finished.begin(), S->finished.begin() + n);
  *n_done = n;
  return TOPS_OK;
}

int tops_server_drain(tops_server *S) {
  if (!S) return TOPS_E_INVALID;
  for (;;) {
    S->progress();
    Slot *busy = nullptr;
    for (Slot &s : S->slots)
      if (s.job) {
        busy = &s;
        break;
      }
    if (!busy) {
      if (S->queue.empty()) return TOPS_OK;
      // nothing runs, yet the head job could not start: its buffers do not
      // fit even the empty arena, so it never will -- end it
      Job *j = S->queue.front();
      S->queue.pop_front();
      S->st.queued--;
      S->finish(j, TOPS_E_NOMEM, S->now());
      continue;
    }
    cudaEventSynchronize(busy->ev);
  }
}

int tops_server_get_stats(const tops_server *S, tops_server_stats *st) {
  if (!S || !st) return TOPS_E_INVALID;
  *st = S->st;
  st->hbm_in_use = S->arena->in_use();
  return TOPS_OK;
}

// ------------------------------------------------------------ arena (tests)
struct tops_arena {
  Arena a;
  tops_arena(size_t base, size_t bytes) : a(base, bytes) {}
};

int tops_arena_create(size_t base, size_t bytes, tops_arena **out) {
  if (!out || bytes < Arena::kAlign || base % Arena::kAlign) return TOPS_E_INVALID;
  *out = new tops_arena(base, bytes);
  return TOPS_OK;
}
int tops_arena_destroy(tops_arena *a) {
  delete a;
  return TOPS_OK;
}
size_t tops_arena_alloc(tops_arena *a, size_t bytes) { return a ? a->a.alloc(bytes) : 0; }
int tops_arena_release(tops_arena *a, size_t addr) {
  return (a && a->a.release(addr)) ? TOPS_OK : TOPS_E_INVALID;
}
size_t tops_arena_in_use(const tops_arena *a) { return a ? a->a.in_use() : 0; }
size_t tops_arena_largest_free(const tops_arena *a) { return a ? a->a.largest_free() : 0; }
int tops_arena_free_ranges(const tops_arena *a) { return a ? a->a.free_ranges() : -1; }

}  // extern "C"

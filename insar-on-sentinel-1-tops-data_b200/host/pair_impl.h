// pair_impl.h -- library-internal layout of a burst-pair plan (tops_pair)
// and the stage job lists built from it; shared by the single-pair run
// (pipeline.cpp) and the batched plans (batch.cpp).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "arena.h"
#include "launch.h"
#include "tops_pipeline.h"

// Coherence launch controls of a plan: the default tile, the accumulation
// mode of its options.
inline tops::TileCfg coh_cfg(const tops_pair_opts &o) {
  tops::TileCfg c;
  c.compensated = o.compensated;
  return c;
}

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct OrbitFit {
  double cx[8], cy[8], cz[8];
  int n = 0;
};

struct Deramp {
  std::vector<double> dc, fm, tref, kt;
};

struct tops_pair {
  tops_swath_info m, s;
  tops_pair_opts o;
  int nb, L, W, dem_lines, dem_pixels;
  OrbitFit fm, fs;
  Deramp dm, ds;
  std::vector<float> kaz, krg;
  std::vector<int> ov;
  std::vector<int> ov_off;  // line offset of each overlap in the band buffers
  int ov_total = 0;
  double spec_sep = 0;
  // device memory
  size_t slc_pitch = 0, cplx_pitch = 0, coh_pitch = 0, dem_pitch = 0;
  char *d_master = nullptr, *d_slave = nullptr, *d_reslave = nullptr, *d_res_esd = nullptr;
  char *d_fwd = nullptr, *d_back = nullptr;  // overlap bands when !reslave_full
  float *d_coh = nullptr, *d_dem = nullptr;
  double *d_kt = nullptr, *d_tref = nullptr, *d_fdc = nullptr;
  double *d_cpm = nullptr, *d_shift = nullptr, *d_sums = nullptr;
  int *d_status = nullptr;
  void *d_geo_scratch = nullptr, *d_esd_scratch = nullptr;
  size_t geo_scratch = 0, esd_scratch = 0;
  tops_lut_dev *lut = nullptr;
  std::vector<tops_geo_job> geo;
  bool dem_set = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t capture_stream = nullptr;  // private: the legacy stream cannot be captured
  // copy streams and per-burst events of the pipelined host-to-host run
  cudaStream_t s_up = nullptr, s_down = nullptr;
  std::vector<cudaEvent_t> pev;
  // coherence stream and per-burst events of the overlapped ReSlaveESD tail
  cudaStream_t s_coh = nullptr;
  std::vector<cudaEvent_t> cev;
  std::vector<void *> allocs;
  int n_launches = 0;
  Arena *arena = nullptr;      // if set, device buffers come from it (no cudaMalloc)
  bool lut_owned = true;       // false: a LUT shared by several plans

  int alloc(void **p, size_t bytes) {
    if (arena) {
      const uintptr_t a = arena->alloc(bytes);
      if (!a) return TOPS_E_NOMEM;
      *p = reinterpret_cast<void *>(a);
    } else {
      cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
      if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? TOPS_E_NOMEM : TOPS_E_CUDA;
    }
    allocs.push_back(*p);
    return TOPS_OK;
  }
  ~tops_pair() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    if (s_up) cudaStreamDestroy(s_up);
    if (s_down) cudaStreamDestroy(s_down);
    if (s_coh) cudaStreamDestroy(s_coh);
    for (cudaEvent_t e : pev) cudaEventDestroy(e);
    for (cudaEvent_t e : cev) cudaEventDestroy(e);
    for (void *p : allocs) {
      if (arena)
        arena->release(reinterpret_cast<uintptr_t>(p));
      else
        cudaFree(p);
    }
    if (lut && lut_owned) tops_lut_destroy(lut);
  }
};

// Plan creation with its options for the serving loop: device buffers from
// `arena` (or cudaMalloc when null), an optional LUT shared by several plans,
// no DEM buffer when dem_lines == 0 (a device-resident tile is bound with
// pair_bind_dem), and the deramp rows copied on `stream` (null: synchronous).
int pair_create(const tops_swath_info *m, const tops_swath_info *s, const tops_pair_opts *o,
                int dem_lines, int dem_pixels, Arena *arena, tops_lut_dev *shared_lut,
                cudaStream_t stream, bool async_copy, tops_pair **out);
// Geocoreg jobs of every burst on a device DEM (float heights, byte pitch).
int pair_bind_dem(tops_pair *P, const float *d_dem, size_t dem_pitch, int dem_lines,
                  int dem_pixels, double lat0, double lon0, double dlat, double dlon,
                  const tops_dem_window *win);

// Stage job lists of one pair, in the reference drivers' order
// (Func.cpp:2215-2763).  `shifts` is the device array holding this pair's ESD
// shifts, one per overlap.
void pair_rs1_jobs(const tops_pair *P, std::vector<tops_resample_job> &jobs);
void pair_esd_overlaps(const tops_pair *P, std::vector<tops_esd_overlap> &ovs);
// With the full ReSlave computed, the first burst's ReSlaveESD is a copy of
// its ReSlave: fills *c and returns 1 (the first rs2 job is then skipped);
// else 0.
int pair_first_burst_copy(const tops_pair *P, tops::RowCopy *c);
void pair_rs2_jobs(const tops_pair *P, const double *shifts,
                   std::vector<tops_resample_job> &jobs);
void pair_coh_jobs(const tops_pair *P, std::vector<tops_coh_job> &cj);

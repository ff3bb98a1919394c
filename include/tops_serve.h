/* tops_serve.h -- serving loop for burst-pair jobs (no counterpart in the
 * reference, whose stage drivers process one product per run).
 *
 * Jobs of different sizes arrive one at a time (tops_server_submit).  The
 * server reserves its HBM budget once and carves each job's buffers out of it
 * (a first-fit arena, so no cudaMalloc / cudaFree runs while jobs are in
 * flight); a job is admitted, in arrival order, as soon as a slot (a stream)
 * is free and its footprint fits the free memory.  An admitted job runs on
 * its own stream -- upload of both SLCs, every stage of the device-resident
 * plan, download of the outputs -- so jobs that arrive while others are on
 * the GPU overlap with them: copies of one job run beside kernels of
 * another.  DEM tiles are uploaded once (tops_server_add_dem) and stay on the
 * device; LUTs are shared by the jobs of equal annotation parameters; orbit
 * fits and deramp rows are computed per job on the host.
 *
 * The API is single-threaded: the caller drives it (submit, progress, poll).
 * Times are seconds since the server was created (host steady clock). */
#ifndef TOPS_SERVE_H
#define TOPS_SERVE_H

#include "tops_pipeline.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tops_server tops_server;

typedef struct {
  size_t hbm_budget;   /* bytes of device memory the jobs may hold at once */
  int slots;           /* jobs in flight at most (one stream each), 1..64 */
} tops_server_cfg;

/* One job: a burst-pair plan's inputs and where its outputs go.  The swath
 * descriptions and windows are copied at submit; the host buffers must stay
 * valid until the job is reported done.  The SLC and image buffers should be
 * pinned: a copy between the device and pageable memory makes the enqueue
 * wait for the job's stream, which serialises the jobs.  cpm and shifts are
 * staged through the server's own pinned memory and copied at completion. */
typedef struct {
  tops_swath_info master, slave;
  tops_pair_opts opts;
  int dem_id;                                /* from tops_server_add_dem */
  tops_dem_window windows[TOPS_MAX_BURSTS];  /* one per burst, in the tile */
  const void *master_slc, *slave_slc;        /* CInt16 [n_bursts*lines][samples] */
  void *reslave;                             /* complex64, may be NULL */
  void *reslave_esd;                         /* complex64 */
  float *coh;                                /* float */
  double *cpm;                               /* [n_bursts][12], may be NULL */
  double *shifts;                            /* [n_bursts-1], may be NULL */
} tops_job_desc;

typedef struct {
  long job_id;
  int status;          /* TOPS_OK, or the error that ended the job */
  double arrival_s;    /* submit */
  double admit_s;      /* slot and memory granted, work enqueued */
  double done_s;       /* outputs in host memory */
  size_t footprint;    /* device bytes the job held */
} tops_job_done;

typedef struct {
  long submitted, admitted, completed, rejected, queued, running;
  size_t hbm_in_use, hbm_peak;
} tops_server_stats;

int tops_server_create(const tops_server_cfg *cfg, tops_server **out);
int tops_server_destroy(tops_server *srv);   /* waits for the jobs in flight */

/* Uploads a DEM tile (host float heights) once; jobs refer to it by id. */
int tops_server_add_dem(tops_server *srv, const float *dem, int lines, int pixels, double lat0,
                        double lon0, double dlat, double dlon, int *dem_id);

/* Queues a job (its arrival time is now) and makes progress.  A job whose
 * footprint exceeds the whole budget is reported done with TOPS_E_BUDGET. */
int tops_server_submit(tops_server *srv, const tops_job_desc *job, long *job_id);

/* Non-blocking: retires finished jobs and admits queued ones. */
int tops_server_progress(tops_server *srv);

/* Moves up to `max` finished jobs into `done` (after a progress step). */
int tops_server_poll(tops_server *srv, tops_job_done *done, int max, int *n_done);

/* Blocks until every submitted job is done (finished jobs stay pollable). */
int tops_server_drain(tops_server *srv);

int tops_server_get_stats(const tops_server *srv, tops_server_stats *stats);

/* Device bytes one job needs (its plan's footprint, no DEM). */
size_t tops_server_job_footprint(const tops_job_desc *job);

/* The arena allocator of the server, exposed for tests: address arithmetic
 * only, over any base value (no device memory is touched). */
typedef struct tops_arena tops_arena;
int tops_arena_create(size_t base, size_t bytes, tops_arena **out);
int tops_arena_destroy(tops_arena *a);
size_t tops_arena_alloc(tops_arena *a, size_t bytes);   /* 0: no room */
int tops_arena_release(tops_arena *a, size_t addr);
size_t tops_arena_in_use(const tops_arena *a);
size_t tops_arena_largest_free(const tops_arena *a);
int tops_arena_free_ranges(const tops_arena *a);

#ifdef __cplusplus
}
#endif
#endif

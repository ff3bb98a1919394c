/*
 * tops_pipeline.h -- burst-pair processing of one master/slave sub-swath.
 *
 * The reference runs its stages per burst from host drivers (Func.cpp:
 * GeometricCoreg 2215-2297, DerampAndResample 2326-2406, ESDAndCoh
 * 2496-2763), round-tripping every intermediate through host memory and
 * GeoTIFF files.  Two forms are provided here:
 *
 *  - tops_plain_pair(): the reference's driver sequence, per burst, through
 *    the reference-compatible entry points with host buffers (the "plain"
 *    form; same dataflow and ordering as the reference).
 *
 *  - tops_pair_*: a device-resident plan.  All inputs, intermediates and
 *    outputs stay in HBM; each stage is one batched launch over all bursts;
 *    the offset polynomials and ESD shifts flow from kernel to kernel through
 *    device memory, so a whole sub-swath pair is a fixed, host-sync-free
 *    sequence of launches that can be captured in one CUDA graph.
 *
 * Dataflow (both forms): geometric coregistration of every burst ->
 * resample every burst (ReSlave) -> ESD over the burst overlaps -> resample
 * bursts after the first with the ESD shift of the preceding overlap
 * (ReSlaveESD; the first burst is not corrected, Func.cpp:2653-2674) ->
 * coherence of master vs ReSlaveESD.
 */
#ifndef TOPS_PIPELINE_H
#define TOPS_PIPELINE_H

#include "tops_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int win_rg, win_az;       /* coherence / ESD window (reference: 24 x 6) */
  float esd_threshold;      /* ESD coherence threshold (reference: 0.3) */
  int reslave_full;         /* 1: ReSlave for every line (reference output);
                               0: only the overlap bands ESD needs */
  int burst0_deramp_rows;   /* 1: deramp rows of burst 0 for every burst, as
                               the reference passes them (Func.cpp:2383) */
  int precision;            /* resample deramp phase: TOPS_PREC_SPLIT (default)
                               or TOPS_PREC_FP64 */
  int compensated;          /* 1: ESD phasor sums with Kahan compensation and
                               coherence window sums without the sliding
                               update (pairwise per output); 0 (default): the
                               plain fixed-order FP32 sums */
  int coh_overlap;          /* 1: the ReSlaveESD resample in up to 3 chunks of
                               bursts, the coherence of each chunk on a second
                               stream as soon as it is resampled, overlapping
                               the resampling of the next chunk (same kernels,
                               same outputs);
                               0 (default): after the whole ReSlaveESD launch */
} tops_pair_opts;

int tops_pair_opts_default(tops_pair_opts *o);

/* DEM window [row0, row0+rows) x [col0, col0+cols) of one burst. */
typedef struct { int row0, col0, rows, cols; } tops_dem_window;

typedef struct tops_pair tops_pair;

/* Device bytes a plan allocates (for HBM-budget admission). */
size_t tops_pair_footprint(const tops_swath_info *master, const tops_pair_opts *o, int dem_lines,
                           int dem_pixels);

/* Create a plan: host precomputes (orbit fits, deramp parameters, LUT,
 * overlaps, spectral separation) and every device buffer. */
int tops_pair_create(const tops_swath_info *master, const tops_swath_info *slave,
                     const tops_pair_opts *o, int dem_lines, int dem_pixels, tops_pair **out);
int tops_pair_destroy(tops_pair *p);

/* DEM heights (host float [dem_lines][dem_pixels]), geotransform and one
 * window per burst.  Asynchronous on `stream`. */
int tops_pair_set_dem(tops_pair *p, const float *dem, double lat0, double lon0, double dlat,
                      double dlon, const tops_dem_window *windows, void *stream);

/* Upload the burst-stacked CInt16 SLCs [n_bursts*lines][samples] (host;
 * pinned memory gives full-bandwidth asynchronous copies). */
int tops_pair_upload(tops_pair *p, const void *master, const void *slave, void *stream);

/* All stages on the device, enqueued on `stream` without host sync. */
int tops_pair_run(tops_pair *p, void *stream);

/* The stages of tops_pair_run timed with CUDA events on `stream` (waits
 * for them): ms[0..4] = geocoreg, ReSlave resample, ESD, ReSlaveESD
 * resample, coherence. */
int tops_pair_stage_times(tops_pair *p, void *stream, float *ms);

/* Same, as one CUDA graph (captured on first use, then replayed). */
int tops_pair_run_graph(tops_pair *p, void *stream);

/* Copy results to the host (NULL skips an output): ReSlave (complex64, only
 * with reslave_full), ReSlaveESD (complex64), coherence (float)
 * [n_bursts*lines][samples]; cpm [n_bursts][12]; shifts [n_bursts-1]. */
int tops_pair_download(tops_pair *p, void *reslave, void *reslave_esd, float *coh, double *cpm,
                       double *shifts, void *stream);

/* Host to host in one call: uploads the SLCs, runs every stage and
 * downloads the outputs, pipelined per burst -- the copies of one burst
 * overlap the kernels of the others, and uploads overlap downloads.  Host
 * buffers as tops_pair_upload / tops_pair_download (pinned memory; pageable
 * buffers make the copies synchronous).  Everything is enqueued behind
 * `stream`'s earlier work; synchronise `stream` for the results.  Same
 * outputs as upload + run + download. */
int tops_pair_process(tops_pair *p, const void *master, const void *slave, void *reslave,
                      void *reslave_esd, float *coh, double *cpm, double *shifts, void *stream);

typedef struct {
  void *master, *slave;            /* CInt16, pitch slc_pitch */
  void *reslave, *reslave_esd;     /* complex64, pitch cplx_pitch */
  float *coh;                      /* pitch coh_pitch */
  double *cpm, *shifts;
  int *geo_status;
  size_t slc_pitch, cplx_pitch, coh_pitch;
  int n_bursts, lines, samples;
  int n_launches;                  /* kernels one tops_pair_run launches */
} tops_pair_buffers;

int tops_pair_buffers_get(const tops_pair *p, tops_pair_buffers *b);

/* Reference-shaped per-burst processing through the reference-compatible
 * entry points (host buffers).  dem_int: int heights of the full DEM;
 * outputs as tops_pair_download. */
int tops_plain_pair(const tops_swath_info *master, const tops_swath_info *slave,
                    const tops_pair_opts *o, const int *dem_int, int dem_lines, int dem_pixels,
                    double lat0, double lon0, double dlat, double dlon,
                    const tops_dem_window *windows, const void *master_slc,
                    const void *slave_slc, void *reslave, void *reslave_esd, float *coh,
                    double *cpm, double *shifts);

/* Every stage launched once per burst (or overlap), as the reference's
 * drivers call their stages, on device-resident data: the per-burst launch
 * loop that the batched forms are compared with.  Same outputs as
 * tops_pair_run. */
int tops_pair_run_per_burst(tops_pair *p, void *stream);

/* ================================================= config.txt-driven run
 * The reference's main program (Main.cpp:11-150) on this library: reads
 * config.txt (tops_config_read: the reference's keys plus the synthetic-scene
 * keys), and for each sub-swath firstsubswath..lastsubswath processes bursts
 * burst0..burstN (1-based) with the device-resident plan and writes
 * <process_dir>/ReSlave-N.tif, ReSlaveESD-N.tif and Coh-N.tif (TIFF rasters,
 * CFloat32 / Float32) -- plus CohStitch-N.tif, the debursted coherence, when
 * the config sets stitch=1 (the reference's stitching step is disabled).
 * With masterpath / slavepath naming SAFE directories, each sub-swath's
 * inputs are read from them (the annotation file whose name holds
 * "-iwN-" and "-slc-<polarisation>", and the measurement raster of the same
 * name), from preciseOrbitMaster /
 * preciseOrbitSlave (the state vectors around the product's first
 * sub-swath) and from SpecificDemPath (an int16 or float32 GeoTIFF); the
 * master's bursts burst0..burstN are matched on the slave
 * (tops_s1_burst_overlap) and each burst's DEM window is its lat/lon box
 * plus 24 DEM pixels.  With masterpath empty or "(synthetic)", the inputs
 * come from the seeded synthetic generator (sub-swath N: seed +
 * 1000 (N - 1)).  Returns TOPS_E_CONFIG for a malformed or unsupported
 * config (npoints other than 12, empty ranges) or missing product files. */
typedef struct {
  int subswaths, burst_pairs;   /* processed */
  double seconds;               /* wall time of the run: loading, processing and writing,
                                   overlapped across sub-swaths */
  double shifts[TOPS_MAX_BURSTS];   /* ESD shifts of the last sub-swath */
  double load_seconds;          /* summed wall times of the sub-swath loads (reader thread) */
  double process_seconds;       /* summed wall times of the sub-swath pair runs, staging
                                   copies and device work included (main thread) */
  double write_seconds;         /* summed wall times of the output writes (writer thread);
                                   seconds < load + process + write shows the overlap */
} tops_run_stats;

int tops_run_config(const char *config_path, tops_run_stats *stats);

/* ============================================== batched sub-swath pairs
 * Several plans -- e.g. the 3 sub-swaths of a product, whose bursts differ in
 * lines and samples -- processed together: one launch per stage for all
 * their bursts (each job keeps its own boxes, LUT and polynomials), the
 * resample and coherence kernels optionally persistent over a work queue,
 * and the whole batch capturable as one CUDA graph.  The plans must have
 * their DEM set and share the window, threshold and precision options; they
 * stay owned by the caller, and their outputs are read with
 * tops_pair_download as usual. */
typedef struct tops_batch tops_batch;

/* Tile and scheduling of the resample and coherence launches. */
typedef struct {
  int rs_seg_rows;      /* resample output rows per work item, 12..252 (0: 252) */
  int rs_persistent;    /* 1: persistent kernel pulling items from a queue */
  int coh_seg_rows;     /* coherence rows per work item, 8..512 (0: 128) */
  int coh_persistent;
} tops_tune;

int tops_batch_create(tops_pair *const *pairs, int n_pairs, tops_batch **out);
int tops_batch_destroy(tops_batch *b);
int tops_batch_run(tops_batch *b, void *stream);
int tops_batch_run_graph(tops_batch *b, void *stream);
/* Kernels the last tops_batch_run launched. */
int tops_batch_launches(const tops_batch *b);
int tops_batch_set_tune(tops_batch *b, const tops_tune *t);
int tops_batch_get_tune(const tops_batch *b, tops_tune *t);
/* Times every candidate tile of the resample and coherence stages on this
 * batch (CUDA events on `stream`, synchronous) and keeps the fastest; best_ms
 * (optional, 2 doubles) receives the two stage times. */
int tops_batch_autotune(tops_batch *b, void *stream, tops_tune *best, double *best_ms);

#ifdef __cplusplus
}
#endif
#endif

/*
 * tops_synth.h -- seeded synthetic Sentinel-1 TOPS burst pairs.
 *
 * Stands in for real SAFE products, precise orbits and SRTM tiles (which
 * this processor's reference reads with tinyxml2/GDAL): it produces, from
 * one seed, everything the four stages consume.
 *
 *   orbits   circular 693 km orbit (17 state vectors, 10 s apart) for the
 *            master; the slave orbit is the master's shifted along track by
 *            `along_track_s` and offset by a perpendicular/parallel baseline
 *   DEM      fractional Brownian surface (Hurst exponent), float32 heights
 *   TOPS     burst timing with `overlap_lines` overlap, S1-like Doppler
 *            centroid and FM-rate polynomial lists, steering rate
 *   SLCs     master: band-limited circular Gaussian reflectivity with the
 *            TOPS azimuth ramp; slave: the same scene seen from the slave
 *            orbit (geocoded through the DEM): each ground point keeps the
 *            Doppler history it has in the master burst, plus the
 *            topographic phase and an optional azimuth misregistration of
 *            `az_shift_true` lines (what ESD must measure)
 *
 * All arrays are host memory owned by the scene object.
 */
#ifndef TOPS_SYNTH_H
#define TOPS_SYNTH_H

#include <stdint.h>

#include "tops_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define TOPS_SYNTH_MAX_BURSTS TOPS_MAX_BURSTS

typedef struct {
  long seed;
  int n_bursts, lines_per_burst, samples_per_burst, overlap_lines;
  double sigma_dn;          /* rms |reflectivity| in DN (I and Q each sigma/sqrt 2) */
  double wavelength;        /* m */
  double dt;                /* azimuth time interval, s */
  double rsr;               /* range sampling rate, Hz */
  double steering_rate_deg; /* deg/s */
  double az_bandwidth;      /* azimuth processing bandwidth, Hz */
  double rg_bandwidth;      /* range bandwidth, Hz */
  double altitude;          /* m */
  double inc_mid_deg;       /* incidence angle at mid swath */
  double lat_center_deg;
  int dem_lines, dem_pixels;
  double hurst, h_min, h_max;
  double dem_spacing_arcsec;  /* requested; stretched if the swath would not fit */
  double bperp, bpar;         /* baseline components, m */
  double along_track_s;       /* slave orbit time shift, s */
  double az_shift_true;       /* injected slave misregistration, lines */
  int topo_phase;             /* 1: add the topographic phase to the slave */
  int interp_taps;            /* slave interpolator taps (even, <= 32) */
  int threads;                /* OpenMP threads (0 = default) */
} tops_synth_cfg;


typedef struct {
  int lines, pixels;
  double lat0, lon0, dlat, dlon;   /* degrees; row r is lat0 - r*dlat */
} tops_dem_info;

typedef struct tops_scene tops_scene;

int tops_synth_defaults(tops_synth_cfg *cfg);
int tops_synth_create(const tops_synth_cfg *cfg, tops_scene **out);
void tops_synth_destroy(tops_scene *s);

/* which = 0 master, 1 slave */
int tops_synth_swath(const tops_scene *s, int which, tops_swath_info *info);
/* CInt16 [n_bursts*lines_per_burst][samples_per_burst], burst-stacked */
const int16_t *tops_synth_slc(const tops_scene *s, int which);
const float *tops_synth_dem(const tops_scene *s, tops_dem_info *info);
/* DEM window of one master burst: its lat/lon box extended by `margin` DEM
 * pixels (reference RefDem::getData semantics, DataTypes.cpp:247-300). */
int tops_synth_burst_dem_window(const tops_scene *s, int burst, int margin, int *row0,
                                int *col0, int *rows, int *cols);
/* Truth of the slave geometry on a coarse grid: n nodes of
 * (master line, master pixel, slave line, slave pixel) in full-image
 * (burst-stacked) coordinates, excluding the injected misregistration. */
int tops_synth_truth(const tops_scene *s, int burst, long *n, const double **nodes);
/* Seconds spent generating each part (orbits+DEM, reflectivity, master,
 * geometry, slave). */
int tops_synth_timing(const tops_scene *s, double t[5]);

#ifdef __cplusplus
}
#endif
#endif

/* tops_s1.h -- Sentinel-1 SAFE front end: annotation and precise-orbit
 * readers and master/slave burst matching, without tinyxml2.
 *
 * The readers fill the tops_swath_info that the pair plans take
 * (tops_b200.h), from the same XML elements the reference reads:
 *   tops_s1_annotation_read   S1_Initialize (Func.cpp:135-574) and the DC /
 *                             FM-rate lists of ComputeDerampPara
 *                             (Func.cpp:1868-2010)
 *   tops_s1_geogrid_read      the geolocation grid of S1_Initialize
 *                             (Func.cpp:437-491)
 *   tops_s1_orbit_read        S1_OrbitInitialize (Func.cpp:695-819)
 *   tops_s1_burst_overlap     ComputerBurstOverlap (Func.cpp:1610-1746)
 * Times are seconds of the day, as the reference's utc2seconds
 * (Func.cpp:630-636) gives them.  All functions return TOPS_OK or a
 * TOPS_E_* status (tops_b200.h); none touches the device. */
#ifndef TOPS_S1_H
#define TOPS_S1_H

#include "tops_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Annotation values the reference reads beyond tops_swath_info. */
typedef struct {
  char polarisation[8];
  char first_line_utc[40], last_line_utc[40];   /* productFirst/LastLineUtcTime */
  char dc_method[40];                           /* processingInformation/dcMethod */
  int number_of_lines, number_of_samples;
  int last_valid_pixel;                         /* largest lastValidSample */
  double azimuth_pixel_spacing, radar_frequency, heading, range_bandwidth;
  double ascending_node_time, slr_time_last_pixel;
  /* per burst: first and last line whose firstValidSample is not -1, and
   * their times (burstFirst/LastValidLineTime) */
  int first_valid_line[TOPS_MAX_BURSTS], last_valid_line[TOPS_MAX_BURSTS];
  double burst_first_valid_time[TOPS_MAX_BURSTS], burst_last_valid_time[TOPS_MAX_BURSTS];
  /* per burst: lat/lon box of the geolocation grid rows b and b + 1
   * (latlonBurst, Func.cpp:494-537) */
  double burst_lat_min[TOPS_MAX_BURSTS], burst_lat_max[TOPS_MAX_BURSTS];
  double burst_lon_min[TOPS_MAX_BURSTS], burst_lon_max[TOPS_MAX_BURSTS];
  int geo_lines, geo_points_per_line;
} tops_s1_annotation;

/* Reads one sub-swath annotation file into info (everything but the state
 * vectors, which come from the orbit file) and, if extra is not NULL, into
 * extra.  DC polynomials are the data polynomials when dcMethod is "Data
 * Analysis", else the geometry polynomials (Func.cpp:1903-1920); FM-rate
 * entries are read from c0/c1/c2 or from azimuthFmRatePolynomial.  The DC
 * and FM lists hold at most TOPS_MAX_BURSTS + 4 entries, bursts at most
 * TOPS_MAX_BURSTS (TOPS_E_INVALID beyond).  TOPS_E_INVALID: unreadable
 * file; TOPS_E_CONFIG: malformed XML or a missing element. */
int tops_s1_annotation_read(const char *xml_path, tops_swath_info *info,
                            tops_s1_annotation *extra);

/* The geolocation grid of an annotation file, row-major [lines][points]:
 * azimuth time (s of day), one-way slant-range time, latitude, longitude,
 * incidence angle.  capacity is the length of each array; *lines and
 * *points receive the grid shape (points per line: the run of equal 'line'
 * values at the start of the list, as the reference counts it).  Any array
 * may be NULL to skip it. */
int tops_s1_geogrid_read(const char *xml_path, int capacity, double *az_time, double *slr_time,
                         double *lat, double *lon, double *incidence, int *lines, int *points);

/* State vectors from a precise-orbit (EOF) file, as S1_OrbitInitialize
 * selects them: the first OSV whose UTC contains first_line_utc truncated to
 * its ten-second step, from 4 vectors before it, (last - first seconds) / 10
 * + 10 vectors.  first/last_line_utc are annotation times
 * ("YYYY-MM-DDTHH:MM:SS.ffffff").  Fills info->n_sv and sv_t/x/y/z (at most
 * 32 vectors, TOPS_E_INVALID beyond); vel, if not NULL, receives
 * [n][3] velocities.  TOPS_E_CONFIG: no matching OSV or too few after it. */
int tops_s1_orbit_read(const char *eof_path, const char *first_line_utc,
                       const char *last_line_utc, tops_swath_info *info, double *vel);

/* Geolocation grid of one sub-swath (tops_s1_geogrid_read's arrays). */
typedef struct {
  int lines, points;
  const double *az_time, *slr_time, *lat, *lon;
} tops_s1_geogrid;

/* Master/slave burst matching (ComputerBurstOverlap, Func.cpp:1610-1746):
 * the burst-centre pixel of master burst burst0 (1-based, as the config
 * file gives it) is geolocated with the master orbit (range-Doppler, from
 * the grid's position as the start) and its zero-Doppler time on the slave
 * orbit picks the slave's first burst; when it falls before the slave, the
 * slave's first burst is matched on the master instead.  The range
 * sampling rate is each info's rsr (Hz).  Outputs are 0-based burst indices.
 * TOPS_E_INVALID: burst0 < 1 or inconsistent inputs; TOPS_E_CONFIG: the
 * images do not overlap. */
int tops_s1_burst_overlap(int burst0, int burstN, const tops_swath_info *master,
                          const tops_s1_geogrid *master_grid, const tops_swath_info *slave,
                          const tops_s1_geogrid *slave_grid, int *m_burst0, int *m_burstN,
                          int *s_burst0, int *s_burstN);

#ifdef __cplusplus
}
#endif

#endif /* TOPS_S1_H */

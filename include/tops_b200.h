/*
 * tops_b200.h -- C ABI of the B200-native TOPS burst-pair processor.
 *
 * Two layers:
 *
 *  1. Reference-compatible entry points.  Same names, argument order, units
 *     and memory layouts as the a787854/InSAR-on-Sentinel-1-TOPS-data GPU
 *     wrappers, so the reference's stage drivers (Func.cpp) link against this
 *     library unchanged.  Differences: they return an int status (TOPS_OK on
 *     success) instead of calling exit(), never call cudaDeviceReset(), and
 *     run on the calling thread's current device.  Host buffers are plain
 *     pointers: CInt16 = interleaved int16 (re, im) (std::complex<short>),
 *     complex64 = interleaved float (std::complex<float> / cuComplex).
 *
 *  2. Device API (tops_*).  Device-resident, stream-ordered, no hidden
 *     allocation or synchronisation: the caller owns every buffer.  Used by
 *     the batched burst-pair pipeline and the serving loop, and by callers
 *     that keep bursts resident in HBM.
 *
 * Every function returns an int status: TOPS_OK (0) or a TOPS_E_* code.
 */
#ifndef TOPS_B200_H
#define TOPS_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */
enum {
  TOPS_OK = 0,
  TOPS_E_INVALID = 1,   /* bad argument (size, box, null pointer, window) */
  TOPS_E_CUDA = 2,      /* CUDA runtime error; see tops_last_cuda_error() */
  TOPS_E_NOMEM = 3,     /* device or pinned allocation failed */
  TOPS_E_NOT_PD = 4,    /* geocoreg normal matrix not positive definite */
  TOPS_E_TIMEOUT = 5,   /* a bounded device wait gave up */
  TOPS_E_BUDGET = 6,    /* serving admission: footprint above the HBM budget */
  TOPS_E_CONFIG = 7,    /* malformed config.txt */
  TOPS_E_NODEVICE = 8   /* no CUDA device */
};

const char *tops_status_string(int status);
/* Last CUDA error code seen by this library on the calling thread. */
int tops_last_cuda_error(void);
/* Library version string. */
const char *tops_version(void);

/* Measured FP64 fused-multiply-add throughput of the current device in
 * TFLOP/s (2 flops per FMA), timed with CUDA events on `stream` under the
 * clocks the device runs at.  No counterpart in the reference: it is the
 * denominator of the geometric coregistration's roofline, a stage bound by
 * FP64 arithmetic rather than by memory. */
int tops_fp64_peak(double *tflops, void *stream);
/* Waits for the work enqueued on `stream` (NULL: the legacy stream). */
int tops_stream_synchronize(void *stream);

/* ============================================ 1. reference-compatible ABI */

/* Replaces Geocoreg_cuda.cu:22-68 (GeoCoreg_warp_cuda).  DEM-assisted
 * geometric coregistration of one burst: fits the 6-term slave azimuth and
 * range polynomials of the normalised master (line, pixel).  inputDEM is the
 * DEM window [DemLines][DemPixels] (int heights, demnodata marks holes) whose
 * first sample is at (lat0, lon0) degrees.  AzCpm/RgCpm receive 6 doubles
 * each.  Unlike the reference the whole DEM window is copied (the reference
 * copies half, Geocoreg_cuda.cu:788). */
int GeoCoreg_warp_cuda(int m_burstIdx, int s_burstIdx, int xmin, int xmax, int ymin, int ymax,
                       double dem_DeltaLat, double dem_DeltaLon, int DemLines, int DemPixels,
                       double *AzCpm, double *RgCpm, double lat0, double lon0, int demnodata,
                       double m_azimuthTimeInterval, double s_azimuthTimeInterval,
                       double wavelength, double m_linesPerBurst, double s_linesPerBurst,
                       double m_burstFirstLineTime, double s_burstFirstLineTime,
                       int m_numOfSamples, int s_numOfSamples, double *m_orbitAzTime,
                       double *s_orbitAzTime, int orb_m_numberofpoints, int orb_m_numbercoefs,
                       int orb_s_numberofpoints, int orb_s_numbercoefs,
                       double m_slrTimeToFirstPixel, double s_slrTimeToFirstPixel,
                       double m_rangeSpacing, double s_rangeSpacing, bool m_nearRangeOnLeft,
                       bool s_nearRangeOnLeft, int *inputDEM, double *m_x_coef, double *m_y_coef,
                       double *m_z_coef, double *s_x_coef, double *s_y_coef, double *s_z_coef,
                       double m_aziInitial, double s_aziInitial);

/* Replaces DerampAndResample.cu:27-47 (DerampDemodResample).  Deramps and
 * demodulates the slave burst SlaveArray [SlaveBox rows][SlaveBox cols]
 * (CInt16), resamples it onto the master grid MasterBox with the 12-point
 * LUT sinc (KernelAz/KernelRg [2048][Npoints]) at the positions given by the
 * offset polynomials CpmAz/CpmRg (+AzimuthShift lines), reramps, and writes
 * output [MasterBox rows][MasterBox cols] complex64.  dopplerRate,
 * referenceTime and dopplerCentroid are indexed by absolute slave sample. */
int DerampDemodResample(void *SlaveArray, double *CpmAz, double *CpmRg, double AzimuthShift,
                        void *output, float *KernelAz, float *KernelRg, int sBurstIdx,
                        int slave_pixels, int slave_lines, int MasterBox[4], int SlaveBox[4],
                        int S_linesPerBurst, int S_SamplesPerBurst, double azimuthTimeInterval,
                        double *dopplerRate, double *referenceTime, double *dopplerCentroid,
                        int Npoints);

/* Replaces DerampAndResample.cu:49-69 (DerampDemodResample_ESD).  Same as
 * DerampDemodResample, and returns the DEVICE copy of the resampled burst
 * (contiguous complex64, MasterBox cols per row).  Ownership passes to the
 * caller: CoherenceEst/CoherenceEst_ESD free it, as in the reference, or
 * release it with tops_free_device().  NULL on error. */
void *DerampDemodResample_ESD(void *SlaveArray, double *CpmAz, double *CpmRg,
                              double AzimuthShift, void *output, float *KernelAz,
                              float *KernelRg, int sBurstIdx, int slave_pixels, int slave_lines,
                              int MasterBox[4], int SlaveBox[4], int linesPerBurst,
                              int SamplesPerBurst, double azimuthTimeInterval,
                              double *dopplerRate, double *referenceTime,
                              double *dopplerCentroid, int Npoints);

/* Replaces DerampAndResample.cu:71-75 (ResampleFirstBurst): uploads a host
 * complex64 burst [hh][ww] and returns the device copy (ownership as above). */
void *ResampleFirstBurst(void *SlaveArray, int ww, int hh);

/* Replaces EstESD.cu:28-44 (EstESDShifts).  Enhanced Spectral Diversity:
 * MasterFor/MasterBack (CInt16) and SlaveFor/SlaveBack (complex64) hold the
 * numOverlap forward/backward overlap bands concatenated [ArrayLines]
 * [ArrayPixels]; OverlapSizeArray gives the lines of each band.  Writes
 * ShiftArray[numOverlap] azimuth shifts in pixels. */
int EstESDShifts(void *MasterFor, void *MasterBack, void *SlaveFor, void *SlaveBack,
                 int *OverlapSizeArray, double *ShiftArray, int numOverlap, int ArrayLines,
                 int ArrayPixels, int CohWinAz, int CohWinRg, int OverlapMaxLines,
                 float CohThresHold, double spectralSeparation, double azimuthTimeInterval);

/* Replaces EstCoh.cu:919-931 (CoherenceEst) and EstCoh.cu:462-474
 * (CoherenceEst_ESD): windowed coherence of masterArray (host CInt16
 * [Dh][Dw]) against d_slaveArray (DEVICE complex64 [Dh][Dw], as returned by
 * DerampDemodResample_ESD / ResampleFirstBurst).  Box rows r-dy..r-dy+winAz-1,
 * cols c-dx..c-dx+winRg-1, zero padded; 0 where |slave| < 0.001.  Frees
 * d_slaveArray like the reference.  Both names compute the same result (the
 * reference's prefix-sum and direct-box variants are equal in exact math). */
int CoherenceEst(int Dx0, int Dy0, int Dw, int Dh, int dx, int dy, int cohWinRg, int cohWinAz,
                 void *masterArray, void *d_slaveArray, float *cohdata);
int CoherenceEst_ESD(int Dx0, int Dy0, int Dw, int Dh, int dx, int dy, int cohWinRg,
                     int cohWinAz, void *masterArray, void *d_slaveArray, float *cohdata);

/* Release a device pointer returned by DerampDemodResample_ESD /
 * ResampleFirstBurst without computing coherence. */
int tops_free_device(void *d_ptr);

/* ======================================================= 2. device API */

#define TOPS_LUT_BINS 2048
#define TOPS_NPOINTS 12

/* Interpolation kernels resident on the device.  Create from host LUTs
 * [2048][12] (e.g. the reference's ResampleTable or tops_lut()). */
typedef struct tops_lut_dev tops_lut_dev;
int tops_lut_create(const float *kaz, const float *krg, tops_lut_dev **out);
int tops_lut_destroy(tops_lut_dev *lut);

/* One burst to resample (deramp + sinc + reramp).  All pointers are device
 * pointers; pitches are in bytes. */
typedef struct {
  const void *slave;        /* CInt16 [sbox rows][sbox cols] */
  size_t slave_pitch;
  void *out;                /* complex64 [mbox rows][mbox cols] */
  size_t out_pitch;
  const double *kt, *tref, *fdc;   /* per absolute slave sample */
  int mbox[4], sbox[4];            /* {x0, x1, y0, y1} inclusive */
  double cpm_az[6], cpm_rg[6];
  double az_shift;                 /* lines added to the azimuth polynomial */
  const double *az_shift_dev;      /* if non-NULL, *az_shift_dev is used (|v| > 100 -> 0) */
  const double *cpm_dev;           /* if non-NULL, 12 device doubles replace cpm_az/cpm_rg */
  int s_first_line;                /* sBurstIdx * linesPerBurst */
  double dt;                       /* azimuth time interval [s] */
  int out_row0, out_rows;          /* master rows to produce; out_rows<0: all.
                                      `out` points at the row out_row0 */
} tops_resample_job;

/* Precision of the deramp phase inside the resample kernel.
 *   TOPS_PREC_SPLIT  FP32 phase residual and reduced phase per sample,
 *                    relative to an FP64 reference-column phase reduced
 *                    mod 2 pi once per row (double-single); the default.
 *   TOPS_PREC_FP64   every sample's deramp phase and its reduction in FP64.
 * Positions, LUT bins and the row phase are FP64 in both. */
#define TOPS_PREC_SPLIT 0
#define TOPS_PREC_FP64 1

/* Resamples njobs bursts in one launch on `stream` (cudaStream_t). */
int tops_resample(const tops_lut_dev *lut, const tops_resample_job *jobs, int njobs,
                  void *stream);
/* As tops_resample, with the precision mode (TOPS_PREC_*) chosen explicitly. */
int tops_resample_ex(const tops_lut_dev *lut, const tops_resample_job *jobs, int njobs,
                     int precision, void *stream);

/* One burst of windowed coherence (device pointers, byte pitches). */
typedef struct {
  const void *master;  size_t master_pitch;   /* CInt16 */
  const void *slave;   size_t slave_pitch;    /* complex64 */
  float *coh;          size_t coh_pitch;
  int lines, pixels;
} tops_coh_job;

int tops_coherence(const tops_coh_job *jobs, int njobs, int win_rg, int win_az, void *stream);

/* ESD over the overlaps of one or more swaths.  Each overlap gives device
 * pointers to its four bands (rows `lines`, `pixels` samples, byte pitches).
 * shifts_dev receives one double per overlap (device).  sums_dev (optional)
 * receives the complex phasor sum per overlap (2 doubles).  scratch_dev must
 * hold tops_esd_scratch_bytes(...) bytes. */
typedef struct {
  const void *mF, *mB;  size_t m_pitch;     /* CInt16 */
  const void *sF, *sB;  size_t s_pitch;     /* complex64 */
  int lines, pixels;
  double spec_sep, dt;
} tops_esd_overlap;

size_t tops_esd_scratch_bytes(const tops_esd_overlap *ovs, int n_ov);
int tops_esd(const tops_esd_overlap *ovs, int n_ov, int win_az, int win_rg, float coh_thr,
             double *shifts_dev, double *sums_dev, void *scratch_dev, size_t scratch_bytes,
             void *stream);

/* Allocation-free variant of tops_esd (no counterpart in the reference).
 * For callers that cannot allocate device memory: code running under an
 * HBM budget owned by someone else (a serving loop that admits work by
 * footprint, a framework whose pool owns the device), or latency-critical
 * loops where cudaMalloc's implicit device synchronisation is not allowed.
 * The per-CTA partial sums live in a static 256 KB array compiled into the
 * library (16384 partials: e.g. 8 overlaps of 100 x 21000 need 3008); every
 * GPU that loads the library holds that array until the process exits.
 * Larger requests return TOPS_E_INVALID with a message; use tops_esd with a
 * caller-provided scratch buffer for those.  At most 32 overlaps per call.
 * The first call on a device looks up the array's device address (once per
 * device, with that device current); make that first call before any stream
 * capture.  All calls share the array: calls whose executions overlap on
 * the GPU (different streams, or concurrent host threads) race and must be
 * serialised by the caller.  Inputs and outputs are as for tops_esd. */
int tops_esd_static(const tops_esd_overlap *ovs, int n_ov, int win_az, int win_rg, float coh_thr,
                    double *shifts_dev, double *sums_dev, void *stream);

/* Geometric coregistration of one burst on a device-resident float DEM
 * window.  Writes cpm_dev[12] (6 azimuth then 6 range coefficients) and
 * status_dev[1] (0 ok, 4 = not positive definite) on the device. */
typedef struct {
  const float *dem;  size_t dem_pitch;      /* float heights */
  int dem_lines, dem_pixels;
  double lat0, lon0, dlat, dlon, nodata;
  int xmin, xmax, ymin, ymax;
  double dt[2], first_line_time[2], slr_time[2], range_spacing[2];
  double mid_time[2], azi_init[2];
  int line_offset[2];
  double coef[2][3][8];                      /* [image][x,y,z][coef] */
  int ncoef[2];
  double *cpm_dev;
  int *status_dev;
} tops_geo_job;

size_t tops_geocoreg_scratch_bytes(const tops_geo_job *jobs, int njobs);
int tops_geocoreg(const tops_geo_job *jobs, int njobs, void *scratch_dev, size_t scratch_bytes,
                  void *stream);

/* ============================================ host-side TOPS precomputes */

/* LUT of the raised-cosine windowed sinc (reference InKernelInit,
 * Func.cpp:2105-2158): kaz/krg [2048][npoints]. */
int tops_lut(int npoints, double prf, double abw, double rsr2x, float *kaz, float *krg);

/* Orbit polynomial fit (reference Polyfit_Orbit, Func.cpp:1050-1126). */
int tops_polyfit_orbit(int npts, const double *t, const double *x, const double *y,
                       const double *z, double *cx, double *cy, double *cz, int *ncoef);

typedef struct { double aztime, t0, c0, c1, c2; } tops_poly;

typedef struct {
  int n_bursts, samples_per_burst, lines_per_burst, first_valid_pixel;
  double slr_time_first_pixel, range_pixel_spacing, azimuth_time_interval;
  double first_line_time, last_line_time, steering_rate_deg, wavelength;
  const double *burst_first_line_time, *burst_last_line_time;
  const tops_poly *dc_list; int n_dc;
  const tops_poly *fm_list; int n_fm;
  const double *orb_cx, *orb_cy, *orb_cz; int orb_ncoef; double orb_mid_time;
} tops_deramp_desc;

/* Deramp parameters (reference ComputeDerampPara, Func.cpp:1868-2099):
 * [n_bursts][samples] Doppler centroid, FM rate, reference time, kt. */
int tops_deramp_params(const tops_deramp_desc *d, double *dc, double *fmrate, double *reftime,
                       double *kt);

/* Reference EstOverlapSize (Func.cpp:2935-2960) and GetSpectralSep
 * (Func.cpp:2962-2976). */
int tops_overlap_size(int n_bursts, const double *first_time, const double *last_time, double dt,
                      int *ov, int *total, int *maximum);
double tops_spectral_sep(int n_bursts, int W, int L, double dt, const double *kt);

/* ====================================================== swath metadata */

#define TOPS_MAX_BURSTS 16

/* Annotation-level description of one sub-swath of one acquisition: what
 * the reference reads from the SAFE annotation and the precise orbit
 * (SubSwathInfo / S1PreciseOrbit, DataTypes.h:41-177).  Times in seconds,
 * slr_time one-way slant-range time of the first sample. */
typedef struct {
  int n_bursts, lines_per_burst, samples_per_burst, first_valid_pixel;
  double dt, prf, slr_time, range_spacing, wavelength, rsr, az_bandwidth, steering_rate_deg;
  double first_line_time, last_line_time;
  double burst_first_line_time[TOPS_MAX_BURSTS];
  double burst_last_line_time[TOPS_MAX_BURSTS];
  int n_dc, n_fm;
  tops_poly dc_list[TOPS_MAX_BURSTS + 4];
  tops_poly fm_list[TOPS_MAX_BURSTS + 4];
  int n_sv;
  double sv_t[32], sv_x[32], sv_y[32], sv_z[32];
} tops_swath_info;

/* =========================================================== stitching */

/* Debursting of one sub-swath (Stitch_OneSubswath / getLineIdxInMetaData,
 * Func.cpp:2766-2933): for every output line, from the first valid line of
 * burst burst0 to the last valid line of burst burstN at the azimuth
 * interval, the row of the burst stack (bursts burst0..burstN, lines_per_burst
 * rows each) it is taken from.  first_valid / last_valid: per-burst valid
 * line indices (the annotation's firstValidLine / lastValidLine).  line_map
 * NULL: only *height is returned.  TOPS_E_INVALID where the reference would
 * stop (a line no burst covers) or a line falls outside the stacked bursts. */
int tops_stitch_line_map(const tops_swath_info *m, const int *first_valid, const int *last_valid,
                         int burst0, int burstN, int *line_map, int capacity, int *height);

/* Row gather on the device: dst row i = src row line_map_dev[i] (device
 * int array), row_bytes per row (a multiple of 4: CInt16, float or complex64
 * rows), pitches in bytes.  Asynchronous on `stream`. */
int tops_stitch(const void *src, size_t src_pitch, void *dst, size_t dst_pitch,
                const int *line_map_dev, int height, size_t row_bytes, void *stream);

/* ======================================================= TIFF raster I/O */

/* Pixel types of the reference's GeoTIFF files (GDAL GDT_CInt16,
 * GDT_Float32, GDT_CFloat32: SLCs, coherence, resampled slaves; GDT_Int16:
 * the DEM it reads, DataTypes.cpp:230-290). */
enum { TOPS_TIFF_CINT16 = 1, TOPS_TIFF_FLOAT32 = 2, TOPS_TIFF_CFLOAT32 = 3, TOPS_TIFF_INT16 = 4 };

/* Writes a single-band, uncompressed, little-endian baseline TIFF
 * (strips, SampleFormat complex int / IEEE float / complex IEEE float), the
 * raster layout of the reference's TiffWrite (DataTypes.cpp:545-666) without
 * GDAL.  rows of `pitch` bytes.  Classic TIFF: the file must stay below
 * 4 GiB (TOPS_E_INVALID otherwise). */
int tops_tiff_write(const char *path, int type, int width, int height, const void *data,
                    size_t pitch);

/* Reads a single-band, uncompressed, strip-organised TIFF of one of the
 * pixel types (little- or big-endian file; 16-bit unsigned samples are read
 * as TOPS_TIFF_INT16, as GDAL's Int16 reads them); data NULL: only the type
 * and size are returned.  Rows are packed (width * pixel bytes). */
int tops_tiff_read(const char *path, int *type, int *width, int *height, void *data,
                   size_t capacity);

/* The geotransform GDAL gives a north-up GeoTIFF (the reference's RefDem::Init,
 * DataTypes.cpp:200-222, reads the DEM's through GDALGetGeoTransform):
 * gt[0] / gt[3] x / y of the upper-left corner, gt[1] pixel width, gt[5]
 * pixel height (negative), gt[2] = gt[4] = 0; from ModelPixelScale and
 * ModelTiepoint, the origin moved half a pixel for PixelIsPoint rasters.
 * TOPS_E_INVALID without those tags. */
int tops_tiff_georef(const char *path, double gt[6]);

/* tops_tiff_write with that georeferencing (north-up, geographic WGS 84,
 * pixel is area), e.g. for a DEM; gt as tops_tiff_georef returns it. */
int tops_tiff_write_georef(const char *path, int type, int width, int height, const void *data,
                           size_t pitch, const double gt[6]);

/* ============================================================ config */

/* config.txt (reference ReadInput, Func.cpp:7-130): key=value lines.
 * Reference keys are kept; synthetic-scene and serving keys are added. */
typedef struct {
  char process_dir[512], masterpath[512], slavepath[512], polarisation[64];
  char preciseOrbitMaster[512], preciseOrbitSlave[512], SpecificDemPath[512];
  int firstsubswath, lastsubswath, multi_az, multi_rg, burst0, burstN;
  /* synthetic scene */
  long seed;
  int n_bursts, lines_per_burst, samples_per_burst, overlap_lines;
  int dem_lines, dem_pixels;
  double sigma_dn, az_shift_true;
  /* processing */
  int coh_win_rg, coh_win_az, npoints;
  double esd_coh_threshold;
  /* serving */
  double hbm_budget_gb, arrival_rate;
  int n_jobs;
  /* 1: tops_run_config also writes the debursted coherence (the reference's
   * disabled stitching step, Main.cpp:123-131) */
  int stitch;
} tops_config;

/* Parse a config file.  Unknown keys are ignored (as in the reference);
 * a line without '=' or a bad integer gives TOPS_E_CONFIG with the line
 * number in *err_line. */
int tops_config_read(const char *path, tops_config *cfg, int *err_line);
int tops_config_defaults(tops_config *cfg);

#ifdef __cplusplus
}
#endif
#endif

// geocoreg_full_dem.cu -- builds the reference's Geocoreg_cuda.cu (included
// unmodified from the reference tree) into oracle/_ref/libref_geocoreg.so.
// Test infrastructure: it produces reference outputs for the golden fixtures.
//
// One host-side fix, applied from outside the reference source: the reference
// copies the int DEM with N * sizeof(short) bytes (Geocoreg_cuda.cu:788), so
// the second half of its device DEM is never written and the fit would depend
// on whatever that memory holds.  While GeoCoreg_warp_cuda_full_dem runs, the
// one host-to-device copy whose source is the caller's DEM is widened to the
// whole array.  Nothing else in the reference's code path changes.
#include <cuda_runtime.h>

#include <cstddef>

namespace {
const void *g_dem_host = nullptr;
size_t g_dem_bytes = 0;

cudaError_t full_dem_memcpy(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
  if (kind == cudaMemcpyHostToDevice && src != nullptr && src == g_dem_host && bytes < g_dem_bytes)
    bytes = g_dem_bytes;
  return cudaMemcpy(dst, src, bytes, kind);
}
}  // namespace

#define cudaMemcpy full_dem_memcpy
#include "Geocoreg_cuda.cu"
#undef cudaMemcpy

// Same argument list as GeoCoreg_warp_cuda (Geocoreg_cuda.cu:22-68).
extern "C" void GeoCoreg_warp_cuda_full_dem(
    int m_burstIdx, int s_burstIdx, int xmin, int xmax, int ymin, int ymax, double dem_DeltaLat,
    double dem_DeltaLon, int DemLines, int DemPixels, double *AzCpm, double *RgCpm, double lat0,
    double lon0, int demnodata, double m_azimuthTimeInterval, double s_azimuthTimeInterval,
    double wavelength, double m_linesPerBurst, double s_linesPerBurst,
    double m_burstFirstLineTime, double s_burstFirstLineTime, int m_numOfSamples,
    int s_numOfSamples, double *m_orbitAzTime, double *s_orbitAzTime, int orb_m_numberofpoints,
    int orb_m_numbercoefs, int orb_s_numberofpoints, int orb_s_numbercoefs,
    double m_slrTimeToFirstPixel, double s_slrTimeToFirstPixel, double m_rangeSpacing,
    double s_rangeSpacing, bool m_nearRangeOnLeft, bool s_nearRangeOnLeft, int *inputDEM,
    double *m_x_coef, double *m_y_coef, double *m_z_coef, double *s_x_coef, double *s_y_coef,
    double *s_z_coef, double m_aziInitial, double s_aziInitial) {
  g_dem_host = inputDEM;
  g_dem_bytes = (size_t)DemLines * (size_t)DemPixels * sizeof(int);
  GeoCoreg_warp_cuda(m_burstIdx, s_burstIdx, xmin, xmax, ymin, ymax, dem_DeltaLat, dem_DeltaLon,
                     DemLines, DemPixels, AzCpm, RgCpm, lat0, lon0, demnodata,
                     m_azimuthTimeInterval, s_azimuthTimeInterval, wavelength, m_linesPerBurst,
                     s_linesPerBurst, m_burstFirstLineTime, s_burstFirstLineTime, m_numOfSamples,
                     s_numOfSamples, m_orbitAzTime, s_orbitAzTime, orb_m_numberofpoints,
                     orb_m_numbercoefs, orb_s_numberofpoints, orb_s_numbercoefs,
                     m_slrTimeToFirstPixel, s_slrTimeToFirstPixel, m_rangeSpacing, s_rangeSpacing,
                     m_nearRangeOnLeft, s_nearRangeOnLeft, inputDEM, m_x_coef, m_y_coef, m_z_coef,
                     s_x_coef, s_y_coef, s_z_coef, m_aziInitial, s_aziInitial);
  g_dem_host = nullptr;
  g_dem_bytes = 0;
}

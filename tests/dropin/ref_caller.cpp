// ref_caller.cpp -- a caller of the burst-pair stage entry points compiled
// against the declarations the reference's host code uses for them
// (Func.cpp:2163-2210, 2304-2324, 2422-2494): the same names and parameter
// lists, `void` returns where the reference declares void, the device
// pointer typed cuComplex*, and std::complex<short> / std::complex<float>
// host arrays.  The test links it against libtops_b200.so with
// --no-undefined, so every declaration must resolve to the library, and on
// a GPU runs it through the reference driver's call sequence.
//
// The library defines these functions with an int status and void*
// pointers; a caller that declares them void ignores the status register,
// and the pointer types have one representation, so the reference's
// objects link and run unchanged.  Parameter names are this file's own.
#include <cuComplex.h>

#include <complex>

using std::complex;

extern "C" {
void GeoCoreg_warp_cuda(int mBurst, int sBurst, int xmin, int xmax, int ymin, int ymax,
                        double dLat, double dLon, int demLines, int demPixels, double *azCpm,
                        double *rgCpm, double lat0, double lon0, int noData, double mDt,
                        double sDt, double lambda, double mLinesPerBurst, double sLinesPerBurst,
                        double mFirstLineTime, double sFirstLineTime, int mSamples, int sSamples,
                        double *mOrbitT, double *sOrbitT, int mOrbitN, int mOrbitCoefs,
                        int sOrbitN, int sOrbitCoefs, double mSlrTime, double sSlrTime,
                        double mRangeSpacing, double sRangeSpacing, bool mNearLeft, bool sNearLeft,
                        int *dem, double *mCx, double *mCy, double *mCz, double *sCx,
                        double *sCy, double *sCz, double mAziInit, double sAziInit);
void DerampDemodResample(complex<short> *slave, double *cpmAz, double *cpmRg, double azShift,
                         complex<float> *out, float *kAz, float *kRg, int sBurst, int sPixels,
                         int sLines, int masterBox[4], int slaveBox[4], int linesPerBurst,
                         int samplesPerBurst, double dt, double *kt, double *tref, double *fdc,
                         int nPoints);
cuComplex *DerampDemodResample_ESD(complex<short> *slave, double *cpmAz, double *cpmRg,
                                   double azShift, complex<float> *out, float *kAz, float *kRg,
                                   int sBurst, int sPixels, int sLines, int masterBox[4],
                                   int slaveBox[4], int linesPerBurst, int samplesPerBurst,
                                   double dt, double *kt, double *tref, double *fdc, int nPoints);
cuComplex *ResampleFirstBurst(complex<float> *reslave, int width, int height);
void EstESDShifts(complex<short> *mFor, complex<short> *mBack, complex<float> *sFor,
                  complex<float> *sBack, int *ovSize, double *shifts, int nOv, int lines,
                  int pixels, int winAz, int winRg, int ovMax, float cohThr, double specSep,
                  double dt);
void CoherenceEst_ESD(int x0, int y0, int w, int h, int dx, int dy, int winRg, int winAz,
                      complex<short> *master, cuComplex *dSlave, float *coh);
void CoherenceEst(int x0, int y0, int w, int h, int dx, int dy, int winRg, int winAz,
                  complex<short> *master, cuComplex *dSlave, float *coh);
}

// One burst of the reference's DerampAndResample + ESDAndCoh drivers: its
// ReSlave, its ESD-corrected resample kept on the device, and the coherence
// of that device copy (which CoherenceEst frees).  A first burst (shift
// ignored) takes its ReSlave through ResampleFirstBurst and
// CoherenceEst_ESD, as the reference's first-burst branch does.  Returns 1
// when the device copy could not be made (the only failure a caller of
// these void declarations can see).
extern "C" int ref_caller_burst(complex<short> *slave, complex<short> *master, double *cpmAz,
                                double *cpmRg, double shift, float *kAz, float *kRg, int sBurst,
                                int pixels, int lines, int *masterBox, int *slaveBox,
                                double sDt, double mDt, double *kt, double *tref, double *fdc,
                                int winRg, int winAz, int first, complex<float> *reslave,
                                complex<float> *reslaveEsd, float *coh) {
  DerampDemodResample(slave, cpmAz, cpmRg, 0.0, reslave, kAz, kRg, sBurst, pixels, lines,
                      masterBox, slaveBox, lines, pixels, sDt, kt, tref, fdc, 12);
  cuComplex *d;
  if (first) {
    for (long i = 0; i < (long)pixels * lines; i++) reslaveEsd[i] = reslave[i];
    d = ResampleFirstBurst(reslave, pixels, lines);
  } else {
    d = DerampDemodResample_ESD(slave, cpmAz, cpmRg, shift, reslaveEsd, kAz, kRg, sBurst, pixels,
                                lines, masterBox, slaveBox, lines, pixels, mDt, kt, tref, fdc, 12);
  }
  if (!d) return 1;
  if (first)
    CoherenceEst_ESD(0, 0, pixels, lines, (winRg - 1) / 2, (winAz - 1) / 2, winRg, winAz, master,
                     d, coh);
  else
    CoherenceEst(0, 0, pixels, lines, (winRg - 1) / 2, (winAz - 1) / 2, winRg, winAz, master, d,
                 coh);
  return 0;
}

// The reference driver's ESD call over concatenated overlap bands.
extern "C" void ref_caller_esd(complex<short> *mFor, complex<short> *mBack, complex<float> *sFor,
                               complex<float> *sBack, int *ovSize, double *shifts, int nOv,
                               int lines, int pixels, int winAz, int winRg, int ovMax,
                               float thr, double specSep, double dt) {
  EstESDShifts(mFor, mBack, sFor, sBack, ovSize, shifts, nOv, lines, pixels, winAz, winRg, ovMax,
               thr, specSep, dt);
}

// The reference driver's geometric coregistration call (int DEM window).
extern "C" void ref_caller_geocoreg(int mBurst, int sBurst, int xmin, int xmax, int ymin,
                                    int ymax, double dLat, double dLon, int demLines,
                                    int demPixels, double *azCpm, double *rgCpm, double lat0,
                                    double lon0, double mDt, double sDt, double linesPerBurst,
                                    double mFirst, double sFirst, int samples, double *mOrbitT,
                                    double *sOrbitT, int mOrbitN, int sOrbitN, int nCoef,
                                    double mSlr,
                                    double sSlr, double mRs, double sRs, int *dem, double *mCx,
                                    double *mCy, double *mCz, double *sCx, double *sCy,
                                    double *sCz, double mAzi, double sAzi) {
  GeoCoreg_warp_cuda(mBurst, sBurst, xmin, xmax, ymin, ymax, dLat, dLon, demLines, demPixels,
                     azCpm, rgCpm, lat0, lon0, -32768, mDt, sDt, 0.05547, linesPerBurst,
                     linesPerBurst, mFirst, sFirst, samples, samples, mOrbitT, sOrbitT, mOrbitN,
                     nCoef, sOrbitN, nCoef, mSlr, sSlr, mRs, sRs, false, false, dem, mCx, mCy,
                     mCz, sCx, sCy, sCz, mAzi, sAzi);
}

// driver.cpp -- the config.txt-driven run of the reference's main program
// (Main.cpp:11-150) on this library.
//
// The reference reads config.txt (ReadInput, Func.cpp:7-130), opens the SAFE
// products, orbits and DEM named there, and for every sub-swath from
// firstsubswath to lastsubswath runs geometric coregistration, deramp and
// resampling, ESD and coherence over the bursts burst0..burstN (1-based),
// writing ReSlave-N.tif, ReSlaveESD-N.tif and Coh-N.tif into process_dir
// (and, in its disabled stitching step, CohStitch-N.tif).  Product readers
// are outside this library, so the inputs of each sub-swath come from the
// seeded synthetic generator, configured by the synthetic keys of the same
// file (seed, n_bursts, lines_per_burst, ...; sub-swath N uses seed +
// 1000 (N - 1)).  The processing is the device-resident burst-pair plan; the
// outputs are written as TIFF rasters of the reference's pixel types.
#include <cuda_runtime.h>
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <chrono>
#include <string>
#include <vector>

#include "tops_pipeline.h"
#include "tops_synth.h"

namespace {

// The description of bursts [b0, b0 + k) of a sub-swath as a k-burst
// sub-swath: burst times, the per-burst FM-rate list and, when the
// annotation holds one DC estimate per burst and more, the DC list.
tops_swath_info sub_swath(const tops_swath_info &in, int b0, int k) {
  tops_swath_info out = in;
  out.n_bursts = k;
  for (int i = 0; i < k; i++) {
    out.burst_first_line_time[i] = in.burst_first_line_time[b0 + i];
    out.burst_last_line_time[i] = in.burst_last_line_time[b0 + i];
  }
  for (int i = 0; i < in.n_fm - b0; i++) out.fm_list[i] = in.fm_list[b0 + i];
  out.n_fm = in.n_fm - b0;
  if (in.n_dc > in.n_bursts) {
    for (int i = 0; i < in.n_dc - b0; i++) out.dc_list[i] = in.dc_list[b0 + i];
    out.n_dc = in.n_dc - b0;
  }
  return out;
}

struct Scene {
  tops_scene *s = nullptr;
  ~Scene() {
    if (s) tops_synth_destroy(s);
  }
};

struct Plan {
  tops_pair *p = nullptr;
  ~Plan() {
    if (p) tops_pair_destroy(p);
  }
};

int make_dir(const std::string &d) {
  if (mkdir(d.c_str(), 0755) == 0 || errno == EEXIST) return TOPS_OK;
  return TOPS_E_INVALID;
}

#define D_TRY(expr)                     \
  do {                                  \
    int _s = (expr);                    \
    if (_s != TOPS_OK) return _s;       \
  } while (0)

int run_subswath(const tops_config &c, int nsub, tops_run_stats *st) {
  tops_synth_cfg sc;
  D_TRY(tops_synth_defaults(&sc));
  sc.seed = c.seed + 1000l * (nsub - 1);
  sc.n_bursts = c.n_bursts;
  sc.lines_per_burst = c.lines_per_burst;
  sc.samples_per_burst = c.samples_per_burst;
  sc.overlap_lines = c.overlap_lines;
  sc.dem_lines = c.dem_lines;
  sc.dem_pixels = c.dem_pixels;
  sc.sigma_dn = c.sigma_dn;
  sc.az_shift_true = c.az_shift_true;
  const int b0 = c.burst0 - 1, k = c.burstN - c.burst0 + 1;
  if (b0 < 0 || k < 1 || b0 + k > c.n_bursts) return TOPS_E_INVALID;
  Scene scene;
  D_TRY(tops_synth_create(&sc, &scene.s));
  tops_swath_info mi, si;
  D_TRY(tops_synth_swath(scene.s, 0, &mi));
  D_TRY(tops_synth_swath(scene.s, 1, &si));
  const tops_swath_info m = sub_swath(mi, b0, k), s = sub_swath(si, b0, k);
  const int L = m.lines_per_burst, W = m.samples_per_burst;
  tops_dem_info di;
  const float *dem = tops_synth_dem(scene.s, &di);
  std::vector<tops_dem_window> win(k);
  for (int i = 0; i < k; i++)
    D_TRY(tops_synth_burst_dem_window(scene.s, b0 + i, 24, &win[i].row0, &win[i].col0,
                                      &win[i].rows, &win[i].cols));
  const size_t burst_elems = (size_t)L * W * 2;   // int16 per burst
  const int16_t *ms = tops_synth_slc(scene.s, 0) + (size_t)b0 * burst_elems;
  const int16_t *ss = tops_synth_slc(scene.s, 1) + (size_t)b0 * burst_elems;

  auto t0 = std::chrono::steady_clock::now();
  tops_pair_opts o;
  D_TRY(tops_pair_opts_default(&o));
  o.win_rg = c.coh_win_rg;
  o.win_az = c.coh_win_az;
  o.esd_threshold = (float)c.esd_coh_threshold;
  o.reslave_full = 1;
  Plan plan;
  D_TRY(tops_pair_create(&m, &s, &o, di.lines, di.pixels, &plan.p));
  D_TRY(tops_pair_set_dem(plan.p, dem, di.lat0, di.lon0, di.dlat, di.dlon, win.data(), nullptr));
  D_TRY(tops_pair_upload(plan.p, ms, ss, nullptr));
  D_TRY(tops_pair_run(plan.p, nullptr));
  const size_t n = (size_t)k * L * W;
  std::vector<float> reslave(2 * n), reslave_esd(2 * n), coh(n);
  std::vector<double> cpm(12 * k), shifts(k > 1 ? k - 1 : 1);
  D_TRY(tops_pair_download(plan.p, reslave.data(), reslave_esd.data(), coh.data(), cpm.data(),
                           shifts.data(), nullptr));
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) return TOPS_E_CUDA;

  // the reference's file names: <process_dir>/ReSlave-N.tif, ... (Main.cpp:98-101)
  const std::string dir = c.process_dir, tag = "-" + std::to_string(nsub) + ".tif";
  D_TRY(tops_tiff_write((dir + "/ReSlave" + tag).c_str(), TOPS_TIFF_CFLOAT32, W, k * L,
                        reslave.data(), (size_t)W * 8));
  D_TRY(tops_tiff_write((dir + "/ReSlaveESD" + tag).c_str(), TOPS_TIFF_CFLOAT32, W, k * L,
                        reslave_esd.data(), (size_t)W * 8));
  D_TRY(tops_tiff_write((dir + "/Coh" + tag).c_str(), TOPS_TIFF_FLOAT32, W, k * L, coh.data(),
                        (size_t)W * 4));
  if (c.stitch) {
    // every line of the synthetic bursts is valid
    std::vector<int> fv(k, 0), lv(k, L - 1);
    int h = 0;
    D_TRY(tops_stitch_line_map(&m, fv.data(), lv.data(), 0, k - 1, nullptr, 0, &h));
    std::vector<int> map(h);
    D_TRY(tops_stitch_line_map(&m, fv.data(), lv.data(), 0, k - 1, map.data(), h, &h));
    tops_pair_buffers b;
    D_TRY(tops_pair_buffers_get(plan.p, &b));
    int *d_map = nullptr;
    float *d_out = nullptr;
    int r = TOPS_OK;
    if (cudaMalloc(&d_map, sizeof(int) * h) != cudaSuccess ||
        cudaMalloc(&d_out, sizeof(float) * (size_t)h * W) != cudaSuccess)
      r = TOPS_E_NOMEM;
    std::vector<float> out((size_t)h * W);
    if (r == TOPS_OK && cudaMemcpy(d_map, map.data(), sizeof(int) * h,
                                   cudaMemcpyHostToDevice) != cudaSuccess)
      r = TOPS_E_CUDA;
    if (r == TOPS_OK)
      r = tops_stitch(b.coh, b.coh_pitch, d_out, (size_t)W * 4, d_map, h, (size_t)W * 4, nullptr);
    if (r == TOPS_OK && cudaMemcpy(out.data(), d_out, sizeof(float) * out.size(),
                                   cudaMemcpyDeviceToHost) != cudaSuccess)
      r = TOPS_E_CUDA;
    cudaFree(d_map);
    cudaFree(d_out);
    D_TRY(r);
    D_TRY(tops_tiff_write((dir + "/CohStitch" + tag).c_str(), TOPS_TIFF_FLOAT32, W, h,
                          out.data(), (size_t)W * 4));
  }
  st->seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  st->subswaths++;
  st->burst_pairs += k;
  for (int i = 0; i + 1 < k && i < TOPS_MAX_BURSTS; i++) st->shifts[i] = shifts[i];
  return TOPS_OK;
}

}  // namespace

extern "C" int tops_run_config(const char *config_path, tops_run_stats *stats) {
  if (!config_path || !stats) return TOPS_E_INVALID;
  memset(stats, 0, sizeof(*stats));
  tops_config c;
  D_TRY(tops_config_defaults(&c));
  int line = 0;
  D_TRY(tops_config_read(config_path, &c, &line));
  if (c.npoints != 12 || c.firstsubswath < 1 || c.lastsubswath < c.firstsubswath ||
      c.n_bursts < 1 || c.n_bursts > TOPS_MAX_BURSTS)
    return TOPS_E_CONFIG;
  D_TRY(make_dir(c.process_dir));   // CheckDir (Main.cpp:26)
  for (int nsub = c.firstsubswath; nsub <= c.lastsubswath; nsub++)
    D_TRY(run_subswath(c, nsub, stats));
  return TOPS_OK;
}

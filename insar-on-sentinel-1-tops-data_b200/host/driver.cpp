// driver.cpp -- the config.txt-driven run of the reference's main program
// (Main.cpp:11-150) on this library.
//
// The reference reads config.txt (ReadInput, Func.cpp:7-130), opens the SAFE
// products, orbits and DEM named there, and for every sub-swath from
// firstsubswath to lastsubswath runs geometric coregistration, deramp and
// resampling, ESD and coherence over the bursts burst0..burstN (1-based),
// writing ReSlave-N.tif, ReSlaveESD-N.tif and Coh-N.tif into process_dir
// (and, in its disabled stitching step, CohStitch-N.tif).
//
// With masterpath set (and not "(synthetic)"), the inputs are the products
// the reference reads: the SAFE directories' annotation files and
// measurement rasters of the configured polarisation, the precise-orbit
// files and the GeoTIFF DEM (tops_s1.h readers, tops_tiff_read /
// tops_tiff_georef), with the master's bursts burst0..burstN matched on the
// slave (ComputerBurstOverlap).  Otherwise each sub-swath comes from the
// seeded synthetic generator,
// configured by the synthetic keys of the same file (seed, n_bursts,
// lines_per_burst, ...; sub-swath N uses seed + 1000 (N - 1)).  The
// processing is the device-resident burst-pair plan; the outputs are
// written as TIFF rasters of the reference's pixel types.
#include <cuda_runtime.h>
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <chrono>
#include <future>
#include <memory>
#include <string>
#include <vector>

#include <dirent.h>
#include <math.h>

#include <algorithm>

#include "tops_pipeline.h"
#include "tops_s1.h"
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

// The inputs of one sub-swath pair for the plan: k bursts each, the DEM with
// its geotransform and one window per burst, the burst-stacked SLC rows and
// the valid lines of each master burst (for debursting).
struct PairInputs {
  tops_swath_info m, s;
  int k = 0;
  const float *dem = nullptr;
  int dem_lines = 0, dem_pixels = 0;
  double lat0 = 0, lon0 = 0, dlat = 0, dlon = 0;
  std::vector<tops_dem_window> win;
  const int16_t *ms = nullptr, *ss = nullptr;
  std::vector<int> first_valid, last_valid;
};

struct Product;

// One sub-swath's inputs and the storage they point into (a generated scene,
// or two products and the DEM).  Loaded on a host thread while the GPU works
// on the previous sub-swath.
struct Loaded {
  int status = TOPS_OK;
  double seconds = 0;   // wall time of the load
  PairInputs in;
  Scene scene;
  std::unique_ptr<Product> M, S;
  std::vector<float> dem;
};

int load_synthetic(const tops_config &c, int nsub, Loaded &out) {
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
  D_TRY(tops_synth_create(&sc, &out.scene.s));
  tops_swath_info mi, si;
  D_TRY(tops_synth_swath(out.scene.s, 0, &mi));
  D_TRY(tops_synth_swath(out.scene.s, 1, &si));
  PairInputs &in = out.in;
  in.m = sub_swath(mi, b0, k);
  in.s = sub_swath(si, b0, k);
  in.k = k;
  const int L = in.m.lines_per_burst, W = in.m.samples_per_burst;
  tops_dem_info di;
  in.dem = tops_synth_dem(out.scene.s, &di);
  in.dem_lines = di.lines;
  in.dem_pixels = di.pixels;
  in.lat0 = di.lat0;
  in.lon0 = di.lon0;
  in.dlat = di.dlat;
  in.dlon = di.dlon;
  in.win.resize(k);
  for (int i = 0; i < k; i++)
    D_TRY(tops_synth_burst_dem_window(out.scene.s, b0 + i, 24, &in.win[i].row0, &in.win[i].col0,
                                      &in.win[i].rows, &in.win[i].cols));
  const size_t burst_elems = (size_t)L * W * 2;   // int16 per burst
  in.ms = tops_synth_slc(out.scene.s, 0) + (size_t)b0 * burst_elems;
  in.ss = tops_synth_slc(out.scene.s, 1) + (size_t)b0 * burst_elems;
  // every line of the synthetic bursts is valid
  in.first_valid.assign(k, 0);
  in.last_valid.assign(k, L - 1);
  return TOPS_OK;
}

// ------------------------------------------------------------ products
// Names in dir that contain `needle` and end in one of the extensions,
// sorted (the reference lists a SAFE directory's files the same way,
// GetFiles, Func.cpp:579-628).
std::vector<std::string> list_files(const std::string &dir, const std::string &needle,
                                    std::initializer_list<const char *> exts) {
  std::vector<std::string> out;
  DIR *d = opendir(dir.c_str());
  if (!d) return out;
  while (struct dirent *e = readdir(d)) {
    const std::string n = e->d_name;
    if (n.find(needle) == std::string::npos) continue;
    for (const char *x : exts) {
      const size_t lx = strlen(x);
      if (n.size() > lx && n.compare(n.size() - lx, lx, x) == 0) {
        out.push_back(n);
        break;
      }
    }
  }
  closedir(d);
  std::sort(out.begin(), out.end());
  return out;
}

// One sub-swath of one product: annotation, geolocation grid, state
// vectors and the measurement raster.
struct Product {
  tops_swath_info info;
  tops_s1_annotation ann;
  std::vector<double> az, rg, lat, lon;
  int geo_lines = 0, geo_points = 0;
  std::vector<int16_t> slc;   // [lines][samples][2]
  int slc_lines = 0, slc_samples = 0;
};

int load_product(const std::string &safe, int nsub, const std::string &pol,
                 const std::string &orbit, Product &P) {
  const std::string adir = safe + "/annotation", mdir = safe + "/measurement";
  const std::string flag = "-slc-" + pol;
  const std::vector<std::string> xmls = list_files(adir, flag, {".xml"});
  const std::string iw = "-iw" + std::to_string(nsub) + "-";
  std::string xml;
  for (const std::string &n : xmls)
    if (n.find(iw) != std::string::npos) xml = n;
  if (xml.empty()) return TOPS_E_CONFIG;
  memset(&P.info, 0, sizeof P.info);
  D_TRY(tops_s1_annotation_read((adir + "/" + xml).c_str(), &P.info, &P.ann));
  // the state vectors around the product's first sub-swath's lines, as the
  // reference reads them once per product (Main.cpp:33-36)
  tops_s1_annotation first;
  tops_swath_info tmp;
  memset(&tmp, 0, sizeof tmp);
  D_TRY(tops_s1_annotation_read((adir + "/" + xmls[0]).c_str(), &tmp, &first));
  D_TRY(tops_s1_orbit_read(orbit.c_str(), first.first_line_utc, first.last_line_utc, &P.info,
                           nullptr));
  int gl = 0, gp = 0;
  D_TRY(tops_s1_geogrid_read((adir + "/" + xml).c_str(), 0, nullptr, nullptr, nullptr, nullptr,
                             nullptr, &gl, &gp));
  const size_t ng = (size_t)gl * gp;
  P.az.resize(ng);
  P.rg.resize(ng);
  P.lat.resize(ng);
  P.lon.resize(ng);
  D_TRY(tops_s1_geogrid_read((adir + "/" + xml).c_str(), (int)ng, P.az.data(), P.rg.data(),
                             P.lat.data(), P.lon.data(), nullptr, &gl, &gp));
  P.geo_lines = gl;
  P.geo_points = gp;
  // the measurement raster of the same name
  const std::string stem = xml.substr(0, xml.size() - 4);
  std::string tif;
  for (const std::string &n : list_files(mdir, stem, {".tiff", ".tif"})) tif = n;
  if (tif.empty()) return TOPS_E_CONFIG;
  const std::string tpath = mdir + "/" + tif;
  int type = 0, w = 0, h = 0;
  D_TRY(tops_tiff_read(tpath.c_str(), &type, &w, &h, nullptr, 0));
  if (type != TOPS_TIFF_CINT16 || w != P.info.samples_per_burst ||
      h < P.info.n_bursts * P.info.lines_per_burst)
    return TOPS_E_CONFIG;
  P.slc.resize((size_t)w * h * 2);
  D_TRY(tops_tiff_read(tpath.c_str(), &type, &w, &h, P.slc.data(), P.slc.size() * 2));
  P.slc_lines = h;
  P.slc_samples = w;
  return TOPS_OK;
}

// The DEM window of one burst: its lat/lon box extended by 24 DEM pixels,
// as the reference's GeometricCoreg asks RefDem::getData for it
// (Func.cpp:2240-2255, DataTypes.cpp:236-262).
tops_dem_window dem_window(const tops_s1_annotation &a, int b, double lat_max, double lon_min,
                           double dlat, double dlon) {
  const double la0 = a.burst_lat_min[b] - 24 * dlat, la1 = a.burst_lat_max[b] + 24 * dlat;
  const double lo0 = a.burst_lon_min[b] - 24 * dlon, lo1 = a.burst_lon_max[b] + 24 * dlon;
  const double ul0 = floor((lat_max - la1) / dlat), ul1 = floor((lo0 - lon_min) / dlon);
  const double lr0 = ceil((lat_max - la0) / dlat), lr1 = ceil((lo1 - lon_min) / dlon);
  tops_dem_window w;
  w.row0 = (int)ul0;
  w.col0 = (int)ul1;
  w.rows = (int)(lr0 - ul0 + 1);
  w.cols = (int)(lr1 - ul1 + 1);
  return w;
}

int load_products(const tops_config &c, int nsub, Loaded &out) {
  out.M.reset(new Product());
  out.S.reset(new Product());
  Product &M = *out.M, &S = *out.S;
  D_TRY(load_product(c.masterpath, nsub, c.polarisation, c.preciseOrbitMaster, M));
  D_TRY(load_product(c.slavepath, nsub, c.polarisation, c.preciseOrbitSlave, S));
  const tops_s1_geogrid mg = {M.geo_lines, M.geo_points, M.az.data(), M.rg.data(), M.lat.data(),
                              M.lon.data()};
  const tops_s1_geogrid sg = {S.geo_lines, S.geo_points, S.az.data(), S.rg.data(), S.lat.data(),
                              S.lon.data()};
  int mb0 = 0, mbN = 0, sb0 = 0, sbN = 0;
  D_TRY(tops_s1_burst_overlap(c.burst0, c.burstN, &M.info, &mg, &S.info, &sg, &mb0, &mbN, &sb0,
                              &sbN));
  const int k = mbN - mb0 + 1;
  if (k < 1 || mbN >= M.info.n_bursts || sbN >= S.info.n_bursts || sbN - sb0 + 1 != k ||
      M.info.lines_per_burst != S.info.lines_per_burst ||
      M.info.samples_per_burst != S.info.samples_per_burst)
    return TOPS_E_CONFIG;
  // the DEM (int16 or float32 heights) and its geotransform
  int type = 0, w = 0, h = 0;
  D_TRY(tops_tiff_read(c.SpecificDemPath, &type, &w, &h, nullptr, 0));
  if (type != TOPS_TIFF_INT16 && type != TOPS_TIFF_FLOAT32) return TOPS_E_CONFIG;
  double gt[6];
  D_TRY(tops_tiff_georef(c.SpecificDemPath, gt));
  std::vector<float> &dem = out.dem;
  dem.resize((size_t)w * h);
  if (type == TOPS_TIFF_INT16) {
    std::vector<int16_t> raw((size_t)w * h);
    D_TRY(tops_tiff_read(c.SpecificDemPath, &type, &w, &h, raw.data(), raw.size() * 2));
    for (size_t i = 0; i < raw.size(); i++) dem[i] = raw[i];
  } else {
    D_TRY(tops_tiff_read(c.SpecificDemPath, &type, &w, &h, dem.data(), dem.size() * 4));
  }
  // RefDem::Init (DataTypes.cpp:200-222): upper-left corner and spacings
  const double lat_max = gt[3], lon_min = gt[0], dlat = fabs(gt[5]), dlon = fabs(gt[1]);
  PairInputs &in = out.in;
  in.m = sub_swath(M.info, mb0, k);
  in.s = sub_swath(S.info, sb0, k);
  in.k = k;
  in.dem = dem.data();
  in.dem_lines = h;
  in.dem_pixels = w;
  in.lat0 = lat_max;
  in.lon0 = lon_min;
  in.dlat = dlat;
  in.dlon = dlon;
  const int L = M.info.lines_per_burst, W = M.info.samples_per_burst;
  for (int i = 0; i < k; i++) {
    in.win.push_back(dem_window(M.ann, mb0 + i, lat_max, lon_min, dlat, dlon));
    in.first_valid.push_back(M.ann.first_valid_line[mb0 + i]);
    in.last_valid.push_back(M.ann.last_valid_line[mb0 + i]);
  }
  in.ms = M.slc.data() + (size_t)mb0 * L * W * 2;
  in.ss = S.slc.data() + (size_t)sb0 * L * W * 2;
  return TOPS_OK;
}

std::unique_ptr<Loaded> load_subswath_untimed(const tops_config &c, int nsub, bool products);

std::unique_ptr<Loaded> load_subswath(const tops_config &c, int nsub, bool products) {
  const auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<Loaded> L = load_subswath_untimed(c, nsub, products);
  L->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return L;
}

std::unique_ptr<Loaded> load_subswath_untimed(const tops_config &c, int nsub, bool products) {
  std::unique_ptr<Loaded> L(new Loaded());
  L->status = products ? load_products(c, nsub, *L) : load_synthetic(c, nsub, *L);
  return L;
}

// Grow-only page-locked host buffer (pageable if the host cannot pin it):
// the plan's pipelined host-to-host call overlaps its per-burst copies with
// the kernels only on page-locked memory.
struct HostBuf {
  void *p = nullptr;
  size_t cap = 0;
  bool pinned = false;
  HostBuf() = default;
  HostBuf(const HostBuf &) = delete;
  HostBuf &operator=(const HostBuf &) = delete;
  ~HostBuf() { release(); }
  void release() {
    if (p) {
      if (pinned)
        cudaFreeHost(p);
      else
        free(p);
    }
    p = nullptr;
    cap = 0;
  }
  void *get(size_t n) {
    if (n > cap) {
      release();
      if (cudaHostAlloc(&p, n, cudaHostAllocDefault) == cudaSuccess) {
        pinned = true;
      } else {
        (void)cudaGetLastError();
        p = malloc(n);
        pinned = false;
      }
      cap = p ? n : 0;
    }
    return p;
  }
};

// One sub-swath's results, written by the writer thread.
struct Outputs {
  HostBuf reslave, reslave_esd, coh, stitched;
  double write_seconds = 0;   // wall time of write_outputs
  int k = 0, W = 0, L = 0, stitch_lines = 0, nsub = 0;
  std::vector<double> shifts;
};

void copy_parallel(void *dst, const void *src, size_t bytes) {
  const size_t chunk = 8u << 20;
  const long n = (long)((bytes + chunk - 1) / chunk);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    const size_t o = (size_t)i * chunk;
    memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o,
           std::min(chunk, bytes - o));
  }
}

// The GPU stage of one sub-swath: the SLCs are copied into page-locked
// staging and run through the plan's pipelined host-to-host call (per-burst
// uploads, kernels and downloads overlapped on three streams), then the
// coherence is debursted on the device.
int process_pair(const tops_config &c, const PairInputs &in, HostBuf &stage_m, HostBuf &stage_s,
                 Outputs &out) {
  const tops_swath_info &m = in.m, &s = in.s;
  const int k = in.k, L = m.lines_per_burst, W = m.samples_per_burst;
  tops_pair_opts o;
  D_TRY(tops_pair_opts_default(&o));
  o.win_rg = c.coh_win_rg;
  o.win_az = c.coh_win_az;
  o.esd_threshold = (float)c.esd_coh_threshold;
  o.reslave_full = 1;
  Plan plan;
  D_TRY(tops_pair_create(&m, &s, &o, in.dem_lines, in.dem_pixels, &plan.p));
  D_TRY(tops_pair_set_dem(plan.p, in.dem, in.lat0, in.lon0, in.dlat, in.dlon, in.win.data(),
                          nullptr));
  const size_t n = (size_t)k * L * W;
  void *ms = stage_m.get(n * 4), *ss = stage_s.get(n * 4);
  float *rs = static_cast<float *>(out.reslave.get(n * 8));
  float *re = static_cast<float *>(out.reslave_esd.get(n * 8));
  float *coh = static_cast<float *>(out.coh.get(n * 4));
  if (!ms || !ss || !rs || !re || !coh) return TOPS_E_NOMEM;
  copy_parallel(ms, in.ms, n * 4);
  copy_parallel(ss, in.ss, n * 4);
  std::vector<double> cpm(12 * k);
  out.shifts.assign(k > 1 ? k - 1 : 1, 0.0);
  D_TRY(tops_pair_process(plan.p, ms, ss, rs, re, coh, cpm.data(), out.shifts.data(), nullptr));
  out.k = k;
  out.W = W;
  out.L = L;
  out.stitch_lines = 0;
  if (c.stitch) {
    const int *fv = in.first_valid.data(), *lv = in.last_valid.data();
    int h = 0;
    D_TRY(tops_stitch_line_map(&m, fv, lv, 0, k - 1, nullptr, 0, &h));
    std::vector<int> map(h);
    D_TRY(tops_stitch_line_map(&m, fv, lv, 0, k - 1, map.data(), h, &h));
    tops_pair_buffers b;
    D_TRY(tops_pair_buffers_get(plan.p, &b));
    int *d_map = nullptr;
    float *d_out = nullptr;
    float *host = static_cast<float *>(out.stitched.get(sizeof(float) * (size_t)h * W));
    int r = host ? TOPS_OK : TOPS_E_NOMEM;
    if (r == TOPS_OK && (cudaMalloc(&d_map, sizeof(int) * h) != cudaSuccess ||
                         cudaMalloc(&d_out, sizeof(float) * (size_t)h * W) != cudaSuccess))
      r = TOPS_E_NOMEM;
    if (r == TOPS_OK && cudaMemcpy(d_map, map.data(), sizeof(int) * h,
                                   cudaMemcpyHostToDevice) != cudaSuccess)
      r = TOPS_E_CUDA;
    if (r == TOPS_OK)
      r = tops_stitch(b.coh, b.coh_pitch, d_out, (size_t)W * 4, d_map, h, (size_t)W * 4, nullptr);
    if (r == TOPS_OK && cudaMemcpy(host, d_out, sizeof(float) * (size_t)h * W,
                                   cudaMemcpyDeviceToHost) != cudaSuccess)
      r = TOPS_E_CUDA;
    cudaFree(d_map);
    cudaFree(d_out);
    (void)cudaGetLastError();
    D_TRY(r);
    out.stitch_lines = h;
  }
  return TOPS_OK;
}

// The writer stage: the reference's file names, <process_dir>/ReSlave-N.tif,
// ReSlaveESD-N.tif, Coh-N.tif (Main.cpp:98-101) and CohStitch-N.tif.
int write_outputs_untimed(const tops_config &c, const Outputs &o);

int write_outputs(const tops_config &c, Outputs &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const int r = write_outputs_untimed(c, o);
  o.write_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

int write_outputs_untimed(const tops_config &c, const Outputs &o) {
  const std::string dir = c.process_dir, tag = "-" + std::to_string(o.nsub) + ".tif";
  const int W = o.W, rows = o.k * o.L;
  D_TRY(tops_tiff_write((dir + "/ReSlave" + tag).c_str(), TOPS_TIFF_CFLOAT32, W, rows,
                        o.reslave.p, (size_t)W * 8));
  D_TRY(tops_tiff_write((dir + "/ReSlaveESD" + tag).c_str(), TOPS_TIFF_CFLOAT32, W, rows,
                        o.reslave_esd.p, (size_t)W * 8));
  D_TRY(tops_tiff_write((dir + "/Coh" + tag).c_str(), TOPS_TIFF_FLOAT32, W, rows, o.coh.p,
                        (size_t)W * 4));
  if (o.stitch_lines > 0)
    D_TRY(tops_tiff_write((dir + "/CohStitch" + tag).c_str(), TOPS_TIFF_FLOAT32, W,
                          o.stitch_lines, o.stitched.p, (size_t)W * 4));
  return TOPS_OK;
}

}  // namespace

// The sub-swaths run as a three-stage pipeline: a host thread loads
// sub-swath n + 1 (product files or the generator) and another writes
// sub-swath n - 1's rasters while the GPU processes sub-swath n.  The
// results are the same as processing the sub-swaths one after another.
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
  // products unless masterpath is empty or "(synthetic)"
  const bool products = c.masterpath[0] != '\0' && strcmp(c.masterpath, "(synthetic)") != 0;
  const auto t0 = std::chrono::steady_clock::now();
  HostBuf stage_m, stage_s;
  Outputs outs[2];
  std::future<std::unique_ptr<Loaded>> next =
      std::async(std::launch::async, load_subswath, std::cref(c), c.firstsubswath, products);
  std::future<int> writing;
  Outputs *pending = nullptr;   // the outputs `writing` writes
  int status = TOPS_OK;
  for (int nsub = c.firstsubswath; nsub <= c.lastsubswath && status == TOPS_OK; nsub++) {
    std::unique_ptr<Loaded> cur = next.get();
    if (nsub < c.lastsubswath)
      next = std::async(std::launch::async, load_subswath, std::cref(c), nsub + 1, products);
    status = cur->status;
    stats->load_seconds += cur->seconds;
    if (status != TOPS_OK) break;
    // the slot written two sub-swaths ago is free once that write is done
    Outputs &o = outs[nsub & 1];
    const auto tp = std::chrono::steady_clock::now();
    status = process_pair(c, cur->in, stage_m, stage_s, o);
    stats->process_seconds +=
        std::chrono::duration<double>(std::chrono::steady_clock::now() - tp).count();
    if (writing.valid()) {
      const int w = writing.get();
      stats->write_seconds += pending->write_seconds;
      if (status == TOPS_OK) status = w;
    }
    if (status != TOPS_OK) break;
    o.nsub = nsub;
    stats->subswaths++;
    stats->burst_pairs += o.k;
    for (int i = 0; i + 1 < o.k && i < TOPS_MAX_BURSTS; i++) stats->shifts[i] = o.shifts[i];
    pending = &o;
    writing = std::async(std::launch::async, write_outputs, std::cref(c), std::ref(o));
  }
  if (writing.valid()) {
    const int w = writing.get();
    stats->write_seconds += pending->write_seconds;
    if (status == TOPS_OK) status = w;
  }
  if (next.valid()) next.wait();   // a load still running when an error ended the loop
  stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return status;
}

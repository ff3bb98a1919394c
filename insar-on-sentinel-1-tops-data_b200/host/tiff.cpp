// tiff.cpp -- single-band raster files in the layout of the reference's
// GeoTIFF outputs, without GDAL.
//
// The reference writes every product (ReSlave, ReSlaveESD, coherence) and
// reads the SLCs through GDAL (TiffRead / TiffWrite, DataTypes.cpp:417-666):
// one band, CInt16, Float32 or CFloat32 pixels, uncompressed.  This file
// writes such rasters as baseline little-endian TIFF (strips of whole rows,
// SampleFormat 5 / 3 / 6 as GDAL writes them, so GDAL and other TIFF readers
// read them back) and reads uncompressed strip-organised single-band TIFFs of
// the same pixel types, little- or big-endian, such as the SLC measurement
// files.  No georeferencing tags are written on the outputs (the reference
// sets none on them either); the DEM path reads the GeoTIFF georeferencing
// of int16 or float32 elevation rasters as GDAL gives it (a geotransform
// from ModelPixelScale and ModelTiepoint), and can write it for test DEMs.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "tops_b200.h"

namespace {

struct PixelType {
  int bits, sample_format, bytes, comp_bytes;   // comp_bytes: byte-swap unit
};

bool pixel_type(int type, PixelType &p) {
  switch (type) {
    case TOPS_TIFF_CINT16: p = {32, 5, 4, 2}; return true;
    case TOPS_TIFF_FLOAT32: p = {32, 3, 4, 4}; return true;
    case TOPS_TIFF_CFLOAT32: p = {64, 6, 8, 4}; return true;
    case TOPS_TIFF_INT16: p = {16, 2, 2, 2}; return true;
    default: return false;
  }
}

struct Out {
  std::vector<uint8_t> b;
  void u16(uint16_t v) { b.push_back(v & 0xff); b.push_back(v >> 8); }
  void u32(uint32_t v) { for (int i = 0; i < 4; i++) b.push_back((v >> (8 * i)) & 0xff); }
  void entry(uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
    u16(tag);
    u16(type);
    u32(count);
    u32(value);
  }
};

constexpr uint16_t kShort = 3, kLong = 4, kDouble = 12;
constexpr uint16_t kTagPixelScale = 33550, kTagTiepoint = 33922, kTagGeoKeys = 34735;

// File reader with the byte order of the file.
struct In {
  FILE *f = nullptr;
  bool big = false;
  bool read(uint64_t off, void *dst, size_t n) {
    return fseeko(f, (off_t)off, SEEK_SET) == 0 && fread(dst, 1, n, f) == n;
  }
  uint32_t val(const uint8_t *p, int n) const {
    uint32_t v = 0;
    for (int i = 0; i < n; i++) v |= (uint32_t)p[big ? n - 1 - i : i] << (8 * i);
    return v;
  }
};

}  // namespace

namespace {

int write_tiff(const char *path, int type, int width, int height, const void *data, size_t pitch,
               const double *gt) {
  PixelType pt;
  if (!path || !data || width <= 0 || height <= 0 || !pixel_type(type, pt)) return TOPS_E_INVALID;
  const uint64_t row = (uint64_t)width * pt.bytes;
  if (pitch < row) return TOPS_E_INVALID;
  const uint64_t image = row * (uint64_t)height;
  // whole rows per strip, about 1 MiB each
  uint32_t rps = (uint32_t)((1u << 20) / row);
  if (rps < 1) rps = 1;
  if (rps > (uint32_t)height) rps = (uint32_t)height;
  const uint32_t nstrips = (uint32_t)((height + rps - 1) / rps);
  const uint64_t arrays = 8ull * nstrips;
  // georeferencing (gt != NULL): pixel scale (3 doubles), one tiepoint (6
  // doubles) and a geokey directory of 3 keys (16 shorts), after the strips'
  // arrays
  const uint64_t geo_bytes = gt ? 24 + 48 + 32 : 0;
  const int n_entries = gt ? 14 : 11;
  const uint64_t ifd_off = 8 + image + arrays + geo_bytes;
  if (ifd_off + 2 + 12 * n_entries + 4 >= (1ull << 32)) return TOPS_E_INVALID;   // classic TIFF
  FILE *f = fopen(path, "wb");
  if (!f) return TOPS_E_INVALID;
  Out h;
  h.b.push_back('I');
  h.b.push_back('I');
  h.u16(42);
  h.u32((uint32_t)ifd_off);
  bool ok = fwrite(h.b.data(), 1, h.b.size(), f) == h.b.size();
  const uint8_t *src = static_cast<const uint8_t *>(data);
  for (int y = 0; ok && y < height; y++) ok = fwrite(src + (size_t)y * pitch, 1, row, f) == row;
  // strip offsets and byte counts, then the IFD
  Out t;
  for (uint32_t i = 0; i < nstrips; i++) t.u32((uint32_t)(8 + (uint64_t)i * rps * row));
  for (uint32_t i = 0; i < nstrips; i++) {
    const uint32_t rows = (i + 1 == nstrips) ? (uint32_t)(height - i * rps) : rps;
    t.u32((uint32_t)(rows * row));
  }
  const uint32_t offs_at = (uint32_t)(8 + image), cnts_at = (uint32_t)(8 + image + 4ull * nstrips);
  const uint32_t scale_at = (uint32_t)(8 + image + arrays), tie_at = scale_at + 24,
                 keys_at = tie_at + 48;
  if (gt) {
    auto f64 = [&](double v) {
      uint64_t u;
      memcpy(&u, &v, 8);
      for (int i = 0; i < 8; i++) t.b.push_back((u >> (8 * i)) & 0xff);
    };
    f64(gt[1]);    // pixel scale x, y, z
    f64(-gt[5]);
    f64(0.0);
    f64(0.0);      // tiepoint: raster (0, 0, 0) -> model (x0, y0, 0)
    f64(0.0);
    f64(0.0);
    f64(gt[0]);
    f64(gt[3]);
    f64(0.0);
    // geokeys: version 1.1.0, 3 keys: model type geographic, raster type
    // pixel-is-area, geographic type WGS 84
    const uint16_t keys[16] = {1, 1, 0, 3, 1024, 0, 1, 2, 1025, 0, 1, 1, 2048, 0, 1, 4326};
    for (uint16_t k : keys) t.u16(k);
  }
  t.u16((uint16_t)n_entries);
  t.entry(256, kLong, 1, (uint32_t)width);
  t.entry(257, kLong, 1, (uint32_t)height);
  t.entry(258, kShort, 1, (uint32_t)pt.bits);
  t.entry(259, kShort, 1, 1);   // no compression
  t.entry(262, kShort, 1, 1);   // min-is-black
  t.entry(273, kLong, nstrips, nstrips == 1 ? 8u : offs_at);
  t.entry(277, kShort, 1, 1);
  t.entry(278, kLong, 1, rps);
  t.entry(279, kLong, nstrips, nstrips == 1 ? (uint32_t)image : cnts_at);
  t.entry(284, kShort, 1, 1);   // chunky
  t.entry(339, kShort, 1, (uint32_t)pt.sample_format);
  if (gt) {
    t.entry(kTagPixelScale, kDouble, 3, scale_at);
    t.entry(kTagTiepoint, kDouble, 6, tie_at);
    t.entry(kTagGeoKeys, kShort, 16, keys_at);
  }
  t.u32(0);
  ok = ok && fwrite(t.b.data(), 1, t.b.size(), f) == t.b.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? TOPS_OK : TOPS_E_INVALID;
}

}  // namespace

extern "C" int tops_tiff_write(const char *path, int type, int width, int height,
                               const void *data, size_t pitch) {
  return write_tiff(path, type, width, height, data, pitch, nullptr);
}

extern "C" int tops_tiff_write_georef(const char *path, int type, int width, int height,
                                      const void *data, size_t pitch, const double gt[6]) {
  if (!gt || gt[2] != 0.0 || gt[4] != 0.0 || !(gt[1] > 0.0) || !(gt[5] < 0.0))
    return TOPS_E_INVALID;
  return write_tiff(path, type, width, height, data, pitch, gt);
}

extern "C" int tops_tiff_read(const char *path, int *type, int *width, int *height, void *data,
                              size_t capacity) {
  if (!path || !type || !width || !height) return TOPS_E_INVALID;
  In in;
  in.f = fopen(path, "rb");
  if (!in.f) return TOPS_E_INVALID;
  int status = TOPS_E_INVALID;
  do {
    uint8_t hdr[8];
    if (!in.read(0, hdr, 8)) break;
    if (hdr[0] == 'I' && hdr[1] == 'I') in.big = false;
    else if (hdr[0] == 'M' && hdr[1] == 'M') in.big = true;
    else break;
    if (in.val(hdr + 2, 2) != 42) break;   // classic TIFF only
    const uint32_t ifd = in.val(hdr + 4, 4);
    uint8_t nb[2];
    if (!in.read(ifd, nb, 2)) break;
    const int n = (int)in.val(nb, 2);
    std::vector<uint8_t> e((size_t)n * 12);
    if (!in.read(ifd + 2, e.data(), e.size())) break;
    uint32_t w = 0, h = 0, bits = 0, comp = 1, spp = 1, planar = 1, fmt = 1, rps = 0;
    uint32_t n_off = 0, n_cnt = 0, off_type = 0, cnt_type = 0, off_val = 0, cnt_val = 0;
    bool tiled = false;
    const uint8_t *e0 = e.data();
    for (int i = 0; i < n; i++) {
      const uint8_t *p = e0 + 12 * i;
      const uint32_t tag = in.val(p, 2), ty = in.val(p + 2, 2), cnt = in.val(p + 4, 4);
      // a single SHORT sits in the first two bytes of the value field
      const uint32_t v = (ty == kShort && cnt == 1) ? in.val(p + 8, 2) : in.val(p + 8, 4);
      switch (tag) {
        case 256: w = v; break;
        case 257: h = v; break;
        case 258: bits = v; break;
        case 259: comp = v; break;
        case 273: n_off = cnt; off_type = ty; off_val = in.val(p + 8, 4);
                  if (ty == kShort && cnt == 1) off_val = v;
                  break;
        case 277: spp = v; break;
        case 278: rps = v; break;
        case 279: n_cnt = cnt; cnt_type = ty; cnt_val = in.val(p + 8, 4);
                  if (ty == kShort && cnt == 1) cnt_val = v;
                  break;
        case 284: planar = v; break;
        case 322: case 323: case 324: tiled = true; break;
        case 339: fmt = v; break;
        default: break;
      }
    }
    if (!w || !h || comp != 1 || spp != 1 || planar != 1 || tiled || !n_off || n_off != n_cnt) break;
    int t = 0;
    if (bits == 32 && fmt == 5) t = TOPS_TIFF_CINT16;
    else if (bits == 32 && fmt == 3) t = TOPS_TIFF_FLOAT32;
    else if (bits == 64 && fmt == 6) t = TOPS_TIFF_CFLOAT32;
    else if (bits == 16 && (fmt == 1 || fmt == 2)) t = TOPS_TIFF_INT16;   // as GDT_Int16
    else break;
    PixelType pt;
    pixel_type(t, pt);
    *type = t;
    *width = (int)w;
    *height = (int)h;
    const uint64_t row = (uint64_t)w * pt.bytes, total = row * h;
    if (!data) {
      status = TOPS_OK;
      break;
    }
    if (capacity < total) break;
    if (rps == 0 || rps > h) rps = h;
    // strip offsets and byte counts (inline when there is one strip)
    auto load = [&](uint32_t count, uint32_t ty, uint32_t val, std::vector<uint32_t> &out) {
      const int sz = ty == kShort ? 2 : 4;
      out.resize(count);
      if ((uint64_t)count * sz <= 4) {
        uint8_t raw[4];
        for (int k = 0; k < 4; k++) raw[k] = in.big ? (val >> (8 * (3 - k))) & 0xff : (val >> (8 * k)) & 0xff;
        for (uint32_t k = 0; k < count; k++) out[k] = count == 1 ? val : in.val(raw + k * sz, sz);
        return true;
      }
      std::vector<uint8_t> raw((size_t)count * sz);
      if (!in.read(val, raw.data(), raw.size())) return false;
      for (uint32_t k = 0; k < count; k++) out[k] = in.val(raw.data() + (size_t)k * sz, sz);
      return true;
    };
    std::vector<uint32_t> offs, cnts;
    if (!load(n_off, off_type, off_val, offs) || !load(n_cnt, cnt_type, cnt_val, cnts)) break;
    uint8_t *dst = static_cast<uint8_t *>(data);
    bool ok = true;
    uint64_t done = 0;
    for (uint32_t k = 0; ok && k < n_off && done < total; k++) {
      uint64_t want = (uint64_t)rps * row;
      if (done + want > total) want = total - done;
      ok = cnts[k] >= want && in.read(offs[k], dst + done, want);
      done += want;
    }
    if (!ok || done != total) break;
    if (in.big) {   // byte-swap each component
      for (uint64_t i = 0; i < total; i += pt.comp_bytes)
        for (int a = 0, b = pt.comp_bytes - 1; a < b; a++, b--) {
          const uint8_t x = dst[i + a];
          dst[i + a] = dst[i + b];
          dst[i + b] = x;
        }
    }
    status = TOPS_OK;
  } while (0);
  fclose(in.f);
  return status;
}

extern "C" int tops_tiff_georef(const char *path, double gt[6]) {
  if (!path || !gt) return TOPS_E_INVALID;
  In in;
  in.f = fopen(path, "rb");
  if (!in.f) return TOPS_E_INVALID;
  int status = TOPS_E_INVALID;
  do {
    uint8_t hdr[8];
    if (!in.read(0, hdr, 8)) break;
    if (hdr[0] == 'I' && hdr[1] == 'I') in.big = false;
    else if (hdr[0] == 'M' && hdr[1] == 'M') in.big = true;
    else break;
    if (in.val(hdr + 2, 2) != 42) break;
    const uint32_t ifd = in.val(hdr + 4, 4);
    uint8_t nb[2];
    if (!in.read(ifd, nb, 2)) break;
    const int n = (int)in.val(nb, 2);
    std::vector<uint8_t> e((size_t)n * 12);
    if (!in.read(ifd + 2, e.data(), e.size())) break;
    auto doubles = [&](const uint8_t *p, std::vector<double> &out) {
      const uint32_t cnt = in.val(p + 4, 4), off = in.val(p + 8, 4);
      if (in.val(p + 2, 2) != kDouble || cnt > 64) return false;
      std::vector<uint8_t> raw((size_t)cnt * 8);
      if (!in.read(off, raw.data(), raw.size())) return false;
      out.resize(cnt);
      for (uint32_t k = 0; k < cnt; k++) {
        uint64_t u = 0;
        for (int i = 0; i < 8; i++) u |= (uint64_t)raw[8 * k + (in.big ? 7 - i : i)] << (8 * i);
        memcpy(&out[k], &u, 8);
      }
      return true;
    };
    std::vector<double> scale, tie;
    int raster_type = 1;   // pixel is area unless the geokeys say otherwise
    bool ok = true;
    for (int i = 0; i < n && ok; i++) {
      const uint8_t *p = e.data() + 12 * i;
      const uint32_t tag = in.val(p, 2);
      if (tag == kTagPixelScale) ok = doubles(p, scale);
      else if (tag == kTagTiepoint) ok = doubles(p, tie);
      else if (tag == kTagGeoKeys && in.val(p + 2, 2) == kShort) {
        const uint32_t cnt = in.val(p + 4, 4);
        if (cnt < 4 || cnt > 4096) continue;   // 4 or more shorts: stored at an offset
        std::vector<uint8_t> raw((size_t)cnt * 2);
        if (!in.read(in.val(p + 8, 4), raw.data(), raw.size())) continue;
        const uint32_t nkeys = in.val(raw.data() + 6, 2);
        for (uint32_t k = 0; k < nkeys && 4 + 4 * k + 3 < cnt; k++) {
          const uint8_t *q = raw.data() + 8 * (k + 1);
          if (in.val(q, 2) == 1025 && in.val(q + 2, 2) == 0) raster_type = (int)in.val(q + 6, 2);
        }
      }
    }
    if (!ok || scale.size() < 2 || tie.size() < 6 || !(scale[0] > 0.0) || !(scale[1] > 0.0))
      break;
    // GDAL's geotransform of a north-up raster with one tiepoint
    gt[1] = scale[0];
    gt[5] = -scale[1];
    gt[2] = gt[4] = 0.0;
    gt[0] = tie[3] - tie[0] * gt[1];
    gt[3] = tie[4] - tie[1] * gt[5];
    if (raster_type == 2) {   // pixel is point: GDAL moves the origin half a pixel
      gt[0] -= 0.5 * gt[1];
      gt[3] -= 0.5 * gt[5];
    }
    status = TOPS_OK;
  } while (0);
  fclose(in.f);
  return status;
}

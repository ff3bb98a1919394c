// s1_front.cpp -- Sentinel-1 SAFE front end without tinyxml2 (tops_s1.h):
// a small XML reader, the annotation and precise-orbit readers, and
// master/slave burst matching.
//
// The element paths, the derived values and the selection rules follow the
// reference's readers: S1_Initialize (Func.cpp:135-574), the DC and FM-rate
// lists of ComputeDerampPara (Func.cpp:1868-2010), S1_OrbitInitialize
// (Func.cpp:695-819) and ComputerBurstOverlap with its geolocation helpers
// (Func.cpp:1133-1746).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <utility>
#include <vector>

#include "tops_s1.h"

namespace {

constexpr double kSol = 299792458.0;   // reference Constants.h

// ------------------------------------------------------------------ XML
struct XNode {
  std::string name, text;
  std::vector<std::pair<std::string, std::string>> attrs;
  std::vector<XNode> kids;
};

void append_decoded(std::string &out, const char *p, const char *e) {
  while (p < e) {
    if (*p != '&') {
      out.push_back(*p++);
      continue;
    }
    const char *semi = (const char *)memchr(p, ';', (size_t)(e - p));
    if (!semi) {
      out.push_back(*p++);
      continue;
    }
    const std::string ent(p + 1, semi);
    if (ent == "lt") out.push_back('<');
    else if (ent == "gt") out.push_back('>');
    else if (ent == "amp") out.push_back('&');
    else if (ent == "quot") out.push_back('"');
    else if (ent == "apos") out.push_back('\'');
    else if (!ent.empty() && ent[0] == '#') {
      const long c = ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X')
                         ? strtol(ent.c_str() + 2, nullptr, 16)
                         : strtol(ent.c_str() + 1, nullptr, 10);
      if (c > 0 && c < 128) out.push_back((char)c);   // ASCII only: the files are
    } else {                                          // ASCII numbers and names
      out.append(p, semi + 1);
    }
    p = semi + 1;
  }
}

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }
bool is_name(char c) {
  return !is_space(c) && c != '>' && c != '/' && c != '=' && c != '<' && c != '\0';
}

// Parses a whole document into root (its single top-level element).
bool parse_xml(const std::string &doc, XNode &root) {
  const char *p = doc.c_str(), *end = p + doc.size();
  std::vector<XNode *> stack;
  bool have_root = false;
  while (p < end) {
    if (*p != '<') {
      const char *q = (const char *)memchr(p, '<', (size_t)(end - p));
      if (!q) q = end;
      if (!stack.empty()) append_decoded(stack.back()->text, p, q);
      p = q;
      continue;
    }
    if (!strncmp(p, "<?", 2)) {
      const char *q = strstr(p, "?>");
      if (!q) return false;
      p = q + 2;
    } else if (!strncmp(p, "<!--", 4)) {
      const char *q = strstr(p + 4, "-->");
      if (!q) return false;
      p = q + 3;
    } else if (!strncmp(p, "<![CDATA[", 9)) {
      const char *q = strstr(p + 9, "]]>");
      if (!q || stack.empty()) return false;
      stack.back()->text.append(p + 9, q);
      p = q + 3;
    } else if (!strncmp(p, "<!", 2)) {
      const char *q = (const char *)memchr(p, '>', (size_t)(end - p));
      if (!q) return false;
      p = q + 1;
    } else if (p[1] == '/') {
      const char *n0 = p + 2, *n1 = n0;
      while (n1 < end && is_name(*n1)) n1++;
      if (stack.empty() || stack.back()->name.compare(0, std::string::npos, n0,
                                                      (size_t)(n1 - n0)) != 0)
        return false;
      const char *q = (const char *)memchr(n1, '>', (size_t)(end - n1));
      if (!q) return false;
      stack.pop_back();
      p = q + 1;
    } else {
      const char *n0 = p + 1, *n1 = n0;
      while (n1 < end && is_name(*n1)) n1++;
      if (n1 == n0) return false;
      XNode *node;
      if (stack.empty()) {
        if (have_root) return false;   // a second top-level element
        have_root = true;
        node = &root;
      } else {
        stack.back()->kids.emplace_back();
        node = &stack.back()->kids.back();
      }
      node->name.assign(n0, n1);
      p = n1;
      bool closed = false;
      for (;;) {
        while (p < end && is_space(*p)) p++;
        if (p >= end) return false;
        if (*p == '>') {
          p++;
          break;
        }
        if (*p == '/' && p + 1 < end && p[1] == '>') {
          p += 2;
          closed = true;
          break;
        }
        const char *a0 = p;
        while (p < end && is_name(*p)) p++;
        const std::string an(a0, p);
        while (p < end && is_space(*p)) p++;
        if (an.empty() || p >= end || *p != '=') return false;
        p++;
        while (p < end && is_space(*p)) p++;
        if (p >= end || (*p != '"' && *p != '\'')) return false;
        const char quote = *p++;
        const char *v1 = (const char *)memchr(p, quote, (size_t)(end - p));
        if (!v1) return false;
        std::string av;
        append_decoded(av, p, v1);
        node->attrs.emplace_back(an, av);
        p = v1 + 1;
      }
      // only the innermost open element's children grow, so the elements
      // on the stack (each in its parent's vector) do not move
      if (!closed) stack.push_back(node);
    }
  }
  return have_root && stack.empty();
}

const XNode *child(const XNode *n, const char *name) {
  if (!n) return nullptr;
  for (const XNode &k : n->kids)
    if (k.name == name) return &k;
  return nullptr;
}

const XNode *path(const XNode *n, std::initializer_list<const char *> names) {
  for (const char *nm : names) n = child(n, nm);
  return n;
}

const char *first_attr(const XNode *n) {
  return (n && !n->attrs.empty()) ? n->attrs[0].second.c_str() : nullptr;
}

bool read_file(const char *fn, std::string &out) {
  FILE *f = fopen(fn, "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t k;
  while ((k = fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, k);
  const bool ok = !ferror(f);
  fclose(f);
  return ok;
}

// status of loading a document: TOPS_E_INVALID unreadable, TOPS_E_CONFIG
// malformed
int load(const char *fn, XNode &root) {
  if (!fn) return TOPS_E_INVALID;
  std::string doc;
  if (!read_file(fn, doc)) return TOPS_E_INVALID;
  return parse_xml(doc, root) ? TOPS_OK : TOPS_E_CONFIG;
}

// ------------------------------------------------------ reference helpers
// utc2seconds (Func.cpp:630-636): seconds of the day; the date is ignored.
double utc2seconds(const char *utc) {
  int year = 0, month = 0, day = 0;
  double hour = 0, min = 0, sec = 0;
  sscanf(utc, "%d-%d-%dT%lf:%lf:%lf", &year, &month, &day, &hour, &min, &sec);
  return hour * 60 * 60 + min * 60 + sec;
}

// getIntArray / getDoubleArray (Func.cpp:638-658, 680-700): a value ends at
// every single space (so two spaces give an empty value, read as 0).
template <class T, class Conv>
std::vector<T> split_values(const std::string &s, Conv conv) {
  std::vector<T> v;
  std::string tmp;
  for (char c : s) {
    tmp.push_back(c);
    if (c == ' ') {
      v.push_back(conv(tmp.c_str()));
      tmp.clear();
    }
  }
  v.push_back(conv(tmp.c_str()));
  return v;
}
std::vector<int> int_array(const std::string &s) {
  return split_values<int>(s, [](const char *t) { return atoi(t); });
}
std::vector<double> double_array(const std::string &s) {
  return split_values<double>(s, [](const char *t) { return atof(t); });
}

// ---- element text as values (missing element: status TOPS_E_CONFIG)
struct Reader {
  int status = TOPS_OK;
  const XNode *need(const XNode *n) {
    if (!n) status = TOPS_E_CONFIG;
    return n;
  }
  const char *text(const XNode *n) {
    n = need(n);
    return n ? n->text.c_str() : "";
  }
  double num(const XNode *n) { return atof(text(n)); }
  int integer(const XNode *n) { return atoi(text(n)); }
  int count(const XNode *n) {   // the element's first attribute, as an int
    const char *a = first_attr(need(n));
    if (n && !a) status = TOPS_E_CONFIG;
    return a ? atoi(a) : 0;
  }
};

void copy_str(char *dst, size_t cap, const char *src) {
  snprintf(dst, cap, "%s", src ? src : "");
}

}  // namespace

// ------------------------------------------------------------ annotation
extern "C" int tops_s1_annotation_read(const char *xml_path, tops_swath_info *info,
                                       tops_s1_annotation *extra) {
  if (!info) return TOPS_E_INVALID;
  XNode root;
  int st = load(xml_path, root);
  if (st) return st;
  Reader R;
  const XNode *r = &root;
  const XNode *ii = path(r, {"imageAnnotation", "imageInformation"});
  const XNode *pi = path(r, {"generalAnnotation", "productInformation"});
  const XNode *spp = path(r, {"imageAnnotation", "processingInformation", "swathProcParamsList",
                              "swathProcParams"});
  tops_s1_annotation ex;
  memset(&ex, 0, sizeof ex);
  tops_swath_info I;
  memset(&I, 0, sizeof I);

  copy_str(ex.polarisation, sizeof ex.polarisation, R.text(path(r, {"adsHeader", "polarisation"})));
  ex.number_of_lines = R.integer(child(ii, "numberOfLines"));
  ex.number_of_samples = R.integer(child(ii, "numberOfSamples"));
  copy_str(ex.first_line_utc, sizeof ex.first_line_utc, R.text(child(ii, "productFirstLineUtcTime")));
  copy_str(ex.last_line_utc, sizeof ex.last_line_utc, R.text(child(ii, "productLastLineUtcTime")));
  I.first_line_time = utc2seconds(ex.first_line_utc);
  I.last_line_time = utc2seconds(ex.last_line_utc);
  I.dt = R.num(child(ii, "azimuthTimeInterval"));
  I.range_spacing = R.num(child(ii, "rangePixelSpacing"));
  ex.azimuth_pixel_spacing = R.num(child(ii, "azimuthPixelSpacing"));
  ex.radar_frequency = R.num(child(pi, "radarFrequency"));
  I.wavelength = kSol / ex.radar_frequency;
  I.rsr = R.num(child(pi, "rangeSamplingRate"));
  I.steering_rate_deg = R.num(child(pi, "azimuthSteeringRate"));
  ex.heading = R.num(child(pi, "platformHeading"));
  ex.ascending_node_time = utc2seconds(R.text(child(ii, "ascendingNodeTime")));
  I.prf = 1.0 / I.dt;
  I.az_bandwidth = R.num(path(spp, {"azimuthProcessing", "processingBandwidth"}));
  ex.range_bandwidth = R.num(path(spp, {"rangeProcessing", "processingBandwidth"}));
  I.slr_time = R.num(child(ii, "slantRangeTime")) / 2.0;
  ex.slr_time_last_pixel = I.slr_time + (ex.number_of_samples - 1) * I.range_spacing / kSol;

  const XNode *bl = path(r, {"swathTiming", "burstList"});
  const int nb = R.count(bl);
  I.lines_per_burst = R.integer(path(r, {"swathTiming", "linesPerBurst"}));
  I.samples_per_burst = R.integer(path(r, {"swathTiming", "samplesPerBurst"}));
  if (R.status) return R.status;
  if (nb < 1 || nb > TOPS_MAX_BURSTS || I.lines_per_burst < 1 || I.samples_per_burst < 1 ||
      !(I.dt > 0.0))
    return TOPS_E_INVALID;
  I.n_bursts = nb;
  const int L = I.lines_per_burst;

  // bursts: times, valid lines, valid pixel range (Func.cpp:330-428)
  int fvp = ex.number_of_samples, lvp = 0;
  int k = 0;
  for (const XNode &b : bl->kids) {
    if (k == nb) break;
    I.burst_first_line_time[k] = utc2seconds(R.text(child(&b, "azimuthTime")));
    I.burst_last_line_time[k] = I.burst_first_line_time[k] + (L - 1) * I.dt;
    const std::vector<int> fv = int_array(R.text(child(&b, "firstValidSample")));
    const std::vector<int> lv = int_array(R.text(child(&b, "lastValidSample")));
    if (R.status) return R.status;
    if ((int)fv.size() != L || (int)lv.size() != L) return TOPS_E_CONFIG;
    int first = -1, last = -1;
    for (int l = 0; l < L; l++) {
      if (fv[l] == -1) continue;
      if (fv[l] < fvp) fvp = fv[l];
      if (first == -1) first = last = l;
      else last++;   // the reference counts valid lines on from the first
    }
    for (int l = 0; l < L; l++)
      if (lv[l] != -1 && lv[l] > lvp) lvp = lv[l];
    ex.first_valid_line[k] = first;
    ex.last_valid_line[k] = last;
    ex.burst_first_valid_time[k] = I.burst_first_line_time[k] + first * I.dt;
    ex.burst_last_valid_time[k] = I.burst_first_line_time[k] + last * I.dt;
    k++;
  }
  if (k != nb) return TOPS_E_CONFIG;
  I.first_valid_pixel = fvp;
  ex.last_valid_pixel = lvp;

  // Doppler centroid estimates (Func.cpp:1885-1925)
  copy_str(ex.dc_method, sizeof ex.dc_method,
           R.text(path(r, {"imageAnnotation", "processingInformation", "dcMethod"})));
  const bool data_dc = strcmp(ex.dc_method, "Data Analysis") == 0;
  const XNode *dcl = path(r, {"dopplerCentroid", "dcEstimateList"});
  const int ndc = R.count(dcl);
  if (R.status) return R.status;
  if (ndc < 1 || ndc > TOPS_MAX_BURSTS + 4 || (int)dcl->kids.size() < ndc) return TOPS_E_INVALID;
  for (int e = 0; e < ndc; e++) {
    const XNode *d = &dcl->kids[e];
    const std::vector<double> c =
        double_array(R.text(child(d, data_dc ? "dataDcPolynomial" : "geometryDcPolynomial")));
    tops_poly &P = I.dc_list[e];
    P.aztime = utc2seconds(R.text(child(d, "azimuthTime")));
    P.t0 = R.num(child(d, "t0"));
    if (c.size() < 3) return TOPS_E_CONFIG;
    P.c0 = c[0];
    P.c1 = c[1];
    P.c2 = c[2];
  }
  I.n_dc = ndc;

  // azimuth FM rates (Func.cpp:1972-2010): c0/c1/c2 elements, or one
  // azimuthFmRatePolynomial
  const XNode *fml = path(r, {"generalAnnotation", "azimuthFmRateList"});
  const int nfm = R.count(fml);
  if (R.status) return R.status;
  if (nfm < 1 || nfm > TOPS_MAX_BURSTS + 4 || (int)fml->kids.size() < nfm) return TOPS_E_INVALID;
  for (int e = 0; e < nfm; e++) {
    const XNode *f = &fml->kids[e];
    tops_poly &P = I.fm_list[e];
    P.aztime = utc2seconds(R.text(child(f, "azimuthTime")));
    P.t0 = R.num(child(f, "t0"));
    const XNode *poly = child(f, "azimuthFmRatePolynomial");
    if (!poly) {
      P.c0 = R.num(child(f, "c0"));
      P.c1 = R.num(child(f, "c1"));
      P.c2 = R.num(child(f, "c2"));
    } else {
      const std::vector<double> c = double_array(poly->text);
      if (c.size() < 3) return TOPS_E_CONFIG;
      P.c0 = c[0];
      P.c1 = c[1];
      P.c2 = c[2];
    }
  }
  I.n_fm = nfm;

  // geolocation grid shape and the per-burst lat/lon boxes (Func.cpp:437-537)
  const XNode *gl = path(r, {"geolocationGrid", "geolocationGridPointList"});
  const int ngp = R.count(gl);
  if (R.status) return R.status;
  if (ngp < 2 || (int)gl->kids.size() < ngp) return TOPS_E_CONFIG;
  int per_line = 0;
  const int line0 = atoi(R.text(child(&gl->kids[0], "line")));
  for (int g = 0; g < ngp; g++) {
    if (atoi(R.text(child(&gl->kids[g], "line"))) != line0) break;
    per_line++;
  }
  if (R.status) return R.status;
  if (per_line < 2) return TOPS_E_CONFIG;
  ex.geo_points_per_line = per_line;
  ex.geo_lines = ngp / per_line;
  if (ex.geo_lines < nb + 1) return TOPS_E_CONFIG;   // rows b and b + 1 of every burst
  for (int b = 0; b < nb; b++) {
    double la[4], lo[4];
    const int idx[4] = {b * per_line, b * per_line + per_line - 1, (b + 1) * per_line,
                        (b + 1) * per_line + per_line - 1};
    for (int q = 0; q < 4; q++) {
      la[q] = R.num(child(&gl->kids[idx[q]], "latitude"));
      lo[q] = R.num(child(&gl->kids[idx[q]], "longitude"));
    }
    ex.burst_lat_max[b] = fmax(fmax(la[0], la[1]), fmax(la[2], la[3]));
    ex.burst_lat_min[b] = fmin(fmin(la[0], la[1]), fmin(la[2], la[3]));
    ex.burst_lon_max[b] = fmax(fmax(lo[0], lo[1]), fmax(lo[2], lo[3]));
    ex.burst_lon_min[b] = fmin(fmin(lo[0], lo[1]), fmin(lo[2], lo[3]));
  }
  if (R.status) return R.status;

  // keep the caller's state vectors (they come from the orbit file)
  I.n_sv = info->n_sv;
  memcpy(I.sv_t, info->sv_t, sizeof I.sv_t);
  memcpy(I.sv_x, info->sv_x, sizeof I.sv_x);
  memcpy(I.sv_y, info->sv_y, sizeof I.sv_y);
  memcpy(I.sv_z, info->sv_z, sizeof I.sv_z);
  *info = I;
  if (extra) *extra = ex;
  return TOPS_OK;
}

extern "C" int tops_s1_geogrid_read(const char *xml_path, int capacity, double *az_time,
                                    double *slr_time, double *lat, double *lon,
                                    double *incidence, int *lines, int *points) {
  if (capacity < 0) return TOPS_E_INVALID;
  XNode root;
  int st = load(xml_path, root);
  if (st) return st;
  Reader R;
  const XNode *gl = path(&root, {"geolocationGrid", "geolocationGridPointList"});
  const int ngp = R.count(gl);
  if (R.status) return R.status;
  if (ngp < 2 || (int)gl->kids.size() < ngp) return TOPS_E_CONFIG;
  int per_line = 0;
  const int line0 = atoi(R.text(child(&gl->kids[0], "line")));
  for (int g = 0; g < ngp; g++) {
    if (atoi(R.text(child(&gl->kids[g], "line"))) != line0) break;
    per_line++;
  }
  if (R.status) return R.status;
  if (per_line < 2) return TOPS_E_CONFIG;
  const int nl = ngp / per_line, n = nl * per_line;
  if (lines) *lines = nl;
  if (points) *points = per_line;
  if (n > capacity && (az_time || slr_time || lat || lon || incidence)) return TOPS_E_INVALID;
  for (int g = 0; g < n; g++) {
    const XNode *p = &gl->kids[g];
    if (az_time) az_time[g] = utc2seconds(R.text(child(p, "azimuthTime")));
    if (slr_time) slr_time[g] = R.num(child(p, "slantRangeTime")) / 2.0;
    if (lat) lat[g] = R.num(child(p, "latitude"));
    if (lon) lon[g] = R.num(child(p, "longitude"));
    if (incidence) incidence[g] = R.num(child(p, "incidenceAngle"));
  }
  return R.status;
}

// ------------------------------------------------------------------ orbit
namespace {

// DiffUTCTime (Func.cpp:660-678): whole seconds from first to last, across
// at most one day boundary.
int diff_utc(const char *first, const char *last) {
  int y1 = 0, mo1 = 0, d1 = 0, h1 = 0, mi1 = 0, s1 = 0;
  int y2 = 0, mo2 = 0, d2 = 0, h2 = 0, mi2 = 0, s2 = 0;
  sscanf(first, "%d-%d-%dT%d:%d:%d", &y1, &mo1, &d1, &h1, &mi1, &s1);
  sscanf(last, "%d-%d-%dT%d:%d:%d", &y2, &mo2, &d2, &h2, &mi2, &s2);
  const int a = h1 * 3600 + mi1 * 60 + s1, b = h2 * 3600 + mi2 * 60 + s2;
  return (y1 == y2 && mo1 == mo2 && d1 == d2) ? b - a : b + 86400 - a;
}

}  // namespace

extern "C" int tops_s1_orbit_read(const char *eof_path, const char *first_line_utc,
                                  const char *last_line_utc, tops_swath_info *info,
                                  double *vel) {
  if (!info || !first_line_utc || !last_line_utc) return TOPS_E_INVALID;
  int y = 0, mo = 0, d = 0, h = 0, mi = 0, s = 0;
  if (sscanf(first_line_utc, "%d-%d-%dT%d:%d:%d", &y, &mo, &d, &h, &mi, &s) != 6)
    return TOPS_E_INVALID;
  char prefix[64];
  snprintf(prefix, sizeof prefix, "%04d-%02d-%02dT%02d:%02d:%01d", y, mo, d, h, mi, s / 10);
  const int n = diff_utc(first_line_utc, last_line_utc) / 10 + 10;
  if (n < 1 || n > 32) return TOPS_E_INVALID;
  XNode root;
  int st = load(eof_path, root);
  if (st) return st;
  Reader R;
  const XNode *osvs = path(&root, {"Data_Block", "List_of_OSVs"});
  if (!R.need(osvs)) return R.status;
  const std::vector<XNode> &v = osvs->kids;
  int index = -1;
  for (int k = 0; k < (int)v.size(); k++) {
    const XNode *u = child(&v[k], "UTC");
    if (u && u->text.find(prefix) != std::string::npos) {
      index = k;
      break;
    }
  }
  // the reference reads from 4 vectors before the match
  if (index < 4 || index - 4 + n > (int)v.size()) return TOPS_E_CONFIG;
  for (int i = 0; i < n; i++) {
    const XNode *o = &v[index - 4 + i];
    const std::string utc = R.text(child(o, "UTC"));
    info->sv_t[i] = utc2seconds(utc.size() > 4 ? utc.c_str() + 4 : "");   // "UTC=..."
    info->sv_x[i] = R.num(child(o, "X"));
    info->sv_y[i] = R.num(child(o, "Y"));
    info->sv_z[i] = R.num(child(o, "Z"));
    if (vel) {
      vel[3 * i] = R.num(child(o, "VX"));
      vel[3 * i + 1] = R.num(child(o, "VY"));
      vel[3 * i + 2] = R.num(child(o, "VZ"));
    }
  }
  if (R.status) return R.status;
  info->n_sv = n;
  return TOPS_OK;
}

// ---------------------------------------------------------- burst matching
namespace {

constexpr double kEllA = 6378137.0;                           // WGS84 (DataTypes.cpp:177-183)
constexpr double kEllB = 6356752.3142451794975639665996337;

// Orbit polynomial of an info's state vectors (Polyfit_Orbit) with the
// reference's time normalisation about the middle vector.
struct Orbit {
  int n = 0;              // coefficients
  int npts = 0;
  double mid = 0.0;       // sv_t[npts / 2]
  double cx[8], cy[8], cz[8];
};

int fit_orbit(const tops_swath_info *s, Orbit &o) {
  if (s->n_sv < 3 || s->n_sv > 32) return TOPS_E_INVALID;
  o.npts = s->n_sv;
  o.mid = s->sv_t[s->n_sv / 2];
  return tops_polyfit_orbit(s->n_sv, s->sv_t, s->sv_x, s->sv_y, s->sv_z, o.cx, o.cy, o.cz, &o.n);
}

// getxyz / getxyzdot (Func.cpp:1409-1454): position and velocity per second
// at time t, the velocity from the power series of the derivative.
void orbit_xyz(const Orbit &o, double t, double p[3]) {
  const double tn = (t - o.mid) / 10.0;
  const double *c[3] = {o.cx, o.cy, o.cz};
  for (int k = 0; k < 3; k++) {
    double sum = 0.0;
    for (int d = o.n - 1; d >= 0; --d) sum = sum * tn + c[k][d];
    p[k] = sum;
  }
}
void orbit_xyzdot(const Orbit &o, double t, double v[3]) {
  const double tn = (t - o.mid) / 10.0;
  const double *c[3] = {o.cx, o.cy, o.cz};
  for (int k = 0; k < 3; k++) {
    double s = c[k][1];
    for (int i = 2; i <= o.n - 1; ++i) s += c[k][i] * (double(i) * pow(tn, double(i - 1)));
    v[k] = s / 10.0;
  }
}

// solve33 (Func.cpp:1462-1490): 3x3 LU without pivoting.
void solve33(double x[3], const double rhs[3], const double A[9]) {
  const double L10 = A[3] / A[0];
  const double L20 = A[6] / A[0];
  const double U11 = A[4] - L10 * A[1];
  const double L21 = (A[7] - (A[1] * L20)) / U11;
  const double U12 = A[5] - L10 * A[2];
  const double U22 = A[8] - L20 * A[2] - L21 * U12;
  const double b0 = rhs[0];
  const double b1 = rhs[1] - b0 * L10;
  const double b2 = rhs[2] - b0 * L20 - b1 * L21;
  x[2] = b2 / U22;
  x[1] = (b1 - U12 * x[2]) / U11;
  x[0] = (b0 - A[1] * x[1] - A[2] * x[2]) / A[0];
}

// lp2xyz (Func.cpp:1492-1584): the ground point of 1-based (line, pixel) of
// a burst on the ellipsoid -- Doppler, range and ellipsoid equations solved
// by Newton from pos (in/out), at most 11 steps, all updates < 1e-6 m.
void lp2xyz(double line, double pixel, const tops_swath_info *im, const Orbit &o, int burst,
            double pos[3]) {
  const double aztime = im->burst_first_line_time[burst] + (line - 1.0) / im->prf;
  const double rangetime = im->slr_time + (pixel - 1.0) / (im->rsr * 2);
  double ps[3], vs[3];
  orbit_xyz(o, aztime, ps);
  orbit_xyzdot(o, aztime, vs);
  for (int iter = 0; iter <= 10; ++iter) {
    const double d[3] = {pos[0] - ps[0], pos[1] - ps[1], pos[2] - ps[2]};
    const double r = kSol * rangetime;
    const double eq[3] = {-(vs[0] * d[0] + vs[1] * d[1] + vs[2] * d[2]),
                          -((d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) - r * r),
                          -((pos[0] * pos[0] + pos[1] * pos[1]) / (kEllA * kEllA) +
                            (pos[2] / kEllB) * (pos[2] / kEllB) - 1.0)};
    const double J[9] = {vs[0], vs[1], vs[2], 2 * d[0], 2 * d[1], 2 * d[2],
                         (2 * pos[0]) / (kEllA * kEllA), (2 * pos[1]) / (kEllA * kEllA),
                         (2 * pos[2]) / (kEllB * kEllB)};
    double x[3];
    solve33(x, eq, J);
    pos[0] += x[0];
    pos[1] += x[1];
    pos[2] += x[2];
    if (fabs(x[0]) < 1e-6 && fabs(x[1]) < 1e-6 && fabs(x[2]) < 1e-6) break;
  }
}

// xyz2aztime (Func.cpp:1349-1391): zero-Doppler time of xyz on an orbit,
// Newton from t0; the reference passes the orbit's middle time as an int.
double xyz2aztime(const double xyz[3], const Orbit &o, double t0) {
  const int mid = (int)o.mid;
  const double *c[3] = {o.cx, o.cy, o.cz};
  double az = t0;
  for (int iter = 0; iter <= 10; ++iter) {
    const double tn = (az - mid) / 10.0;
    double p[3], v[3], a[3];
    for (int k = 0; k < 3; k++) {
      double s = 0.0;
      for (int i = o.n - 1; i >= 0; --i) s = s * tn + c[k][i];
      p[k] = s;
      double sv = c[k][1], sa = 0.0;
      for (int i = 2; i < o.n; ++i) {
        sv += c[k][i] * (double(i) * pow(tn, i - 1));
        sa += c[k][i] * (double((i - 1) * i) * pow(tn, i - 2));
      }
      v[k] = sv / 10.0;
      a[k] = sa / 100.0;
    }
    const double d[3] = {xyz[0] - p[0], xyz[1] - p[1], xyz[2] - p[2]};
    const double sol = -(v[0] * d[0] + v[1] * d[1] + v[2] * d[2]) /
                       ((a[0] * d[0] + a[1] * d[1] + a[2] * d[2]) - v[0] * v[0] - v[1] * v[1] -
                        v[2] * v[2]);
    az += sol;
    if (fabs(sol) < 1e-010) break;
  }
  return az;
}

// Locating + getLatitude / getLontitude (Func.cpp:1133-1245): the grid cell
// around (aztime, rgtime).  The reference stores the bilinear weights in
// ints, so the value is that of a cell corner; it only seeds lp2xyz.
bool grid_latlon(const tops_s1_geogrid *g, double aztime, double rgtime, double &lat,
                 double &lon) {
  const int P = g->points, NL = g->lines;
  int j0 = -1, j1 = -1;
  if (rgtime < g->slr_time[0]) {
    j0 = 0;
    j1 = 1;
  } else if (rgtime > g->slr_time[P - 1]) {
    j0 = P - 2;
    j1 = P - 1;
  } else {
    for (int j = 0; j < P - 1; j++)
      if (g->slr_time[j] <= rgtime && g->slr_time[j + 1] > rgtime) {
        j0 = j;
        j1 = j + 1;
        break;
      }
  }
  if (j0 < 0) return false;
  const double muX = (rgtime - g->slr_time[j0]) / (g->slr_time[j1] - g->slr_time[j0]);
  int i0 = -1, i1 = -1;
  double muY = 0.0;
  for (int i = 0; i < NL - 1; i++) {
    const double a0 = (1 - muX) * g->az_time[i * P + j0] + muX * g->az_time[i * P + j1];
    const double a1 =
        (1 - muX) * g->az_time[(i + 1) * P + j0] + muX * g->az_time[(i + 1) * P + j1];
    if ((i == 0 && aztime < a0) || (i == NL - 2 && aztime >= a1) || (a0 <= aztime && a1 > aztime)) {
      i0 = i;
      i1 = i + 1;
      muY = (aztime - a0) / (a1 - a0);
      break;
    }
  }
  if (i0 < 0) return false;
  const int mx = (int)muX, my = (int)muY;   // the reference's int weights
  auto interp = [&](const double *v) {
    return (1 - my) * ((1 - mx) * v[i0 * P + j0] + mx * v[i0 * P + j1]) +
           my * ((1 - mx) * v[i1 * P + j0] + mx * v[i1 * P + j1]);
  };
  lat = interp(g->lat);
  lon = interp(g->lon);
  return true;
}

// Geodetic2Geographic (Func.cpp:1247-1260) at height 0.
void geodetic_xyz(double lat_deg, double lon_deg, double xyz[3]) {
  const double kPi = 3.1415926535897931;   // reference Constants.h
  const double e2 = 1.0 - (kEllB / kEllA) * (kEllB / kEllA);
  const double lat = lat_deg * kPi / 180.0, lon = lon_deg * kPi / 180.0;
  const double N = kEllA / sqrt(1.0 - e2 * (sin(lat) * sin(lat)));
  xyz[0] = N * cos(lat) * cos(lon);
  xyz[1] = N * cos(lat) * sin(lon);
  xyz[2] = (N - e2 * N) * sin(lat);
}

bool grid_ok(const tops_s1_geogrid *g) {
  return g && g->lines >= 2 && g->points >= 2 && g->az_time && g->slr_time && g->lat && g->lon;
}

// First burst whose first line comes at or after t, minus one (the
// reference's scan, bounded here by the burst count).
int burst_before(const tops_swath_info *s, double t) {
  int cc = 0;
  while (cc < s->n_bursts && t > s->burst_first_line_time[cc]) cc++;
  return cc - 1;
}

}  // namespace

extern "C" int tops_s1_burst_overlap(int burst0, int burstN, const tops_swath_info *M,
                                     const tops_s1_geogrid *mg, const tops_swath_info *S,
                                     const tops_s1_geogrid *sg, int *m_burst0, int *m_burstN,
                                     int *s_burst0, int *s_burstN) {
  if (!M || !S || !grid_ok(mg) || !grid_ok(sg) || !m_burst0 || !m_burstN || !s_burst0 ||
      !s_burstN)
    return TOPS_E_INVALID;
  const int B0 = burst0 - 1, BN = burstN - 1;
  if (B0 < 0 || BN < B0 || B0 >= M->n_bursts || M->n_bursts > TOPS_MAX_BURSTS ||
      S->n_bursts < 1 || S->n_bursts > TOPS_MAX_BURSTS || !(M->prf > 0) || !(S->prf > 0) ||
      !(M->rsr > 0) || !(S->rsr > 0))
    return TOPS_E_INVALID;
  Orbit mo, so;
  int st = fit_orbit(M, mo);
  if (!st) st = fit_orbit(S, so);
  if (st) return st;
  int mb0, mbN, sb0, sbN;
  // master burst centre on the slave orbit (Func.cpp:1627-1683)
  double az = M->burst_first_line_time[B0] + M->lines_per_burst / 2.0 * M->dt;
  double rg = (M->slr_time + M->slr_time) / 2.0;   // as the reference forms it
  double lat, lon, xyz[3];
  if (!grid_latlon(mg, az, rg, lat, lon)) return TOPS_E_INVALID;
  geodetic_xyz(lat, lon, xyz);
  lp2xyz(M->lines_per_burst / 2, M->samples_per_burst / 2, M, mo, B0, xyz);
  double zdt = xyz2aztime(xyz, so, az);
  if (zdt > S->last_line_time) return TOPS_E_CONFIG;   // no overlap
  if (zdt < S->last_line_time && zdt > S->first_line_time) {
    mb0 = B0;
    sb0 = burst_before(S, zdt);
    if (BN - mb0 <= S->n_bursts - 1 - sb0) {
      mbN = BN;
      sbN = sb0 + (mbN - mb0);
    } else {
      sbN = S->n_bursts - 1;
      mbN = mb0 + (sbN - sb0);
    }
  } else {
    // slave's first burst centre on the master orbit (Func.cpp:1685-1741);
    // the slave's last-pixel time from its samples per burst
    az = S->burst_first_line_time[0] + S->lines_per_burst / 2 * S->dt;
    rg = (S->slr_time + (S->slr_time + (S->samples_per_burst - 1) * S->range_spacing / kSol)) / 2.0;
    if (!grid_latlon(sg, az, rg, lat, lon)) return TOPS_E_INVALID;
    geodetic_xyz(lat, lon, xyz);
    lp2xyz(S->lines_per_burst / 2, S->samples_per_burst / 2, S, so, 0, xyz);
    zdt = xyz2aztime(xyz, mo, az);
    if (!(zdt < M->last_line_time && zdt > M->first_line_time)) return TOPS_E_CONFIG;
    sb0 = 0;
    mb0 = burst_before(M, zdt);
    if (BN - mb0 <= S->n_bursts - 1) {
      mbN = BN;
      sbN = sb0 + (mbN - mb0);
    } else {
      sbN = S->n_bursts - 1;
      mbN = mb0 + (sbN - sb0);
    }
  }
  // a match before the first burst (the reference would index burst -1)
  if (mb0 < 0 || sb0 < 0 || mbN < mb0 || sbN < sb0) return TOPS_E_CONFIG;
  *m_burst0 = mb0;
  *m_burstN = mbN;
  *s_burst0 = sb0;
  *s_burstN = sbN;
  return TOPS_OK;
}

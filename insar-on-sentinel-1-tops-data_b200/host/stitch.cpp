// stitch.cpp -- debursting of one sub-swath: which burst line each output
// line takes (host), for the row gather of csrc/stitch.cu.
//
// The reference (Stitch_OneSubswath and getLineIdxInMetaData,
// Func.cpp:2766-2933) walks the output lines from the first valid line of
// burst b0 to the last valid line of burst bN at the azimuth interval.  A
// line covered by one burst takes that burst's nearest line; a line covered
// by two (an overlap) takes the earlier burst up to the midpoint between the
// earlier burst's last line time and the later burst's first line time and
// the later burst after it, except that the burst before b0 and the burst
// after bN are never chosen.  A line in the interval after the swath's last
// line takes the swath's last line.  The reference writes the rows from a
// file; here the map drives a device gather.
#include <math.h>

#include "tops_b200.h"

namespace {

// getLineIdxInMetaData (Func.cpp:2766-2820): full-swath line of time t, or -1.
int line_of_time(const tops_swath_info &m, double t, int b0, int bN) {
  int sy0 = -1, sy1 = -1, k0 = -1, k1 = -1, hits = 0;
  for (int i = 0; i < m.n_bursts && hits < 2; i++) {
    if (!(t >= m.burst_first_line_time[i] && t < m.burst_last_line_time[i])) continue;
    const int sy = i * m.lines_per_burst + (int)((t - m.burst_first_line_time[i]) / m.dt + 0.5);
    if (hits == 0) {
      sy0 = sy;
      k0 = i;
    } else {
      sy1 = sy;
      k1 = i;
    }
    hits++;
  }
  if (sy0 != -1 && sy1 != -1) {
    if (k1 == b0) return sy1;
    if (k1 == bN + 1) return sy0;
    const double mid = (m.burst_last_line_time[k0] + m.burst_first_line_time[k1]) / 2.0;
    if (t > mid) return sy1;
  }
  const double tl = m.burst_last_line_time[m.n_bursts - 1];
  if (t < tl + m.dt && t >= tl) sy0 = m.n_bursts * m.lines_per_burst - 1;
  return sy0;
}

}  // namespace

extern "C" int tops_stitch_line_map(const tops_swath_info *m, const int *first_valid,
                                    const int *last_valid, int burst0, int burstN, int *line_map,
                                    int capacity, int *height) {
  if (!m || !first_valid || !last_valid || !height || burst0 < 0 || burstN < burst0 ||
      burstN >= m->n_bursts || m->n_bursts > TOPS_MAX_BURSTS || !(m->dt > 0.0))
    return TOPS_E_INVALID;
  // Stitch_OneSubswath (Func.cpp:2822-2860): output lines and their times
  const double t_first = m->burst_first_line_time[burst0] + first_valid[burst0] * m->dt;
  const double t_last = m->burst_first_line_time[burstN] + last_valid[burstN] * m->dt;
  const int y_min = (int)((t_first - m->first_line_time) / m->dt);
  const int y_max = (int)((t_last - m->first_line_time) / m->dt);
  const int h = y_max - y_min + 1;
  *height = h;
  if (h <= 0) return TOPS_E_INVALID;
  if (!line_map) return TOPS_OK;   // size query
  if (capacity < h) return TOPS_E_INVALID;
  const int rows = (burstN - burst0 + 1) * m->lines_per_burst;   // rows of the burst stack
  for (int yy = 0; yy < h; yy++) {
    const double t = t_first + yy * m->dt;
    int idx = line_of_time(*m, t, burst0, burstN);
    if (idx == -1) return TOPS_E_INVALID;   // the reference stops here (Func.cpp:2866-2873)
    idx -= burst0 * m->lines_per_burst;
    if (idx < 0 || idx >= rows) return TOPS_E_INVALID;   // outside the stacked bursts
    line_map[yy] = idx;
  }
  return TOPS_OK;
}

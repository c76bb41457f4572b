// shard.cpp -- splitting one batch of sources or templates over devices.
//
// Sources and likelihood templates are independent units whose device cost is
// close to (samples x harmonics); a batch is divided over devices by greedy
// longest-processing-time (LPT) scheduling: units in decreasing cost, each to
// the device with the least cost so far (ties to the lowest index, so that the
// split is a pure function of the costs).  LPT's makespan is within 4/3 of the
// optimum.  No data moves between devices: every device generates its own
// units, and only per-unit results (waveform rows, or (d_h, h_h) pairs of a
// likelihood batch) are gathered.
#include <stdint.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "aak.h"

extern "C" int aak_lpt_partition(const double *cost, int64_t n, int32_t parts, int32_t *assign, double *load) {
  if (n < 0 || parts <= 0 || (n > 0 && (!cost || !assign))) return AAK_ERR_INVALID_PARAM;
  for (int64_t i = 0; i < n; ++i)
    if (!(cost[i] >= 0.0)) return AAK_ERR_INVALID_PARAM;  // NaN or negative
  std::vector<int64_t> order(n);
  std::iota(order.begin(), order.end(), (int64_t)0);
  // decreasing cost; equal costs keep their input order
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cost[a] > cost[b]; });
  std::vector<double> acc(parts, 0.0);
  for (const int64_t i : order) {
    int best = 0;
    for (int p = 1; p < parts; ++p)
      if (acc[p] < acc[best]) best = p;
    assign[i] = best;
    acc[best] += cost[i];
  }
  if (load)
    for (int p = 0; p < parts; ++p) load[p] = acc[p];
  return AAK_OK;
}

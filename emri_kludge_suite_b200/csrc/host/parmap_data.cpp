// parmap_data.cpp -- see parmap_data.hpp.
#include "parmap_data.hpp"

#include <cmath>

#include "../aak_common.hpp"
#include "kerr.hpp"
#include "pipeline.hpp"

namespace aak {

namespace {
// SplitMix64 (Steele, Lea & Flood 2014) as a counter-based stream.
inline uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
struct Stream {
  uint64_t key, ctr = 0;
  double uniform() { return (double)(splitmix(key + 0x632BE59BD9B4E019ull * ++ctr) >> 11) * 0x1.0p-53; }
};
}  // namespace

double separatrix_p(double e, double cosi, double a, double tol) {
  auto stable = [&](double p) {
    KerrGeodesic g;
    g.set_full(p, e, cosi, a);
    return g.stable == 1 || g.stable == 0;
  };
  double lo = 1.0, hi = 15.0;
  while (!stable(hi) && hi < 1e3) hi *= 1.5;
  while (hi - lo > tol) {
    const double mid = 0.5 * (lo + hi);
    if (stable(mid)) hi = mid;
    else lo = mid;
  }
  return hi;
}

void parmap_draw(uint64_t seed, uint64_t index, double x[4]) {
  Stream s{splitmix(seed) ^ splitmix(index * 0xD1B54A32D192ED03ull + 1)};
  double e;
  do e = 0.7 * s.uniform();
  while (e < 1e-3);
  const double iota = kPi * s.uniform();
  const double a = 0.95 * s.uniform();
  const double ps = separatrix_p(e, std::cos(iota), a, 1e-9);
  const double p = ps + 0.1 + (20.0 - ps - 0.1) * s.uniform();
  x[0] = p;
  x[1] = e;
  x[2] = iota;
  x[3] = a;
}

void parmap_to_coords(const double x[4], double M, const double map[3], double y[3]) {
  y[0] = map[0] * std::sqrt(x[0]);
  y[1] = map[1] / M;
  y[2] = map[2] - x[3];
}

void parmap_from_coords(const double x[4], double M, const double y[3], double map[3]) {
  map[0] = y[0] / std::sqrt(x[0]);
  map[1] = y[1] * M;
  map[2] = y[2] + x[3];
}

void kerr_frequencies(const double x[4], double Omega[3]) {
  KerrGeodesic g;
  g.set_full(x[0], x[1], std::cos(x[2]), x[3]);
  g.frequencies(Omega);
}

}  // namespace aak

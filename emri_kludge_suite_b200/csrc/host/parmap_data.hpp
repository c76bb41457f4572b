// parmap_data.hpp -- points, labels and batched solves for the learned warm
// start of the Kerr -> AK parameter map (ParMap, src/suite/KSParMap.cc:397-440).
//
// A point is x = (p, e, iota, a).  Its label is the solution of the plain map
// solve in "map coordinates" y = (v_map sqrt(p), M_map / M, s_map - a), which
// are O(1), vary smoothly over the domain and do not depend on M (the map
// equations are homogeneous in M).
#pragma once

#include <stdint.h>

namespace aak {

// Mass at which labels are generated (the map coordinates do not depend on it).
constexpr double kParmapLabelMass = 1.0e6;

// Separatrix: the smallest stable semi-latus rectum at (e, cos iota, a), by
// bisection on the stability flag of the generic Kerr geodesic -- the test the
// reference's LSO search bisects on (src/suite/GKTrajFast.cc constructor, with
// IEKG::Stable).  Roots that are not finite count as unstable.
double separatrix_p(double e, double cosi, double a, double tol = 1e-9);

// Point `index` of the seeded distribution p ~ U(p_sep + 0.1, 20),
// e ~ U(0, 0.7) (redrawn below 1e-3: the reference's IEKG rejects e = 0),
// iota ~ U(0, pi), a ~ U(0, 0.95).  Counter-based: independent of threading.
void parmap_draw(uint64_t seed, uint64_t index, double x[4]);

void parmap_to_coords(const double x[4], double M, const double map[3], double y[3]);
void parmap_from_coords(const double x[4], double M, const double y[3], double map[3]);

// |f|_1 of the map residual at `map` (the reference's convergence measure).
double parmap_residual_norm(const double Omega[3], double M, double e, double iota, const double map[3]);

// Kerr fundamental frequencies at x (cycles per unit M).
void kerr_frequencies(const double x[4], double Omega[3]);

}  // namespace aak

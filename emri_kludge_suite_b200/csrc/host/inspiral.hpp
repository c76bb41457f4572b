// inspiral.hpp -- coarse generic-Kerr inspiral in radiation-reaction time
// (the role of the reference class GKTrajFast, src/suite/GKTrajFast.cc).
#pragma once

namespace aak {

struct TrajPoint {
  double t;  // radiation-reaction time (units of M^2/mu)
  double p, e, cosi;
};

// Outcome codes of KerrInspiral::eccentric (same meaning as the reference's
// Eccentric return values, src/suite/GKTrajFast.cc:135-141).
enum InspiralFlag {
  kInspMaxSteps = 2,
  kInspCircularised = 1,
  kInspPlunged = 0,
  kInspUnstableStart = -1,
  kInspInvalid = -2,
};

class KerrInspiral {
 public:
  // Builds the 2x2 last-stable-orbit table (equatorial pro/retrograde,
  // e = 0 and e = 0.9995) used to keep steps outside the LSO.
  KerrInspiral(double cosi0, double spin);

  // Coarse inspiral from (p0, e0) with radiation-reaction step dt_start;
  // writes up to steps_max points, returns an InspiralFlag.
  int eccentric(double p0, double e0, double dt_start, int steps_max, TrajPoint *out, int *steps_taken);

  double p_lso(double csi, double e) const;
  double lso_table(int j, int i) const { return p_lso_[j][i]; }

  // dp/dt, de/dt, d(cos iota)/dt; false when the rates are not defined.
  bool derivs(const double x[3], double dxdt[3]) const;

 private:
  int take_step(double x[3], double t1, double &dt) const;
  int integrate(double y[3], double x1, double x2) const;
  bool midpoint(const double y[3], const double dydx[3], double h, int nsub, double out[3]) const;

  double cosi0_, a_;
  double p_lso_[2][2];  // [cos-iota index: 0 -> +1, 1 -> -1][e index: 0 -> 0, 1 -> 0.9995]
};

}  // namespace aak

// ak_rates.hpp -- the AK radiation-reaction rates dv/dt and de/dt (3PN,
// O(e^6); src/suite/KSParMap.cc:86-144), shared by the host planning
// (pipeline.cpp, where T is also a vector of doubles, one source per lane)
// and the device evolution of the coarse trajectories (ak_evolve.cu).
#pragma once

#include <cmath>

#include "aak_common.hpp"

#ifdef __CUDACC__
#define AAK_HD_FI __host__ __device__ __forceinline__
#else
#define AAK_HD_FI inline __attribute__((always_inline))
#endif

namespace aak {

// dv/dt and de/dt of the AK equations (KSParMap.cc:86-144); lv = log(v) and
// ome15 = (1 - e^2)^1.5 are shared by the two.  T is double, or a vector of
// doubles (one source per lane: the same operations lane by lane).
template <class T>
AAK_HD_FI T dvdt_core(T v, T e, T Y, T m, T M, T q, T lv, T ome15) {
  const T v2 = v * v, v3 = v2 * v, v6 = v3 * v3;
  const T e2 = e * e, e4 = e2 * e2, e6 = e4 * e2;
  const T Y2 = Y * Y, q2 = q * q;
  const double l2 = std::log(2.), l3 = std::log(3.), l5 = std::log(5.);
  T s = 1. + 7. * e2 * (1. / 8.);
  s += (-5944. - 7040. * e2 + 8539. * e4) * v2 * (1. / 2688.);
  s -= v3 * ((-18432. - 55872. * e2 - 7056. * e4 + 49. * e6) * kPi + 48. * (1064. + 1516. * e2 + 475. * e4) * q * Y) * (1. / 4608.);
  s += v3 * v2 *
       ((-4791168. - 28113984. * e2 + 12239226. * e4 + 4005097. * e6) * kPi -
        144. * (139296. + 58408. * e2 + 249968. * e4 + 106707. * e6) * q * Y) /
       774144.;
  s += v2 * v2 *
       (953325. * e6 + 8. * (34103. + 189. * q2 * (-329. + 815. * Y2)) + 12. * e2 * (-526955. + 126. * q2 * (-929. + 1431. * Y2)) +
        3. * e4 * (-1232809. + 63. * q2 * (-1051. + 2997. * Y2))) /
       145152.;
  T c6 = 117.72574285227559 - 1712. * kEulerGamma * (1. / 105.) + 16. * kPi2Trunc * (1. / 3.) - 331. * q2 * (1. / 192.) -
              289. * kPi * q * Y * (1. / 6.) + 145759. * q2 * Y2 * (1. / 1344.) - 3424. * l2 * (1. / 105.);
  c6 += e2 * (764.5906705662063 - 24503. * kEulerGamma * (1. / 210.) + 229. * kPi2Trunc * (1. / 6.) + 2129. * q2 * (1. / 42.) -
              4225. * kPi * q * Y * (1. / 24.) + 27191. * q2 * Y2 * (1. / 224.) + 1391. * l2 * (1. / 30.) - 78003. * l3 * (1. / 280.));
  c6 += e4 * (723.1604428881717 - 11663. * kEulerGamma * (1. / 140.) + 109. * kPi2Trunc * (1. / 4.) - 56239. * q2 * (1. / 10752.) -
              17113. * kPi * q * Y * (1. / 192.) + 414439. * q2 * Y2 * (1. / 3584.) - 418049. * l2 * (1. / 84.) + 3042117. * l3 * (1. / 1120.));
  c6 += e6 * (202.0979603432282 - 2461. * kEulerGamma * (1. / 560.) + 23. * kPi2Trunc * (1. / 16.) - 3571. * q2 * (1. / 3584.) -
              108577. * kPi * q * Y * (1. / 13824.) + 41071. * q2 * Y2 * (1. / 1536.) + 94138279. * l2 * (1. / 2160.) - 42667641. * l3 * (1. / 3584.) -
              1044921875. * l5 * (1. / 96768.));
  c6 -= 107. * (256. + 1832. * e2 + 1308. * e4 + 69. * e6) * lv * (1. / 1680.);
  s += v6 * c6;
  // the source's constant factor first and no division: the step's critical path is a serial recurrence
  return (32. / 5.) * (m / (M * M)) * ome15 * v6 * v3 * s;
}

template <class T>
AAK_HD_FI T dedt_core(T v, T e, T Y, T m, T M, T q, T lv, T ome15) {
  const T v2 = v * v, v3 = v2 * v, v6 = v3 * v3;
  const T e2 = e * e, e4 = e2 * e2;
  const T Y2 = Y * Y, q2 = q * q;
  const double l2 = std::log(2.), l3 = std::log(3.), l5 = std::log(5.);
  T s = 2451456. + 975744. * e2;
  s += 144. * (-54792. - 18600. * e2 + 22579. * e4) * v2;
  s += 84. * v3 * ((189120. + 286512. * e2 + 24217. * e4) * kPi - 48. * (7032. + 5592. * e2 + 1313. * e4) * q * Y);
  s += 3. * v3 * v2 * ((-16885824. - 42474444. * e2 + 5678971. * e4) * kPi - 48. * (106568. + 187862. * e2 + 442811. * e4) * q * Y);
  s += 8. * v2 * v2 *
       (6. * e2 * (-2070667. + 126. * q2 * (-2975. + 4009. * Y2)) + 8. * (-286397. + 63. * q2 * (-3179. + 5869. * Y2)) +
        e4 * (-3506201. + 63. * q2 * (-3191. + 9009. * Y2)));
  T c6 = 241.02948298890263 - 82283. * kEulerGamma * (1. / 1995.) + 769. * kPi2Trunc * (1. / 57.) + 180255. * q2 * (1. / 8512.) -
              11809. * kPi * q * Y * (1. / 152.) + 598987. * q2 * Y2 * (1. / 8512.) - 11021. * l2 * (1. / 285.) - 234009. * l3 * (1. / 5320.);
  c6 += e2 * (1048.5728116817568 - 297674. * kEulerGamma * (1. / 1995.) + 2782. * kPi2Trunc * (1. / 57.) + 536653. * q2 * (1. / 8512.) -
              91375. * kPi * q * Y * (1. / 608.) + 356845. * q2 * Y2 * (1. / 8512.) - 2982946. * l2 * (1. / 1995.) + 1638063. * l3 * (1. / 3040.));
  c6 += e4 * (725.9069951397873 - 1147147. * kEulerGamma * (1. / 15960.) + 10721. * kPi2Trunc * (1. / 456.) + 56509. * q2 * (1. / 9728.) -
              1739605. * kPi * q * Y * (1. / 29184.) + 3248951. * q2 * Y2 * (1. / 68096.) + 760314287. * l2 * (1. / 47880.) -
              1022385321. * l3 * (1. / 340480.) - 1044921875. * l5 * (1. / 204228.));
  c6 -= 107. * (6152. + 22256. * e2 + 10721. * e4) * lv * (1. / 15960.);
  s += 2451456. * v6 * c6;
  return -((1. / 120960.) * (m / (M * M)) * e * ome15 * v6 * v2 * s);
}

// Inlined into the evolution loops, so that the compiler keeps the terms that
// depend only on the source (spin, inclination) out of the per-knot work.
AAK_HD_FI void ak_rates(double v, double e, double Y, double m, double M, double q,
                                                    double *edot, double *vdot) {
  const double ome = 1. - e * e;
  const double lv = std::log(v), ome15 = ome * std::sqrt(ome);
  *edot = dedt_core(v, e, Y, m, M, q, lv, ome15);
  *vdot = dvdt_core(v, e, Y, m, M, q, lv, ome15);
}

}  // namespace aak

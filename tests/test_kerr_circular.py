"""The circular-orbit constants of the inspiral rates: fast path against the plain bisection.

CircularConstants::set (csrc/host/kerr.cpp) finds the energy of an inclined
circular Kerr orbit as the reference's CKG does (src/circ/CKG.cc:86-127): a
bisection between the prograde and retrograde equatorial energies that stops
at the first midpoint whose cos(iota) is within 1e-9.  Its fast path finds
the root by Newton, then replays the bisection, evaluating only the midpoints
near the root.  The result must be the bisection's, bit for bit (the inspiral
rates, and through them the coarse trajectory, depend on it).  This test
builds a small program against kerr.cpp and compares the two on random
radii, inclinations and spins, small spins and nearly equatorial orbits
included.
"""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(REPO, "emri_kludge_suite_b200", "csrc", "host")

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include "kerr.hpp"
using namespace aak;
int main() {
  std::mt19937_64 rng(11);
  std::uniform_real_distribution<double> U(0, 1);
  long bad = 0, n = 0;
  for (int k = 0; k < 300000; ++k) {
    const double a = (k % 10 == 0) ? 1e-3 * U(rng) : 0.99 * U(rng);
    const double c = (k % 7 == 0) ? (U(rng) < 0.5 ? -1 : 1) * (1 - 1e-4 * U(rng)) : 2 * U(rng) - 1;
    const double r = kerr_isco_pro(a) + 0.3 + 40 * U(rng) * U(rng);
    CircularConstants x, y;
    x.set(r, c, a, false);
    y.set(r, c, a, true);
    ++n;
    if (std::memcmp(&x, &y, sizeof(x)) != 0 && !(std::isnan(x.E) && std::isnan(y.E))) ++bad;
    // a run of close calls, as the inspiral makes them (the fast path starts from the previous root)
    if (k % 1000 == 0)
      for (int j = 0; j < 200; ++j) {
        CircularConstants u, w;
        u.set(r * (1 - 1e-6 * j), c, a, false);
        w.set(r * (1 - 1e-6 * j), c, a, true);
        ++n;
        if (std::memcmp(&u, &w, sizeof(u)) != 0) ++bad;
      }
  }
  std::printf("%ld %ld\n", n, bad);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_fast_circular_energy_equals_bisection(tmp_path):
    src = tmp_path / "circ.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "circ"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", HOST, "-I", os.path.join(REPO, "emri_kludge_suite_b200", "csrc"),
                    "-I", os.path.join(REPO, "include"), str(src), os.path.join(HOST, "kerr.cpp"), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    n, bad = int(out[0]), int(out[1])
    assert n > 300000 and bad == 0, (n, bad)

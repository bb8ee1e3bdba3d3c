/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the OpenCFD-Comb hot path.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load
 * it, and only as the checker. The product (opencfd-comb_b200/) never includes or links it.
 *
 * Shared helpers of the oracle: array indexing in the reference's Fortran layout and the
 * integer-power expansion gfortran -O3 emits for x**n with a constant n (GCC's powi
 * addition chain: x**3 = x**2*x, x**4 = x**2*x**2, x**5 = x**2*x**3).
 */
#pragma once
#include <cmath>

namespace ocfd_oracle {

inline double p2(double x) { return x * x; }
inline double p3(double x) { double a = x * x; return a * x; }
inline double p4(double x) { double a = x * x; return a * a; }
inline double p5(double x) { double a = x * x; double b = a * x; return a * b; }

/* libgcc __powidf2 (used by gfortran for x**n with a run-time integer n) */
inline double powi_rt(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

/* Fortran SIGN(1.d0, x) */
inline double fsign1(double x) { return std::signbit(x) ? -1.0 : 1.0; }

}  // namespace ocfd_oracle

// ref_cubic_prelude.hpp — included by ref_access_prelude.hpp in the
// cubic-spline build of the reference (MATTER_REF_CUBIC).  TEST INFRASTRUCTURE ONLY.
//
// tools.hpp:21 fixes SPLINEDEG at 2 and the reference directory is read-only,
// so this prelude includes tools.hpp first with its quadratic basis functions
// renamed out of the way, then supplies the cubic basis under the original
// names.  The cubic formulas are the ones of tools.hpp:110-134 (the uniform
// cubic B-spline and its derivative), evaluated in the same operation order so
// that the cubic reference build and the C restatement agree to the last bit.  apicDinverse
// (simulation.cpp:94-96) is set to 3/dx^2 by ref_harness.cpp.
#include <assert.h>

#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <Eigen/Core>
#include <Eigen/Dense>

#define N matter_ref_quadratic_N
#define dNdu matter_ref_quadratic_dNdu
#define d2Ndu2 matter_ref_quadratic_d2Ndu2
#define wip matter_ref_quadratic_wip
#define grad_wip matter_ref_quadratic_grad_wip
#define laplace_wip matter_ref_quadratic_laplace_wip
#include "tools.hpp"
#undef N
#undef dNdu
#undef d2Ndu2
#undef wip
#undef grad_wip
#undef laplace_wip

#define MATTER_REF_SPLINEDEG 3

inline T N(T u) {
  T a = std::abs(u);
  if (a < 1.0) return 0.5 * a * a * a - a * a + 2.0 / 3.0;
  if (a < 2.0) return (1.0 / 6.0) * (2.0 - a) * (2.0 - a) * (2.0 - a);
  return 0;
}
inline T dNdu(T u) {
  T a = std::abs(u);
  if (a < 1.0) return u * (1.5 * a - 2.0);
  if (a < 2.0) return -0.5 * sgn(u) * (2.0 - a) * (2.0 - a);
  return 0;
}
#ifdef THREEDIM
inline T wip(T xp, T yp, T zp, T xi, T yi, T zi, T h) {
  return N((xp - xi) * h) * N((yp - yi) * h) * N((zp - zi) * h);
}
inline TV grad_wip(T xp, T yp, T zp, T xi, T yi, T zi, T h) {
  TV g;
  g(0) = dNdu((xp - xi) * h) * N((yp - yi) * h) * N((zp - zi) * h) * h;
  g(1) = dNdu((yp - yi) * h) * N((xp - xi) * h) * N((zp - zi) * h) * h;
  g(2) = dNdu((zp - zi) * h) * N((xp - xi) * h) * N((yp - yi) * h) * h;
  return g;
}
#else
// the 2D forms (tools.hpp:247-258)
inline T wip(T xp, T yp, T xi, T yi, T h) { return N((xp - xi) * h) * N((yp - yi) * h); }
inline TV grad_wip(T xp, T yp, T xi, T yi, T h) {
  TV g;
  g(0) = dNdu((xp - xi) * h) * N((yp - yi) * h) * h;
  g(1) = dNdu((yp - yi) * h) * N((xp - xi) * h) * h;
  return g;
}
#endif

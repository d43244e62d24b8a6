/*
 * Forward-mode dual numbers for building the reference's stepping code as a
 * tangent-linear (directional-derivative) program.  Test infrastructure.
 *
 * qd carries a value and one tangent.  Every value operation is the same IEEE
 * double operation as in the plain build (no contraction on x86-64 -O2), so the
 * value part reproduces the reference bit-for-bit while the tangent part is the
 * exact derivative of the branch taken.  Conventions at non-smooth points match
 * the adjoint kernels: d|x| = sign(x) dx with sign(0) = 0, d sqrt(x) = 0 at x = 0,
 * comparisons, max/min and integer casts act on the value.
 *
 * Used two ways: qas_dual_define.h force-included into the reference sources
 * (after every system header they use) turns their `double` into qd; the dual
 * harness includes this header directly.
 */
#ifndef QAS_DUAL_H
#define QAS_DUAL_H

/* every system header the reference sources and the harness use, before `double` is redefined */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <omp.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

struct qd {
  double v, d;
  qd() = default;
  qd(double x) : v(x), d(0.0) {}
  qd(double x, double t) : v(x), d(t) {}
  explicit operator double() const { return v; }
  explicit operator float() const { return (float)v; }
  explicit operator int() const { return (int)v; }
  qd &operator+=(const qd &b) { d = d + b.d; v = v + b.v; return *this; }
  qd &operator-=(const qd &b) { d = d - b.d; v = v - b.v; return *this; }
  qd &operator*=(const qd &b) { d = d * b.v + v * b.d; v = v * b.v; return *this; }
  qd &operator/=(const qd &b) { const double q = v / b.v; d = (d - q * b.d) / b.v; v = q; return *this; }
};

inline qd operator+(const qd &a) { return a; }
inline qd operator-(const qd &a) { return qd(-a.v, -a.d); }
inline qd operator+(const qd &a, const qd &b) { return qd(a.v + b.v, a.d + b.d); }
inline qd operator-(const qd &a, const qd &b) { return qd(a.v - b.v, a.d - b.d); }
inline qd operator*(const qd &a, const qd &b) { return qd(a.v * b.v, a.d * b.v + a.v * b.d); }
inline qd operator/(const qd &a, const qd &b)
{
  const double q = a.v / b.v;
  return qd(q, (a.d - q * b.d) / b.v);
}
inline bool operator<(const qd &a, const qd &b) { return a.v < b.v; }
inline bool operator>(const qd &a, const qd &b) { return a.v > b.v; }
inline bool operator<=(const qd &a, const qd &b) { return a.v <= b.v; }
inline bool operator>=(const qd &a, const qd &b) { return a.v >= b.v; }
inline bool operator==(const qd &a, const qd &b) { return a.v == b.v; }
inline bool operator!=(const qd &a, const qd &b) { return a.v != b.v; }

inline qd sqrt(const qd &a)
{
  const double s = ::sqrt(a.v);
  return qd(s, a.v > 0.0 ? 0.5 * a.d / s : 0.0);
}
inline qd fabs(const qd &a)
{
  if (a.v > 0.0) return a;
  if (a.v < 0.0) return -a;
  return qd(::fabs(a.v), 0.0);
}
/* the reference's max/min templates (common/common_func.h:4-14) for mixed qd/double arguments */
inline qd max(qd a, qd b) { return (a >= b) ? a : b; }
inline qd min(qd a, qd b) { return (a >= b) ? b : a; }

#endif

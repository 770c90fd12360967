// Sign predicates with escalating precision: a binary32 stage with a proved
// error bound, a binary64 stage with a proved error bound, and an exact stage
// in floating-point expansion arithmetic (Shewchuk 1997, "Adaptive Precision
// Floating-Point Arithmetic and Fast Robust Geometric Predicates": two-sum,
// two-product and expansion growth, restated here from the paper).  Each
// predicate returns the exact sign of its quantity for binary64 inputs and
// reports the stage that decided it, so callers can count escalations.
//
// Assumptions: inputs finite and, for the exact stage, products neither
// overflowing nor underflowing binary64 (coordinates of this project's
// normalised windows and planes lie far inside that range).  The binary32
// stage guards its own range and steps aside outside it.
//
// Header-only, for device and host code alike (the host build lets the CPU
// tests compare every sign with rational arithmetic).
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define EDP_HD __host__ __device__
#define EDP_COLD __noinline__
#else
#define EDP_HD
#define EDP_COLD __attribute__((noinline))
#endif

namespace edp {
namespace pred {

enum Stage : int { kBinary32 = 0, kBinary64 = 1, kExact = 2 };

constexpr double kU64 = 1.0 / 9007199254740992.0;  // 2^-53, unit roundoff of binary64
constexpr float kU32 = 1.0f / 16777216.0f;         // 2^-24, unit roundoff of binary32

EDP_HD inline int sign_of(double x) { return (x > 0.0) - (x < 0.0); }

// ---------------------------------------------------------------- expansions

// a + b = x + y exactly, x = fl(a + b) (Knuth's two-sum: no ordering needed).
EDP_HD inline void two_sum(double a, double b, double &x, double &y) {
  x = a + b;
  const double bv = x - a;
  const double av = x - bv;
  y = (a - av) + (b - bv);
}

// a * b = x + y exactly, x = fl(a * b): the product's rounding error is what
// a fused multiply-add of a, b and -x returns, exactly.
EDP_HD inline void two_product(double a, double b, double &x, double &y) {
  x = a * b;
  y = fma(a, b, -x);
}

// Adds b to the nonoverlapping expansion e[0..n) (increasing magnitude) in
// place, giving n + 1 components: e[0..n] (Shewchuk's Grow-Expansion).
EDP_HD inline void grow(double *e, int n, double b) {
  double q = b;
  for (int i = 0; i < n; ++i) {
    double s, t;
    two_sum(q, e[i], s, t);
    e[i] = t;
    q = s;
  }
  e[n] = q;
}

// Sign of a nonoverlapping expansion: the sign of its largest nonzero part.
EDP_HD inline int expansion_sign(const double *e, int n) {
  for (int i = n - 1; i >= 0; --i)
    if (e[i] != 0.0) return sign_of(e[i]);
  return 0;
}

// ---------------------------------------------------------------- orient2d

// Exact stage of orient2d: the determinant is ax by - ay bx + bx cy - by cx +
// cx ay - cy ax; each product is exactly a two-component expansion, and
// growing one expansion by all twelve components keeps the sum exact.  Out
// of line: it is rare, and its expansion would otherwise take registers
// from every caller.
EDP_HD inline EDP_COLD int orient2d_exact(double ax, double ay, double bx, double by, double cx,
                                   double cy) {
  double e[12];
  int n = 0;
  const double xs[6] = {ax, -ay, bx, -by, cx, -cy};
  const double ys[6] = {by, bx, cy, cx, ay, ax};
  for (int k = 0; k < 6; ++k) {
    double x, y;
    two_product(xs[k], ys[k], x, y);
    grow(e, n, y);
    ++n;
    grow(e, n, x);
    ++n;
  }
  return expansion_sign(e, n);
}

// Sign of the doubled signed area of (a, b, c): of
// (bx - ax)(cy - ay) - (by - ay)(cx - ax), positive when c lies left of a->b.
// With first32 false the binary32 stage is skipped (the binary64 filter
// decides first); the sign is the same.
EDP_HD inline int orient2d(double ax, double ay, double bx, double by, double cx, double cy,
                           int *stage = nullptr, bool first32 = true) {
  // Binary32 stage: differences in binary64 (relative error <= 2^-53), then
  // converted, multiplied and subtracted in binary32.  For exact products
  // p1, p2 with S = |p1| + |p2|, each rounded product carries a relative
  // error <= 3.01 u and the subtraction u more, so the computed difference
  // is within 4.02 u S of the true one, and S <= s32 (1 + 4.1 u): |det32|
  // above 4.1 u s32 (taken as 5 u s32, the bound's own rounding included)
  // fixes the sign.  Differences outside [2^-60, 2^60] (zero excepted) could
  // underflow or overflow binary32 products, so they skip this stage.
  const double dx1 = bx - ax, dy1 = by - ay, dx2 = cx - ax, dy2 = cy - ay;
  const double lo = 8.673617379884035e-19, hi = 1.152921504606847e18;  // 2^-60, 2^60
  auto in_range = [&](double v) {
    const double m = fabs(v);
    return m == 0.0 || (m >= lo && m <= hi);
  };
  if (first32 && in_range(dx1) && in_range(dy1) && in_range(dx2) && in_range(dy2)) {
    const float f1 = float(dx1) * float(dy2);
    const float f2 = float(dy1) * float(dx2);
    const float det32 = f1 - f2;
    const float bound32 = (fabsf(f1) + fabsf(f2)) * (5.0f * kU32);
    if (det32 > bound32 || -det32 > bound32) {
      if (stage) *stage = kBinary32;
      return det32 > 0.0f ? 1 : -1;
    }
  }
  // Binary64 stage (Shewchuk's orient2d first filter): with a, b taken
  // relative to c, the computed determinant is within (3 + 16 e) e S of
  // the exact one, e = 2^-53, S = |detleft| + |detright|.
  const double detleft = (ax - cx) * (by - cy);
  const double detright = (ay - cy) * (bx - cx);
  const double det = detleft - detright;
  double detsum;
  if (detleft > 0.0) {
    if (detright <= 0.0) {
      if (stage) *stage = kBinary64;
      return sign_of(det);
    }
    detsum = detleft + detright;
  } else if (detleft < 0.0) {
    if (detright >= 0.0) {
      if (stage) *stage = kBinary64;
      return sign_of(det);
    }
    detsum = -detleft - detright;
  } else {
    if (stage) *stage = kBinary64;
    return sign_of(det);
  }
  const double bound64 = (3.0 + 16.0 * kU64) * kU64 * detsum;
  if (det >= bound64 || -det >= bound64) {
    if (stage) *stage = kBinary64;
    return sign_of(det);
  }
  if (stage) *stage = kExact;
  return orient2d_exact(ax, ay, bx, by, cx, cy);
}

// orient2d without the binary32 stage and without sign-case branches:
// Shewchuk's first binary64 filter as one bound test, then the exact stage.
// Same sign as orient2d (inputs whose products underflow excepted, as for
// Shewchuk's filter).
// Result of a filter-only predicate that its filter cannot decide: the
// caller defers the whole decision to a pass with the exact stage.
constexpr int kUndecided = 2;

// orient2d_lean's binary64 filter alone: the sign, or kUndecided.
EDP_HD inline int orient2d_filter(double ax, double ay, double bx, double by, double cx,
                                  double cy, int *stage = nullptr) {
  const double detleft = (ax - cx) * (by - cy);
  const double detright = (ay - cy) * (bx - cx);
  const double det = detleft - detright;
  const double bound = (3.0 + 16.0 * kU64) * kU64 * (fabs(detleft) + fabs(detright));
  if (det > bound || -det > bound || bound == 0.0) {
    if (stage) *stage = kBinary64;
    return sign_of(det);
  }
  if (stage) *stage = kExact;
  return kUndecided;
}

EDP_HD inline int orient2d_lean(double ax, double ay, double bx, double by, double cx,
                                double cy, int *stage = nullptr) {
  const int s = orient2d_filter(ax, ay, bx, by, cx, cy, stage);
  return s != kUndecided ? s : orient2d_exact(ax, ay, bx, by, cx, cy);
}

// ---------------------------------------------------------------- linear forms

// Exact stage of dot_sign: every product as a two-component expansion, all
// grown into one (out of line, as orient2d_exact).
EDP_HD inline EDP_COLD int dot_sign_exact(const double *p, const double *q, int n) {
  double e[16];
  int m = 0;
  for (int k = 0; k < n; ++k) {
    double x, y;
    two_product(p[k], q[k], x, y);
    grow(e, m, y);
    ++m;
    grow(e, m, x);
    ++m;
  }
  return expansion_sign(e, m);
}

// dot_sign's binary64 stage alone: the bound of its binary32 stage with
// binary64's unit roundoff, (n + 2) u S, taken with a margin as
// 2 (n + 2) u s64.  The sign, or kUndecided.
EDP_HD inline int dot_sign_filter(const double *p, const double *q, int n, int *stage = nullptr) {
  double s64 = 0.0, a64 = 0.0;
  for (int k = 0; k < n; ++k) {
    const double t = p[k] * q[k];
    s64 += t;
    a64 += fabs(t);
  }
  const double bound64 = a64 * (2.0 * double(n + 2) * kU64);
  if (s64 > bound64 || -s64 > bound64) {
    if (stage) *stage = kBinary64;
    return sign_of(s64);
  }
  if (stage) *stage = kExact;
  return kUndecided;
}

// Sign of sum_k p[k] q[k] for n <= 8 terms (a plane evaluated at a point, or
// the difference of two planes there: the depth order of two sources).
EDP_HD inline int dot_sign(const double *p, const double *q, int n, int *stage = nullptr,
                           bool first32 = true) {
  // Binary32 stage: inputs rounded (relative error <= u each), products
  // (u) and a sequential sum of n terms (the classical bound (n - 1) u on
  // the absolute values): the computed sum is within (n + 2) u S (1 + O(u))
  // of the exact one, S = sum |p q|, and S <= s32 (1 + (n + 3) u).  The
  // stage decides when |sum32| exceeds 2 (n + 3) u s32.  Inputs outside
  // [2^-60, 2^60] (zero excepted) skip it.
  const double lo = 8.673617379884035e-19, hi = 1.152921504606847e18;
  bool ok = first32;
  for (int k = 0; k < n && ok; ++k) {
    const double a = fabs(p[k]), b = fabs(q[k]);
    ok = (a == 0.0 || (a >= lo && a <= hi)) && (b == 0.0 || (b >= lo && b <= hi));
  }
  if (ok) {
    float s32 = 0.0f, a32 = 0.0f;
    for (int k = 0; k < n; ++k) {
      const float t = float(p[k]) * float(q[k]);
      s32 += t;
      a32 += fabsf(t);
    }
    const float bound32 = a32 * (2.0f * float(n + 3) * kU32);
    if (s32 > bound32 || -s32 > bound32) {
      if (stage) *stage = kBinary32;
      return s32 > 0.0f ? 1 : -1;
    }
  }
  const int s = dot_sign_filter(p, q, n, stage);
  return s != kUndecided ? s : dot_sign_exact(p, q, n);
}

}  // namespace pred
}  // namespace edp

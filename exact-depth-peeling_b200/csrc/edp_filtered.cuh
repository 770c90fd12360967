// The kernels' sign predicates in two forms, chosen per workspace by
// Dev::predicates:
//   0  plain binary64: the sign of the rounded expression, as the reference's
//      Warp kernels compute it;
//   1  filtered: the exact sign of the expression's real value for the
//      binary64 inputs, decided in binary32 when a static forward error bound
//      certifies it, else in binary64 under Shewchuk's bound, else exactly in
//      expansion arithmetic (edp_predicates.cuh);
//   2  filtered and counted: as 1, and every call is tallied by predicate
//      class and deciding stage into Dev::pred_counts;
//   3  filtered from binary64: the same exact signs with the binary32 stage
//      skipped (orientation through orient2d_lean, the binary64 filter as one
//      bound test, then expansion arithmetic);
//   4  the binary64 filters of form 3 alone, for kernels whose undecided
//      cases go to a second pass in form 3 (pred::kUndecided marks them).
//      Where form 4 decides, it gives form 3's sign.
// Constructions (intersection points, clip parameters, depths stored for the
// hit sort's radix fallback) stay binary64 in every form.
#pragma once
#include "edp_internal.h"
#include "edp_predicates.cuh"

namespace edp {

// Predicate classes (rows of Dev::pred_counts, three stages each).
enum PredClass : int {
  kPredSide = 0,     // patch vertex against a contour segment's line (subdivision)
  kPredSegment = 1,  // contour segment end against a patch edge (subdivision)
  kPredDepth = 2,    // patch plane against a segment end's near plane (subdivision)
  kPredContain = 3,  // sample point against a source edge (ray hits)
  kPredOrder = 4,    // depth order of two sources at a sample (hit order, ranks)
  kPredClip = 5,     // piece against occluder edges and depth (iterative clipping)
  kPredClasses = 6
};
static_assert(3 * kPredClasses == kPredCounters, "one counter per class and stage");

// One thread's tally of one class: calls decided in binary32, in binary64,
// and exactly.
struct Tally {
  unsigned s32 = 0, s64 = 0, sx = 0;
  __device__ void add(int stage) {
    s32 += stage == pred::kBinary32;
    s64 += stage == pred::kBinary64;
    sx += stage == pred::kExact;
  }
  // Adds the tallies of the calling warp's active lanes to class `cls`, one
  // atomic per counter and warp.
  __device__ void flush(const Dev &d, int cls) const {
    const unsigned mask = __activemask();
    const unsigned a = __reduce_add_sync(mask, s32);
    const unsigned b = __reduce_add_sync(mask, s64);
    const unsigned c = __reduce_add_sync(mask, sx);
    if (int(threadIdx.x & 31) == __ffs(int(mask)) - 1) {
      unsigned long long *row = d.pred_counts + 3 * cls;
      if (a) atomicAdd(&row[0], (unsigned long long)a);
      if (b) atomicAdd(&row[1], (unsigned long long)b);
      if (c) atomicAdd(&row[2], (unsigned long long)c);
    }
  }
};

// The kernels that evaluate these predicates are templates on the form F
// (the value of Dev::predicates), so the plain form compiles to the
// reference's expressions alone and the filtered forms carry no test of the
// mode.  The filtered forms report the deciding stage in `stage`; the
// caller tallies it when F == 2.

__device__ inline int sign_of(double v) { return (v > 0.0) - (v < 0.0); }

// Side of c against the line a->b: +1 left, -1 right, 0 on it.  In the
// filtered forms a point equal to an end of the line is on it without
// arithmetic (the filters cannot certify a zero; shared mesh vertices make
// this case common); it is counted with the binary64 stage.
template <int F>
__device__ inline int side_sign(V2 a, V2 b, V2 c, int &stage) {
  if constexpr (F != 0) {
    if ((c.x == a.x && c.y == a.y) || (c.x == b.x && c.y == b.y)) {
      stage = pred::kBinary64;
      return 0;
    }
  }
  if constexpr (F == 0) {
    return sign_of(cross(a, b, c));
  } else if constexpr (F == 3) {
    return pred::orient2d_lean(a.x, a.y, b.x, b.y, c.x, c.y, &stage);
  } else if constexpr (F == 4) {
    return pred::orient2d_filter(a.x, a.y, b.x, b.y, c.x, c.y, &stage);
  } else {
    return pred::orient2d(a.x, a.y, b.x, b.y, c.x, c.y, &stage);
  }
}

// Sign of s1(x) - s2(x): positive when source 1 lies behind source 2 at x.
// z1, z2 are the binary64 depths value(s1, x), value(s2, x), which the plain
// form compares.  Two identical planes are equal without arithmetic (counted
// as decided in the first stage).
template <int F>
__device__ inline int order_sign(const Plane &s1, double z1, const Plane &s2, double z2, V2 x,
                                 int &stage) {
  if constexpr (F == 0) {
    return sign_of(z1 - z2);
  } else {
    if (s1.a == s2.a && s1.b == s2.b && s1.c == s2.c) {  // one plane: equal everywhere
      stage = pred::kBinary32;
      return 0;
    }
    const double p[6] = {s1.a, s1.b, s1.c, s2.a, s2.b, s2.c};
    const double q[6] = {x.x, x.y, 1.0, -x.x, -x.y, -1.0};
    if constexpr (F == 4)
      return pred::dot_sign_filter(p, q, 6, &stage);
    else
      return pred::dot_sign(p, q, 6, &stage, F != 3);
  }
}

// u / (u - v), the parameter where a linear function with values u and v at
// the ends of a segment vanishes, clamped to [0, 1]; 0.5 when u == v (the
// filtered forms can see opposite exact signs where binary64 rounds both
// values alike).
__device__ inline double crossing(double u, double v) {
  const double den = u - v;
  if (den == 0.0) return 0.5;
  return fmin(1.0, fmax(0.0, u / den));
}

// Launches kernel template K<F> for the workspace's form.
#define EDP_LAUNCH_FORM(form, kernel, grid, block, stream, ...)          \
  do {                                                                   \
    switch (form) {                                                      \
      case 0: kernel<0><<<grid, block, 0, stream>>>(__VA_ARGS__); break; \
      case 1: kernel<1><<<grid, block, 0, stream>>>(__VA_ARGS__); break; \
      case 2: kernel<2><<<grid, block, 0, stream>>>(__VA_ARGS__); break; \
      default: kernel<3><<<grid, block, 0, stream>>>(__VA_ARGS__); break; \
    }                                                                    \
  } while (0)

}  // namespace edp

// Host build of the escalating sign predicates (exact-depth-peeling_b200/
// csrc/edp_predicates.cuh) for the CPU tests: batch entry points that return
// each sign and the stage that decided it.
#include "../../exact-depth-peeling_b200/csrc/edp_predicates.cuh"

extern "C" void orient2d_batch(const double *points, long count, int *signs, int *stages) {
  for (long i = 0; i < count; ++i) {
    const double *p = points + 6 * i;
    signs[i] = edp::pred::orient2d(p[0], p[1], p[2], p[3], p[4], p[5], &stages[i]);
  }
}

extern "C" void dot_sign_batch(const double *p, const double *q, int terms, long count,
                               int *signs, int *stages) {
  for (long i = 0; i < count; ++i)
    signs[i] = edp::pred::dot_sign(p + terms * i, q + terms * i, terms, &stages[i]);
}

extern "C" void orient2d_lean_batch(const double *points, long count, int *signs, int *stages) {
  for (long i = 0; i < count; ++i) {
    const double *p = points + 6 * i;
    signs[i] = edp::pred::orient2d_lean(p[0], p[1], p[2], p[3], p[4], p[5], &stages[i]);
  }
}

// The filter-only stages of the two-pass form: a sign, or kUndecided (2).
extern "C" void orient2d_filter_batch(const double *points, long count, int *signs) {
  for (long i = 0; i < count; ++i) {
    const double *p = points + 6 * i;
    signs[i] = edp::pred::orient2d_filter(p[0], p[1], p[2], p[3], p[4], p[5]);
  }
}

extern "C" void dot_sign_filter_batch(const double *p, const double *q, int terms, long count,
                                      int *signs) {
  for (long i = 0; i < count; ++i)
    signs[i] = edp::pred::dot_sign_filter(p + terms * i, q + terms * i, terms);
}

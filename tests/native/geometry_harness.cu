// Host build of the kernels' polygon helpers (exact-depth-peeling_b200/csrc/
// edp_device.cuh: clean, split_edge, separated) for the CPU tests.  Points
// are passed as interleaved x, y doubles.
#include "../../exact-depth-peeling_b200/csrc/edp_device.cuh"

using edp::V2;

extern "C" int geometry_clean(double *xy, int n) {
  return edp::clean(reinterpret_cast<V2 *>(xy), n);
}

extern "C" void geometry_split_edge(const double *xy, int n, const double *ab, double *in,
                                    int *ni, double *out, int *no) {
  edp::split_edge(reinterpret_cast<const V2 *>(xy), n, V2{ab[0], ab[1]}, V2{ab[2], ab[3]},
                  reinterpret_cast<V2 *>(in), *ni, reinterpret_cast<V2 *>(out), *no);
}

extern "C" int geometry_separated(const double *a, int na, const double *b, int nb) {
  return edp::separated(reinterpret_cast<const V2 *>(a), na, reinterpret_cast<const V2 *>(b),
                        nb);
}

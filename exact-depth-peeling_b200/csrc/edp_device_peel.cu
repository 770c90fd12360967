// DevicePeeler: iterative per-layer clipping (warp_peel/solver.py:92-519).
#include "../../include/edp.h"
#include "edp_internal.h"

extern "C" int edp_device_create(const double *, int64_t, const int32_t *, int64_t,
                                 const double *, const double *, const edp_device_capacities *,
                                 int32_t, void *, edp_peeler **out) {
  if (out) *out = nullptr;
  return EDP_ERR_STATE;
}

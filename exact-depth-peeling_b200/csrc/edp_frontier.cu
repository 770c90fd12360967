// Contour-guided convex subdivision: one round of the device-controlled loop
// (warp_peel/frontier.py:81-245, event_kernels.py:12-25).
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kBlock = 128;

// Does the part of segment a->b inside the convex patch lie strictly in front
// of it somewhere?  za, zb are patch depth minus segment depth at the ends
// (positive: segment nearer).  Clips the parameter range by each patch edge
// half-plane and by the depth half-plane (frontier.py:81-103).
__device__ inline bool front_segment(const V2 *p, int n, V2 a, V2 b, double za, double zb) {
  double low = 0.0, high = 1.0;
  for (int j = 0; j <= n; ++j) {
    double da = za, db = zb;
    if (j < n) {
      V2 u = p[j], v = p[(j + 1) % n];
      da = cross(u, v, a);
      db = cross(u, v, b);
    }
    if (da <= 0.0 && db <= 0.0) return false;
    if (da < 0.0) low = fmax(low, da / (da - db));
    if (db < 0.0) high = fmin(high, da / (da - db));
  }
  return high > low;
}

// One frontier round.  Each patch visits at most kCandidatesPerPass contour
// segments of the segment hierarchy, continuing from its cursor.  The first
// segment that crosses the patch interior and is nearer somewhere splits the
// patch along its supporting line into two next-round patches that inherit the
// cursor; a patch whose traversal completes is final and goes to the output
// pool; otherwise it carries over (frontier.py:106-223).  Slots are reserved
// once per converged group of threads and counters are flushed once per thread.
__global__ void __launch_bounds__(kBlock) k_subdivide(Dev d) {
  enum Action { kSkip = 0, kSplit = 1, kCarry = 2, kDone = 3 };
  const int par = *d.parity;
  const V2 *fv = d.fv[par];
  const int *fn = d.fn[par], *fsrc = d.fsrc[par], *fcur = d.fcur[par];
  V2 *nv = d.fv[par ^ 1];
  int *nn = d.fn[par ^ 1], *nsrc = d.fsrc[par ^ 1], *ncur = d.fcur[par ^ 1];
  const int live = int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  const int leaves = *d.seg_tree.size;
  long long visits = 0, tests = 0, splits = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < live;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (d.status[kError] != 0) return;
    const int n = fn[i];
    if (n == 0) continue;
    ++visits;
    const int source = fsrc[i];
    int node = fcur[i];
    const V2 *p = fv + int64_t(kMaxVertices) * i;
    const Plane sc = d.scores[source];
    float4 lo, hi;
    polygon_bounds(p, n, sc, lo, hi);
    lo.z = -1.0e30f;
    int action = kCarry;
    V2 a = v2(0.0, 0.0), b = a;
    for (int task = 0; task < kCandidatesPerPass; ++task) {
      int c;
      node = query_next(d.seg_tree, leaves, lo, hi, node, 0, c);
      if (c < 0) {
        action = kDone;
        break;
      }
      ++tests;
      a = d.seg_a[c];
      b = d.seg_b[c];
      bool positive = false, negative = false;
      for (int j = 0; j < n; ++j) {
        double side = cross(a, b, p[j]);
        positive |= side > 0.0;
        negative |= side < 0.0;
      }
      if (!(positive && negative)) continue;
      const V2 near = d.seg_near[c];
      double za = value(sc, a) - near.x, zb = value(sc, b) - near.y;
      if (front_segment(p, n, a, b, za, zb)) {
        action = kSplit;
        break;
      }
    }
    const int slot = reserve(&d.status[kNextResidual],
                             action == kSplit ? 2 : action == kCarry ? 1 : 0);
    const int out = reserve(&d.status[kPolygons], action == kDone ? 1 : 0);
    if (action == kDone) {
      if (out >= d.cap.regions) {
        set_error(d.status, kErrOutput);
        continue;
      }
      V2 *dst = d.out_v + int64_t(kMaxVertices) * out;
      for (int j = 0; j < n; ++j) dst[j] = p[j];
      d.out_n[out] = n;
      d.out_src[out] = source;
      d.out_layer[out] = 0;
      continue;
    }
    if (action == kCarry) {
      if (slot >= d.cap.frontier) {
        set_error(d.status, kErrResidual);
        continue;
      }
      V2 *dst = nv + int64_t(kMaxVertices) * slot;
      for (int j = 0; j < n; ++j) dst[j] = p[j];
      nn[slot] = n;
      nsrc[slot] = source;
      ncur[slot] = node;
      continue;
    }
    if (int64_t(slot) + 1 >= d.cap.frontier) {
      set_error(d.status, kErrResidual);
      continue;
    }
    V2 *left_v = nv + int64_t(kMaxVertices) * slot;
    V2 *right_v = left_v + kMaxVertices;
    int left = 0, right = 0;
    V2 dir = b - a;
    Plane s{-dir.y, dir.x, 0.0, 0.0};
    for (int j = 0; j < n; ++j) {
      V2 u = p[j], v = p[(j + 1) % n];
      double du = value(s, u - a), dv = value(s, v - a);
      if (du >= 0.0) left = append(left_v, left, u);
      if (du <= 0.0) right = append(right_v, right, u);
      if ((du > 0.0 && dv < 0.0) || (du < 0.0 && dv > 0.0)) {
        V2 x = u + (du / (du - dv)) * (v - u);
        left = append(left_v, left, x);
        right = append(right_v, right, x);
      }
    }
    left = clean(left_v, left);
    right = clean(right_v, right);
    if (left > kMaxVertices || right > kMaxVertices) {
      set_error(d.status, kErrPolygon);
      continue;
    }
    if (left > 0 && right > 0) {
      ++splits;
    } else {
      // A collapsed child cancels this cut; the parent continues next round.
      left = n;
      right = 0;
      for (int j = 0; j < n; ++j) left_v[j] = p[j];
    }
    nn[slot] = left;
    nn[slot + 1] = right;
    nsrc[slot] = source;
    nsrc[slot + 1] = source;
    ncur[slot] = node;
    ncur[slot + 1] = node;
  }
  count_add(&d.metrics[kTargetVisits], visits);
  count_add(&d.metrics[kContourTests], tests);
  count_add(&d.metrics[kSplits], splits);
}

// Swap frontiers and decide whether another round runs (event_kernels.py:12-25).
__global__ void k_advance(Dev d) {
  int next = d.status[kNextResidual];
  d.status[kResidual] = next;
  d.status[kNextResidual] = 0;
  long long rounds = ++d.metrics[kRounds];
  if (rounds >= d.cap.rounds && next > 0) set_error(d.status, kErrRounds);
  d.status[kPeakResidual] = max(d.status[kPeakResidual], next);
  *d.parity ^= 1;
  int c = next > 0 && d.status[kError] == 0;
  *d.condition = c;
  if (d.use_handle) cudaGraphSetConditional(d.cond_handle, unsigned(c));
}

}  // namespace

cudaError_t stage_step(const Dev &d, cudaStream_t st) {
  int64_t g = ceil_div(d.cap.frontier, kBlock);
  if (g > 148 * 32) g = 148 * 32;
  k_subdivide<<<unsigned(g), kBlock, 0, st>>>(d);
  note_launch();
  k_advance<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

}  // namespace edp

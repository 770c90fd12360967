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

// Resident threads of a B200 (148 SMs x 2048): while fewer patches than this
// remain, each may test proportionally more candidates per round.
constexpr int kResidentThreads = 148 * 2048;
constexpr int kMaxBudget = 4096;

__device__ inline void push(const Dev &d, V2 *nv, int *nn, int *nsrc, int *ncur, const V2 *p,
                            int n, int source, int node) {
  const int slot = reserve(&d.status[kNextResidual], 1);
  if (slot >= d.cap.frontier) {
    set_error(d.status, kErrResidual);
    return;
  }
  V2 *dst = nv + int64_t(kMaxVertices) * slot;
  for (int j = 0; j < n; ++j) dst[j] = p[j];
  nn[slot] = n;
  nsrc[slot] = source;
  ncur[slot] = node;
}

// One frontier round (frontier.py:106-223).  A patch walks the contour-segment
// hierarchy from its cursor.  The first segment that crosses the patch
// interior and is nearer somewhere splits it along the segment's supporting
// line; a patch whose walk completes is final and goes to the output pool.
// Differences from the reference's schedule, which leave every patch's fate
// unchanged: after a split the thread continues at once with the left child
// (from the same cursor) and only the right child waits for the next round;
// and the per-round candidate budget grows as the frontier shrinks (32 per
// patch when the GPU is full, up to kMaxBudget), so long contour walks need
// far fewer rounds.
__global__ void __launch_bounds__(kBlock) k_subdivide(Dev d) {
  const int par = *d.parity;
  const V2 *fv = d.fv[par];
  const int *fn = d.fn[par], *fsrc = d.fsrc[par], *fcur = d.fcur[par];
  V2 *nv = d.fv[par ^ 1];
  int *nn = d.fn[par ^ 1], *nsrc = d.fsrc[par ^ 1], *ncur = d.fcur[par ^ 1];
  const int live = int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  const int leaves = *d.seg_tree.size;
  const int budget = live >= kResidentThreads / kCandidatesPerPass
                         ? kCandidatesPerPass
                         : int(min(int64_t(kMaxBudget),
                                   int64_t(kResidentThreads) / max(live, 1)));
  long long visits = 0, tests = 0, splits = 0;
  V2 cur[kMaxVertices], left_v[kMaxVertices], right_v[kMaxVertices];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < live;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (d.status[kError] != 0) return;
    int n = fn[i];
    if (n == 0) continue;
    ++visits;
    const int source = fsrc[i];
    int node = fcur[i];
    {
      const V2 *p = fv + int64_t(kMaxVertices) * i;
      for (int j = 0; j < n; ++j) cur[j] = p[j];
    }
    const Plane sc = d.scores[source];
    int left_budget = budget;
    while (true) {
      float4 lo, hi;
      polygon_bounds(cur, n, sc, lo, hi);
      lo.z = -1.0e30f;
      bool done = false, split = false;
      V2 a = v2(0.0, 0.0), b = a;
      while (left_budget > 0) {
        int c;
        node = query_next(d.seg_tree, leaves, lo, hi, node, 0, c);
        if (c < 0) {
          done = true;
          break;
        }
        --left_budget;
        ++tests;
        a = d.seg_a[c];
        b = d.seg_b[c];
        bool positive = false, negative = false;
        for (int j = 0; j < n; ++j) {
          double side = cross(a, b, cur[j]);
          positive |= side > 0.0;
          negative |= side < 0.0;
        }
        if (!(positive && negative)) continue;
        const V2 near = d.seg_near[c];
        double za = value(sc, a) - near.x, zb = value(sc, b) - near.y;
        if (front_segment(cur, n, a, b, za, zb)) {
          split = true;
          break;
        }
      }
      if (done) {
        const int out = reserve(&d.status[kPolygons], 1);
        if (out >= d.cap.regions) {
          set_error(d.status, kErrOutput);
          break;
        }
        V2 *dst = d.out_v + int64_t(kMaxVertices) * out;
        for (int j = 0; j < n; ++j) dst[j] = cur[j];
        d.out_n[out] = n;
        d.out_src[out] = source;
        d.out_layer[out] = 0;
        break;
      }
      if (!split) {  // budget spent: carry the patch and its cursor over
        push(d, nv, nn, nsrc, ncur, cur, n, source, node);
        break;
      }
      int left = 0, right = 0;
      const V2 dir = b - a;
      const Plane s{-dir.y, dir.x, 0.0, 0.0};
      for (int j = 0; j < n; ++j) {
        V2 u = cur[j], v = cur[(j + 1) % n];
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
        break;
      }
      if (left > 0 && right > 0) {
        ++splits;
        push(d, nv, nn, nsrc, ncur, right_v, right, source, node);
        for (int j = 0; j < left; ++j) cur[j] = left_v[j];
        n = left;
      }
      // A collapsed child cancels the cut; the parent continues past it.
    }
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

// Contour-guided convex subdivision: one round of the device-controlled loop
// (warp_peel/frontier.py:81-245, event_kernels.py:12-25).
#include "edp_filtered.cuh"
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kBlock = 128;

constexpr int kWarps = kBlock / 32;
constexpr unsigned kFull = 0xffffffffu;
// Dev::step_budget: group tests one patch may spend per round before it
// carries over.  The budget decides only how the work is spread over rounds,
// never which cut a patch takes: every patch meets its candidates in leaf
// order in any case.

// The smallest power of two holding n lanes: a butterfly over it reduces
// lanes [0, n), the lanes that hold a patch's vertices.
__device__ inline int lane_width(int n) { return n <= 1 ? 1 : 1 << (32 - __clz(n - 1)); }

__device__ inline V2 shfl(V2 x, int lane) {
  return v2(__shfl_sync(kFull, x.x, lane), __shfl_sync(kFull, x.y, lane));
}

// polygon_bounds() of the patch held one vertex per lane (min and max are
// exact, so the butterfly order does not matter).  The plane comes and the
// box goes by value, which keeps this out-of-line helper's call frame small.
__device__ __noinline__ Box warp_bounds(V2 p, int n, Plane score) {
  const bool mine = int(threadIdx.x & 31) < n;
  const double z = value(score, p);
  double lx = mine ? p.x : 1.0e30, ly = mine ? p.y : 1.0e30, lz = mine ? z : 1.0e30;
  double hx = mine ? p.x : -1.0e30, hy = mine ? p.y : -1.0e30, hz = mine ? z : -1.0e30;
  // Lanes [0, width) hold every vertex; a butterfly over them leaves the
  // result in lane 0, which every lane then reads.
  const int width = lane_width(n);
  for (int off = width >> 1; off > 0; off >>= 1) {
    lx = fmin(lx, __shfl_xor_sync(kFull, lx, off));
    ly = fmin(ly, __shfl_xor_sync(kFull, ly, off));
    lz = fmin(lz, __shfl_xor_sync(kFull, lz, off));
    hx = fmax(hx, __shfl_xor_sync(kFull, hx, off));
    hy = fmax(hy, __shfl_xor_sync(kFull, hy, off));
    hz = fmax(hz, __shfl_xor_sync(kFull, hz, off));
  }
  lx = __shfl_sync(kFull, lx, 0);
  ly = __shfl_sync(kFull, ly, 0);
  lz = __shfl_sync(kFull, lz, 0);
  hx = __shfl_sync(kFull, hx, 0);
  hy = __shfl_sync(kFull, hy, 0);
  hz = __shfl_sync(kFull, hz, 0);
  double pz = 2.0e-7 * fmax(1.0, fmax(fabs(lz), fabs(hz)));
  return Box{make_float4(float(lx - 2.0e-7), float(ly - 2.0e-7), float(lz - pz), 0.f),
             make_float4(float(hx + 2.0e-7), float(hy + 2.0e-7), float(hz + pz), 0.f)};
}

// Does segment a->b cut the patch?  Its line has patch vertices strictly on
// both sides, and the part of the segment inside the patch lies strictly in
// front of it somewhere: the segment's parameter range clipped by each patch
// edge and by the depth half-plane stays open (frontier.py:81-103).  za, zb
// are patch depth minus segment depth at the ends (positive: segment nearer).
//
// The warp takes a batch's candidates one by one in leaf order with a lane per
// patch edge (p -> q): ballots decide the sides and the closed edges, and warp
// maxima / minima give the clip range, which is a max / min of the same
// quotients as the sequential clip and so is order-free.  Each lane first
// loads one candidate of the batch, so the loop itself reads no memory.

// The contour segments: hierarchy leaf ids, end points and depth at the ends.
struct Segments {
  const int *ids;
  const V2 *a, *b, *near;
  const int2 *near_src;  // the sources whose planes give `near`
  const V2 *near_mag;    // their |a x| + |b y| + |c| at the ends
  const Plane *scores;
  const int2 *vid;       // the welded mesh vertex at each end, or -1
  const int *faces, *canonical, *clipped, *src_n;
};

// Source `s` is an unclipped triangle with welded vertex `v`.
__device__ inline bool has_vertex(const Segments &g, int s, int v) {
  if (v < 0 || g.clipped[s] || g.src_n[s] != 3) return false;
  const int *f = g.faces + 3 * int64_t(s);
  return g.canonical[f[0]] == v || g.canonical[f[1]] == v || g.canonical[f[2]] == v;
}

// Predicate tallies of one subdivision warp (counted form only).
struct CutTally {
  Tally side, segment, depth;
};

// First cutting lane of a batch, or -1; a, b are its segment and `side` this
// lane's vertex against its line (the split reuses it).  F is the predicate
// form (edp_filtered.cuh): the plain form evaluates the reference's binary64
// expressions; the filtered forms take exact signs of the sides, of the
// segment ends against the patch edges and of the depth differences, and
// keep binary64 for the clip parameters.  The filter-only form returns
// kDeferAt - k when its filters cannot decide candidate k (no candidate
// before k cuts): the patch is then finished by the exact pass from k on.
constexpr int kDeferAt = -2;

template <int F>
__device__ inline int first_cut(Segments g, unsigned batch, int first, V2 p, V2 q, int n,
                                const Plane &sc, int source, V2 &a, V2 &b, int &side,
                                CutTally &tally) {
  const int lane = threadIdx.x & 31;
  const bool mine = lane < n;
  const int width = lane_width(n);
  V2 ca = v2(0.0, 0.0), cb = ca, cn = ca;
  int cid = 0;  // the lane's candidate: its near sources and vertices are read only
                // where a depth filter leaves the sign open (rare)
  if ((batch >> lane) & 1u) {
    const int c = __ldg(&g.ids[first + lane]);
    cid = c;
    ca = g.a[c];
    cb = g.b[c];
    cn = g.near[c];
  }
  while (batch) {
    const int k = __ffs(int(batch)) - 1;
    batch &= batch - 1;
    a = shfl(ca, k);
    b = shfl(cb, k);
    int stage = 0;
    if constexpr (F == 0) {
      side = sign_of(cross(a, b, p));
    } else {
      side = mine ? side_sign<F>(a, b, p, stage) : 0;
      if constexpr (F == 2)
        if (mine) tally.side.add(stage);
      if constexpr (F == 4)
        if (__any_sync(kFull, side == pred::kUndecided)) return kDeferAt - k;
    }
    if (!__ballot_sync(kFull, mine && side > 0) || !__ballot_sync(kFull, mine && side < 0))
      continue;
    const V2 near = shfl(cn, k);
    const double za = value(sc, a) - near.x, zb = value(sc, b) - near.y;
    int sza, szb;
    if constexpr (F == 0) {
      sza = sign_of(za);
      szb = sign_of(zb);
    } else {
      // The patch's depth plane against the plane of the source that gives
      // the segment its near depth, at the segment's ends.  Each binary64
      // evaluation is within 3.01 u of its terms' magnitudes (two products,
      // two sums), so a difference above 4 u of both magnitudes has its sign.
      // Otherwise: zero when the end is a mesh vertex of both triangles (both
      // planes pass through it: the projected mesh's exact depths tie there,
      // which the rounded plane coefficients can only approximate), else the
      // two planes compared exactly (zero when the source is the patch's
      // own).
      int stage_b = 0;
      const V2 mag = g.near_mag[__shfl_sync(kFull, cid, k)];
      const double bound_a = 4.0 * pred::kU64 *
          (fabs(sc.a * a.x) + fabs(sc.b * a.y) + fabs(sc.c) + mag.x);
      const double bound_b = 4.0 * pred::kU64 *
          (fabs(sc.a * b.x) + fabs(sc.b * b.y) + fabs(sc.c) + mag.y);
      const int c = __shfl_sync(kFull, cid, k);
      if (fabs(za) > bound_a) {
        sza = sign_of(za);
        stage = pred::kBinary64;
      } else {
        const int sa = g.near_src[c].x, va = g.vid[c].x;
        if (has_vertex(g, source, va) && has_vertex(g, sa, va)) {
          sza = 0;
          stage = pred::kBinary64;
        } else {
          sza = order_sign<F>(sc, value(sc, a), g.scores[sa], near.x, a, stage);
        }
      }
      if (fabs(zb) > bound_b) {
        szb = sign_of(zb);
        stage_b = pred::kBinary64;
      } else {
        const int sb = g.near_src[c].y, vb = g.vid[c].y;
        if (has_vertex(g, source, vb) && has_vertex(g, sb, vb)) {
          szb = 0;
          stage_b = pred::kBinary64;
        } else {
          szb = order_sign<F>(sc, value(sc, b), g.scores[sb], near.y, b, stage_b);
        }
      }
      if constexpr (F == 2) {
        if (lane == 0) {  // the same test on every lane: count it once
          tally.depth.add(stage);
          tally.depth.add(stage_b);
        }
      }
      if constexpr (F == 4)
        if (sza == pred::kUndecided || szb == pred::kUndecided) return kDeferAt - k;
    }
    if (sza <= 0 && szb <= 0) continue;
    const double da = cross(p, q, a), db = cross(p, q, b);
    int sda, sdb;
    if constexpr (F == 0) {
      sda = sign_of(da);
      sdb = sign_of(db);
    } else {
      int stage_b = 0;
      sda = mine ? side_sign<F>(p, q, a, stage) : 0;
      sdb = mine ? side_sign<F>(p, q, b, stage_b) : 0;
      if constexpr (F == 2) {
        if (mine) {
          tally.segment.add(stage);
          tally.segment.add(stage_b);
        }
      }
      if constexpr (F == 4)
        if (__any_sync(kFull, sda == pred::kUndecided || sdb == pred::kUndecided))
          return kDeferAt - k;
    }
    if (__ballot_sync(kFull, mine && sda <= 0 && sdb <= 0)) continue;
    double low, high, rz;
    if constexpr (F == 0) {
      const double r = da / (da - db);
      low = mine && da < 0.0 ? fmax(0.0, r) : 0.0;
      high = mine && db < 0.0 ? fmin(1.0, r) : 1.0;
    } else {
      const double r = crossing(da, db);
      low = mine && sda < 0 ? r : 0.0;
      high = mine && sdb < 0 ? r : 1.0;
    }
    for (int off = width >> 1; off > 0; off >>= 1) {  // lanes [0, width) hold the edges
      low = fmax(low, __shfl_xor_sync(kFull, low, off));
      high = fmin(high, __shfl_xor_sync(kFull, high, off));
    }
    low = __shfl_sync(kFull, low, 0);
    high = __shfl_sync(kFull, high, 0);
    if constexpr (F == 0)
      rz = za / (za - zb);
    else
      rz = crossing(za, zb);
    if (sza < 0) low = fmax(low, rz);
    if (szb < 0) high = fmin(high, rz);
    if (high > low) return k;
  }
  return -1;
}

// clean() of the polygon held one vertex per lane (x, m <= kMaxVertices
// vertices).  When no two consecutive points are near duplicates every point
// stays and only the closing merge and the area / perimeter test remain; their
// sums run in the sequential order through shuffles, so they round exactly as
// clean() does.  Otherwise lane 0 runs clean() itself on `buf` (a per-warp
// scratch of kMaxVertices points).  Returns the new size; x holds the result.
__device__ __noinline__ int serial_clean(V2 &x, int m, V2 *buf) {
  const int lane = threadIdx.x & 31;
  if (lane < m) buf[lane] = x;
  __syncwarp();
  int count = 0;
  if (lane == 0) count = clean(buf, m);
  __syncwarp();
  count = __shfl_sync(kFull, count, 0);
  if (lane < count) x = buf[lane];
  __syncwarp();
  return count;
}

__device__ inline int warp_clean(V2 &x, int m, V2 *buf) {
  const int lane = threadIdx.x & 31;
  const double merge = kEps * 0.01;
  const V2 prev = shfl(x, lane > 0 ? lane - 1 : 0);
  const bool near = lane > 0 && lane < m && !(length(x - prev) > merge);
  if (__ballot_sync(kFull, near)) return serial_clean(x, m, buf);
  int count = m;
  if (count > 1 && length(shfl(x, 0) - shfl(x, count - 1)) <= merge) --count;
  if (count < 3) return 0;
  const V2 origin = shfl(x, 0), next = shfl(x, lane + 1 < count ? lane + 1 : 0);
  const double term = cross(origin, x, next);
  const double step = fabs(next.x - x.x) + fabs(next.y - x.y);
  double area2 = 0.0, perimeter = 0.0;
  for (int j = 0; j < count; ++j) {
    area2 += __shfl_sync(kFull, term, j);
    perimeter += __shfl_sync(kFull, step, j);
  }
  return area2 <= kEps * perimeter ? 0 : count;
}

// Split the patch (one vertex per lane, q the next vertex) by the supporting
// line of a->b into the part on the left (pl, nl) and on the right (pr, nr),
// both cleaned: the vertex sequence of the sequential split (kernels.py:184-203)
// placed with ballots and prefix counts.  Returns false when a part exceeds
// kMaxVertices.
// The filtered forms (F > 0) classify the vertices by `side`, the exact sign
// first_cut found, and place the cut points with the binary64 values.
template <int F>
__device__ inline bool warp_split(V2 p, V2 q, int n, V2 a, V2 b, int side, V2 *left, V2 *right,
                                  V2 &pl, int &nl, V2 &pr, int &nr) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const V2 dir = b - a;
  const Plane s{-dir.y, dir.x, 0.0, 0.0};
  const bool mine = lane < n;
  const double du = value(s, p - a);
  const double dv = __shfl_sync(kFull, du, lane + 1 < n ? lane + 1 : 0);
  bool in, out, cut;
  if constexpr (F == 0) {
    in = mine && du >= 0.0;
    out = mine && du <= 0.0;
    cut = mine && ((du > 0.0 && dv < 0.0) || (du < 0.0 && dv > 0.0));
  } else {
    const int sv = __shfl_sync(kFull, side, lane + 1 < n ? lane + 1 : 0);
    in = mine && side >= 0;
    out = mine && side <= 0;
    cut = mine && ((side > 0 && sv < 0) || (side < 0 && sv > 0));
  }
  const unsigned bin = __ballot_sync(kFull, in), bout = __ballot_sync(kFull, out);
  const unsigned bcut = __ballot_sync(kFull, cut);
  nl = __popc(bin) + __popc(bcut);
  nr = __popc(bout) + __popc(bcut);
  if (nl > kMaxVertices || nr > kMaxVertices) return false;
  const int at_l = __popc(bin & below) + __popc(bcut & below);
  const int at_r = __popc(bout & below) + __popc(bcut & below);
  if (in) left[at_l] = p;
  if (out) right[at_r] = p;
  if (cut) {
    const V2 x = p + (F == 0 ? du / (du - dv) : crossing(du, dv)) * (q - p);
    left[at_l + (in ? 1 : 0)] = x;
    right[at_r + (out ? 1 : 0)] = x;
  }
  __syncwarp();
  pl = left[lane];
  pr = right[lane];
  __syncwarp();
  nl = warp_clean(pl, nl, left);
  nr = warp_clean(pr, nr, right);
  return true;
}

// The next round's frontier.
struct Frontier {
  V2 *v;
  int *n, *src, *cur;
  int *count, *status;
  int64_t capacity;
};

// Append a patch (one vertex per lane) to the next frontier; false on overflow.
__device__ __noinline__ bool push_patch(Frontier f, V2 p, int n, int source, int cursor) {
  const int lane = threadIdx.x & 31;
  int slot = 0;
  if (lane == 0) slot = atomicAdd(f.count, 1);
  slot = __shfl_sync(kFull, slot, 0);
  if (slot >= f.capacity) {
    if (lane == 0) set_error(f.status, kErrResidual);
    return false;
  }
  if (lane < n) f.v[int64_t(kMaxVertices) * slot + lane] = p;
  if (lane == 0) {
    f.n[slot] = n;
    f.src[slot] = source;
    f.cur[slot] = cursor;
  }
  return true;
}

// Park a patch at the top of the next frontier `f` for this round's exact
// pass (from its cursor on); false when the frontier is full.  `parked`
// counts the parked patches.
__device__ __noinline__ bool defer_patch(Frontier f, int *parked, V2 p, int n, int source,
                                         int cursor) {
  const int lane = threadIdx.x & 31;
  int k = 0;
  if (lane == 0) k = atomicAdd(parked, 1);
  k = __shfl_sync(kFull, k, 0);
  const int64_t slot = f.capacity - 1 - k;
  if (slot < 0) {
    if (lane == 0) set_error(f.status, kErrResidual);
    return false;
  }
  if (lane < n) f.v[int64_t(kMaxVertices) * slot + lane] = p;
  if (lane == 0) {
    f.n[slot] = n;
    f.src[slot] = source;
    f.cur[slot] = cursor;
  }
  return true;
}

// One frontier round, one patch per warp (frontier.py:106-223).  A patch
// meets the contour segments whose boxes overlap its own in leaf order,
// starting at its cursor (the first leaf it has not met).  The first segment
// that cuts it splits it along the segment's line: the right part goes to the
// next round, the left part continues in this warp, both with the cursor just
// past the cutting leaf (a collapsed part cancels the cut and the patch
// continues).  The continuing part keeps its walk: only the cut's leaf group
// is tested again, against the part's box; pending groups above it are
// tested against the part's box when they are expanded.  A patch that has
// met every candidate is final and goes to the output pool; one that spends
// its budget carries over.  Warps take patches from a shared counter.
//
// With filtered binary64 predicates the round runs twice: the filter-only
// form (F = 4, no exact stage, so fewer registers and less code) over the
// frontier, parking every patch whose filters cannot decide a test at the top
// of the next frontier with its cursor at that test; then form 3, with the
// exact stages, over the parked patches (`deferred_pass`).  Each patch meets
// the same tests in the same order as in one form-3 pass, so the output is
// the same.
template <int F>
__global__ void __launch_bounds__(kBlock, (F == 0 || F == 4) ? 5 : 4)
    k_subdivide(Dev d, int deferred_pass) {
  __shared__ V2 s_parts[kWarps][2][kMaxVertices];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  V2 *left_part = s_parts[warp][0], *right_part = s_parts[warp][1];
  const int par = *d.parity;
  const int from = deferred_pass ? par ^ 1 : par;
  const V2 *fv = d.fv[from];
  const int *fn = d.fn[from], *fsrc = d.fsrc[from], *fcur = d.fcur[from];
  const int parked = deferred_pass ? int(min(int64_t(d.sc[kDeferred]), d.cap.frontier)) : 0;
  const int live = deferred_pass ? parked : int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  int *taken = deferred_pass ? &d.sc[kDeferredNext] : &d.sc[kFrontierNext];
  const int leaves = *d.seg_tree.size;
  const int next_lane = lane + 1;
  const Segments segs{d.seg_tree.ids, d.seg_a, d.seg_b, d.seg_near, d.seg_near_src,
                      d.seg_near_mag, d.scores, d.seg_vid, d.faces, d.canonical, d.clipped,
                      d.src_n};
  const Frontier next{d.fv[par ^ 1], d.fn[par ^ 1], d.fsrc[par ^ 1], d.fcur[par ^ 1],
                      &d.status[kNextResidual], d.status, d.cap.frontier - parked};
  long long visits = 0, tests = 0, splits = 0;  // lane 0's tallies
  CutTally tally;
  for (;;) {
    int i = 0, failed = 0;
    if (lane == 0) {
      i = atomicAdd(taken, 1);
      failed = *(volatile int *)&d.status[kError];
    }
    i = __shfl_sync(kFull, i, 0);
    if (i >= live || __shfl_sync(kFull, failed, 0) != 0) break;
    if (deferred_pass) i = int(d.cap.frontier) - 1 - i;  // parked from the top down
    int n = fn[i];
    if (n == 0) continue;
    ++visits;
    const int source = fsrc[i];
    int cursor = fcur[i];
    V2 p = lane < n ? fv[int64_t(kMaxVertices) * i + lane] : v2(0.0, 0.0);
    V2 q = shfl(p, next_lane < n ? next_lane : 0);
    const Plane sc = d.scores[source];
    int budget = d.step_budget;
    float4 lo, hi;
    {
      const Box box = warp_bounds(p, n, sc);
      lo = box.lo;
      hi = box.hi;
    }
    lo.z = -1.0e30f;
    WarpWalk w;
    walk_begin(w, d.seg_tree, leaves, lo, hi, cursor);
    for (;;) {
      unsigned batch;
      int first, resume = leaves, cut = -1, side = 0, defer = -1;
      V2 a, b;
      while (walk_next(w, d.seg_tree, leaves, lo, hi, cursor, budget, batch, first, resume)) {
        cut = first_cut<F>(segs, batch, first, p, q, n, sc, source, a, b, side, tally);
        if constexpr (F == 4) {
          if (cut <= kDeferAt) {
            defer = first + (kDeferAt - cut);
            break;
          }
        }
        tests += __popc(cut >= 0 ? batch & (kFull >> (31 - cut)) : batch);  // met up to the cut
        if (cut >= 0) break;
      }
      if constexpr (F == 4) {
        if (defer >= 0) {
          defer_patch(next, &d.sc[kDeferred], p, n, source, defer);
          break;
        }
      }
      if (cut < 0) {
        if (resume < leaves) {
          push_patch(next, p, n, source, resume);
          break;
        }
        int out = 0;
        if (lane == 0) out = atomicAdd(&d.status[kPolygons], 1);
        out = __shfl_sync(kFull, out, 0);
        if (out >= d.cap.regions) {
          if (lane == 0) set_error(d.status, kErrOutput);
          break;
        }
        if (lane < n) d.out_v[int64_t(kMaxVertices) * out + lane] = p;
        if (lane == 0) {
          d.out_n[out] = n;
          d.out_src[out] = source;
          d.out_layer[out] = 0;
        }
        break;
      }
      cursor = first + cut + 1;
      V2 pl, pr;
      int nl, nr;
      if (!warp_split<F>(p, q, n, a, b, side, left_part, right_part, pl, nl, pr, nr)) {
        if (lane == 0) set_error(d.status, kErrPolygon);
        break;
      }
      if (nl > 0 && nr > 0) {
        ++splits;
        if (!push_patch(next, pr, nr, source, cursor)) break;
        p = pl;
        n = nl;
        q = shfl(p, next_lane < n ? next_lane : 0);
        {
      const Box box = warp_bounds(p, n, sc);
      lo = box.lo;
      hi = box.hi;
    }
        lo.z = -1.0e30f;
      }
      w.set_pending(walk_test(d.seg_tree, leaves, w, lo, hi, cursor));
      __syncwarp();  // the part buffers are rewritten by the next cut
    }
  }
  if (lane == 0) {
    count_add(&d.metrics[kTargetVisits], visits);
    count_add(&d.metrics[kContourTests], tests);
    count_add(&d.metrics[kSplits], splits);
  }
  if constexpr (F == 2) {
    tally.side.flush(d, kPredSide);
    tally.segment.flush(d, kPredSegment);
    tally.depth.flush(d, kPredDepth);
  }
}

// Swap frontiers and decide whether another round runs (event_kernels.py:12-25).
// Patches parked for the exact pass shared the next frontier's slots from the
// top: together with the pushed ones they must have fit.
__global__ void k_advance(Dev d) {
  int next = d.status[kNextResidual];
  if (int64_t(next) + d.sc[kDeferred] > d.cap.frontier) set_error(d.status, kErrResidual);
  d.metrics[kParkedPatches] += d.sc[kDeferred];
  d.sc[kDeferred] = 0;
  d.sc[kDeferredNext] = 0;
  d.status[kResidual] = next;
  d.status[kNextResidual] = 0;
  d.sc[kFrontierNext] = 0;
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
  int64_t g = ceil_div(d.cap.frontier, kWarps);
  if (g > 148 * int64_t(d.subdivide_blocks)) g = 148 * int64_t(d.subdivide_blocks);
  if (d.predicates == 3) {  // filtered binary64: filter-only pass, then the exact pass
    k_subdivide<4><<<unsigned(g), kBlock, 0, st>>>(d, 0);
    note_launch();
    // Few patches are parked (a few thousand per extraction on the knot): a
    // small grid takes them from the counter.
    k_subdivide<3><<<unsigned(g < 296 ? g : 296), kBlock, 0, st>>>(d, 1);
  } else {
    EDP_LAUNCH_FORM(d.predicates, k_subdivide, unsigned(g), kBlock, st, d, 0);
  }
  note_launch();
  k_advance<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

}  // namespace edp

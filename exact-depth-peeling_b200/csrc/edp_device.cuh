// Device-side building blocks shared by every kernel of the depth peeler.
//
// Geometry is binary64 in the normalised image window [0,1]^2, exactly as in
// the reference GPU route (warp_peel/kernels.py:9-21,139-250).  Bounding boxes
// for the hierarchies are padded binary32 (kernels.py:235-250).  All code here
// is compiled with -fmad=false, so every predicate is plain IEEE binary64 and a
// CPU restatement of the same expression gives the same bits.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include <cstdint>
#include <cuda_runtime.h>

namespace edp {

constexpr int kMaxVertices = 32;      // polygon register width (kernels.py:10)
constexpr int kSourceVertices = 8;    // triangle + near plane + 4 window planes
constexpr double kEps = 1.0e-10;      // cleanup scale in the unit window (kernels.py:11)
constexpr float kPad = 2.0e-7f;       // binary32 box padding (kernels.py:244-249)
// The reference's per-pass candidate bound (frontier.py:149,
// event_kernels.py:196-245): the primary ray pass of the hierarchy path and
// the definition of a heavy ray.
constexpr int kCandidatesPerPass = 32;

// Status slots (kernels.py:17-21, warp_peel/README.md:175-184).
enum StatusSlot : int {
  kResidual = 0, kNextResidual = 1, kPolygons = 2, kTriangles = 3, kLayers = 4,
  kPass = 5, kBoundaryVertices = 6, kDepthTies = 8, kError = 9, kMaxHidden = 10,
  kPeakResidual = 12, kStatusSlots = 16
};
// Error bits (kernels.py:20-21, warp_peel/EVENTS.md:203-207).
enum ErrorBit : int {
  kErrPolygon = 1, kErrWorker = 2, kErrResidual = 4, kErrOutput = 8, kErrVertices = 16,
  kErrTriangles = 32, kErrLayers = 64, kErrEdgeNoding = 128, kErrInput = 256,
  kErrHits = 1024, kErrRounds = 2048
};
// EventPeeler counters (warp_peel/events.py:816-844).
enum Metric : int {
  kTargetVisits = 0, kContourTests, kSplits, kRayGroups, kRayCandidateTests, kRayHits,
  kRounds, kUniqueContours, kHeavyRayGroups, kBeamAttempts, kCertifiedBeams,
  kBeamCandidateTests, kHeavyBeams, kRankComponents, kRankConnections,
  kConnectionContourTests, kMergedPolygons, kMatchedPatchEdges, kEdgeHashMisses,
  kHeavyNodedPolygons,
  // Filtered binary64 predicates: work the filter-only kernels left to the
  // exact passes (parked patches, containment tests, hit groups, polygons).
  kParkedPatches, kDeferredContainTests, kDeferredHitGroups, kDeferredPolygons, kMetrics
};

// ---------------------------------------------------------------- vectors
struct V2 { double x, y; };
__host__ __device__ inline V2 v2(double x, double y) { return V2{x, y}; }
__host__ __device__ inline V2 operator+(V2 a, V2 b) { return V2{a.x + b.x, a.y + b.y}; }
__host__ __device__ inline V2 operator-(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
__host__ __device__ inline V2 operator*(double s, V2 a) { return V2{s * a.x, s * a.y}; }
__host__ __device__ inline V2 operator/(V2 a, double s) { return V2{a.x / s, a.y / s}; }
__host__ __device__ inline bool operator==(V2 a, V2 b) { return a.x == b.x && a.y == b.y; }
__host__ __device__ inline bool operator!=(V2 a, V2 b) { return !(a == b); }
__host__ __device__ inline double dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
__host__ __device__ inline double length(V2 a) { return sqrt(a.x * a.x + a.y * a.y); }
// Lexicographic order of points (event_kernels.py:66-68).
__host__ __device__ inline bool less(V2 a, V2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); }

// Orientation of c relative to a->b: positive on the left (kernels.py:139-143).
__host__ __device__ inline double cross(V2 a, V2 b, V2 c) {
  V2 u = b - a, v = c - a;
  return u.x * v.y - u.y * v.x;
}

// Affine depth plane s = (a, b, c): value a x + b y + c (kernels.py:179-181).
struct Plane { double a, b, c, pad; };
__host__ __device__ inline double value(const Plane &s, V2 x) { return s.a * x.x + s.b * x.y + s.c; }

// ---------------------------------------------------------------- polygons
// The polygon helpers below are host and device functions so that the CPU
// tests can run the kernels' own code (binary64 without contraction rounds
// the same on both).
// Remove near-duplicate points and collapse slivers (kernels.py:146-176):
// points closer than EPS/100 merge, and a translation-stable area/perimeter
// test drops polygons narrower than about EPS.  Returns the new size (0 when
// the polygon collapsed); sizes above kMaxVertices are returned unchanged so
// that the caller can raise the polygon-capacity error.
__host__ __device__ inline int clean(V2 *p, int n) {
  if (n > kMaxVertices) return n;
  int count = 0;
  const double merge = kEps * 0.01;
  for (int j = 0; j < n; ++j) {
    V2 x = p[j];
    if (count == 0 || length(x - p[count - 1]) > merge) p[count++] = x;
  }
  if (count > 1 && length(p[0] - p[count - 1]) <= merge) --count;
  if (count < 3) return 0;
  V2 origin = p[0];
  double area2 = 0.0, perimeter = 0.0;
  for (int j = 0; j < count; ++j) {
    V2 a = p[j], b = p[(j + 1) % count];
    area2 += cross(origin, a, b);
    perimeter += fabs(b.x - a.x) + fabs(b.y - a.y);
  }
  if (area2 <= kEps * perimeter) return 0;
  return count;
}

__host__ __device__ inline int append(V2 *p, int n, V2 x) {
  if (n < kMaxVertices) p[n] = x;
  return n + 1;
}

// Split a convex polygon by the line s(x - anchor) = 0 into the part with
// s >= 0 (inside) and s <= 0 (outside), then clean both (kernels.py:184-203).
// Evaluating relative to the anchor keeps short clipping edges in place.
__host__ __device__ inline void split_at(const V2 *p, int n, const Plane &s, V2 anchor, V2 *in,
                                         int &ni, V2 *out, int &no) {
  ni = 0;
  no = 0;
  for (int j = 0; j < n; ++j) {
    V2 a = p[j], b = p[(j + 1) % n];
    double da = value(s, a - anchor), db = value(s, b - anchor);
    if (da >= 0.0) ni = append(in, ni, a);
    if (da <= 0.0) no = append(out, no, a);
    if ((da > 0.0 && db < 0.0) || (da < 0.0 && db > 0.0)) {
      V2 x = a + (da / (da - db)) * (b - a);
      ni = append(in, ni, x);
      no = append(out, no, x);
    }
  }
  ni = clean(in, ni);
  no = clean(out, no);
}

// Split by the supporting line of edge a->b: inside is to the left.
__host__ __device__ inline void split_edge(const V2 *p, int n, V2 a, V2 b, V2 *in, int &ni,
                                           V2 *out, int &no) {
  V2 d = b - a;
  Plane s{-d.y, d.x, 0.0, 0.0};
  split_at(p, n, s, a, in, ni, out, no);
}

// Some edge of a has no vertex of b strictly on its left (kernels.py:219-232).
__host__ __device__ inline bool separated(const V2 *a, int na, const V2 *b, int nb) {
  for (int j = 0; j < na; ++j) {
    bool positive = false;
    for (int k = 0; k < nb; ++k)
      if (cross(a[j], a[(j + 1) % na], b[k]) > 0.0) positive = true;
    if (!positive) return true;
  }
  return false;
}

// ---------------------------------------------------------------- boxes
struct Box { float4 lo, hi; };
__device__ inline float4 empty_lo() { return make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.f); }
__device__ inline float4 empty_hi() { return make_float4(-1.0e30f, -1.0e30f, -1.0e30f, 0.f); }

// Padded binary32 bounds of a polygon with depth (kernels.py:235-250).
__device__ inline void polygon_bounds(const V2 *p, int n, const Plane &score, float4 &lo,
                                      float4 &hi) {
  double lx = 1.0e30, ly = 1.0e30, lz = 1.0e30, hx = -1.0e30, hy = -1.0e30, hz = -1.0e30;
  for (int j = 0; j < n; ++j) {
    double z = value(score, p[j]);
    lx = fmin(lx, p[j].x); ly = fmin(ly, p[j].y); lz = fmin(lz, z);
    hx = fmax(hx, p[j].x); hy = fmax(hy, p[j].y); hz = fmax(hz, z);
  }
  double pz = 2.0e-7 * fmax(1.0, fmax(fabs(lz), fabs(hz)));
  lo = make_float4(float(lx - 2.0e-7), float(ly - 2.0e-7), float(lz - pz), 0.f);
  hi = make_float4(float(hx + 2.0e-7), float(hy + 2.0e-7), float(hz + pz), 0.f);
}

// ---------------------------------------------------------------- hierarchy
// A complete binary tree over a power-of-two number of Morton-ordered leaves,
// one item per leaf; node 1 is the root, node i has children 2i and 2i+1 and
// leaves are nodes [size, 2 size).  A node's two corners share one 32-byte
// sector and siblings are adjacent, so a traversal step costs one miss.  The size lives in device memory so one
// captured graph serves any leaf count up to the allocated capacity
// (solver.py:34-89, kernels.py:24-116).
struct Tree {
  const float4 *nodes;  // node i: nodes[2i] = lower corner, nodes[2i+1] = upper corner
  const int *ids;
  const int *size;  // device scalar: number of leaves (power of two)
};

__device__ inline int successor(int node) {
  while (node > 0 && (node & 1) != 0) node >>= 1;
  if (node > 0) node += 1;
  return node;
}

__device__ inline bool overlaps(float4 a, float4 b, float4 lo, float4 hi) {
  return a.x <= hi.x && a.y <= hi.y && a.z <= hi.z && b.x >= lo.x && b.y >= lo.y &&
         b.z >= lo.z;
}

// Stackless depth-first step: advance from `node` to the next overlapping
// leaf, stopping at `end` (0 for a whole-tree walk).  Returns the item id in
// `found` (or -1) and the node at which to resume (kernels.py:41-64,
// event_kernels.py:172-193).
__device__ inline int query_next(const Tree &t, int leaves, float4 lo, float4 hi, int node,
                                 int end, int &found) {
  found = -1;
  while (node > 0 && node != end) {
    float4 a = __ldg(&t.nodes[2 * node]), b = __ldg(&t.nodes[2 * node + 1]);
    if (overlaps(a, b, lo, hi)) {
      if (node < leaves) {
        node = 2 * node;
      } else {
        found = __ldg(&t.ids[node - leaves]);
        node = successor(node);
        break;
      }
    } else {
      node = successor(node);
    }
  }
  return node;
}

// ---------------------------------------------------------------- warp walk
// A warp walks the tree 32 nodes at a time: the descendants of node k five
// levels down are the contiguous nodes 32k .. 32k+31, so one step is one
// coalesced 1 KB load and one ballot.  The first group sits r = 1..5 levels
// below the root so that every later group, leaf groups included, is 32 wide.
// Groups are expanded depth first, lowest lane first, so leaf batches come out
// in increasing leaf order: the candidates, and their order, are exactly those
// of the binary successor walk above.  Only leaves in [cursor, end) are
// produced.  Every member is warp-uniform; all 32 lanes must call together.
struct WarpWalk {
  int levels;      // leaves = 2^levels
  int top;         // level of the first group
  int end;         // first leaf past the walked range
  int depth, level, base, width;
  // Overlapping, not yet expanded nodes per depth (lane bits).  Leaves fit an
  // int, so there are at most 30 levels and depths 0..5; the depth is
  // warp-uniform, so named registers and a uniform switch keep the stack out
  // of local memory.
  unsigned p0, p1, p2, p3, p4, p5;
  __device__ unsigned pending() const {
    switch (depth) {
      case 0: return p0;
      case 1: return p1;
      case 2: return p2;
      case 3: return p3;
      case 4: return p4;
      default: return p5;
    }
  }
  __device__ void set_pending(unsigned v) {
    switch (depth) {
      case 0: p0 = v; break;
      case 1: p1 = v; break;
      case 2: p2 = v; break;
      case 3: p3 = v; break;
      case 4: p4 = v; break;
      default: p5 = v; break;
    }
  }
};

__device__ inline unsigned walk_test(const Tree &t, int leaves, const WarpWalk &w, float4 lo,
                                     float4 hi, int cursor) {
  const int lane = threadIdx.x & 31;
  bool hit = false;
  if (lane < w.width) {
    const int node = w.base + lane;
    const int first = (node << (w.levels - w.level)) - leaves;  // leaves below: [first, last]
    const int last = ((node + 1) << (w.levels - w.level)) - leaves - 1;
    if (last >= cursor && first < w.end)
      hit = overlaps(__ldg(&t.nodes[2 * node]), __ldg(&t.nodes[2 * node + 1]), lo, hi);
  }
  return __ballot_sync(0xffffffffu, hit);
}

__device__ inline void walk_begin(WarpWalk &w, const Tree &t, int leaves, float4 lo, float4 hi,
                                  int cursor, int end = 0x7fffffff) {
  w.end = end;
  w.levels = 31 - __clz(leaves);
  w.top = w.levels == 0 ? 0 : (w.levels - 1) % 5 + 1;
  w.depth = 0;
  w.level = w.top;
  w.base = 1 << w.top;
  w.width = 1 << w.top;
  w.p1 = w.p2 = w.p3 = w.p4 = w.p5 = 0u;
  w.p0 = cursor < leaves && cursor < end ? walk_test(t, leaves, w, lo, hi, cursor) : 0u;
}

// Advance to the next leaf batch: bit i of `batch` marks an overlapping leaf
// `first + i`.  Returns false when no leaf is left (resume = leaves) or when
// `budget` group tests are spent first (resume = the first leaf not walked;
// every overlapping leaf before it has been produced).
__device__ inline bool walk_next(WarpWalk &w, const Tree &t, int leaves, float4 lo, float4 hi,
                                 int cursor, int &budget, unsigned &batch, int &first,
                                 int &resume) {
  for (;;) {
    unsigned pending = w.pending();
    if (w.level == w.levels && pending != 0) {
      batch = pending;
      w.set_pending(0u);
      first = w.base - leaves;
      return true;
    }
    while (pending == 0) {
      if (w.depth == 0) {
        resume = leaves;
        return false;
      }
      --w.depth;
      w.level -= 5;
      w.base = w.depth == 0 ? 1 << w.top : (w.base >> 5) & ~31;
      w.width = w.depth == 0 ? 1 << w.top : 32;
      pending = w.pending();
    }
    const int node = w.base + __ffs(int(pending)) - 1;
    if (budget <= 0) {
      resume = max(cursor, (node << (w.levels - w.level)) - leaves);
      return false;
    }
    --budget;
    w.set_pending(pending & (pending - 1));
    ++w.depth;
    w.level += 5;
    w.base = node << 5;
    w.width = 32;
    w.set_pending(walk_test(t, leaves, w, lo, hi, cursor));
  }
}

// 15 bits per axis Morton code of a box centre clamped to [0,1] (kernels.py:67-91).
__host__ __device__ inline uint32_t part1by1(uint32_t x) {
  x &= 0x0000ffffu;
  x = (x | (x << 8)) & 0x00ff00ffu;
  x = (x | (x << 4)) & 0x0f0f0f0fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// ---------------------------------------------------------------- hashing
// SplitMix64 finaliser (Steele, Lea and Flood 2014), a public-domain mixer.
__host__ __device__ inline uint64_t mix64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
// Bits of a double with -0 folded onto +0, so that equal values hash equally.
__device__ inline uint64_t key_bits(double v) {
  return v == 0.0 ? 0ull : static_cast<uint64_t>(__double_as_longlong(v));
}

// Order-preserving map of a double onto uint64 (for radix sorting).
__device__ inline uint64_t ordered_bits(double v) {
  uint64_t b = static_cast<uint64_t>(__double_as_longlong(v == 0.0 ? 0.0 : v));
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__device__ inline double atomic_min_double(double *addr, double v) {
  unsigned long long *a = reinterpret_cast<unsigned long long *>(addr);
  unsigned long long old = *a, assumed;
  while (v < __longlong_as_double(old)) {
    assumed = old;
    old = atomicCAS(a, assumed, static_cast<unsigned long long>(__double_as_longlong(v)));
    if (old == assumed) break;
  }
  return __longlong_as_double(old);
}
__device__ inline double atomic_max_double(double *addr, double v) {
  unsigned long long *a = reinterpret_cast<unsigned long long *>(addr);
  unsigned long long old = *a, assumed;
  while (v > __longlong_as_double(old)) {
    assumed = old;
    old = atomicCAS(a, assumed, static_cast<unsigned long long>(__double_as_longlong(v)));
    if (old == assumed) break;
  }
  return __longlong_as_double(old);
}

__device__ inline void set_error(int *status, int bit) { atomicOr(&status[kError], bit); }

// Reserve `count` consecutive slots of an append counter for this thread,
// with a single atomic per group of converged threads (the group's scan gives
// each thread its offset).  Avoids serialising millions of appends on one
// address.
__device__ inline int reserve(int *counter, int count) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  int offset = cg::exclusive_scan(g, count);
  int total = g.shfl(offset + count, g.size() - 1);
  int base = 0;
  if (g.thread_rank() == 0 && total) base = atomicAdd(counter, total);
  return g.shfl(base, 0) + offset;
}
__device__ inline long long reserve(long long *counter, int count) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  int offset = cg::exclusive_scan(g, count);
  int total = g.shfl(offset + count, g.size() - 1);
  unsigned long long base = 0;
  if (g.thread_rank() == 0 && total)
    base = atomicAdd(reinterpret_cast<unsigned long long *>(counter),
                     static_cast<unsigned long long>(total));
  return static_cast<long long>(g.shfl(base, 0)) + offset;
}
// Add to a counter with one atomic per group of converged threads.
__device__ inline void count_add(long long *counter, long long v) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  long long total = cg::reduce(g, v, cg::plus<long long>());
  if (g.thread_rank() == 0 && total)
    atomicAdd(reinterpret_cast<unsigned long long *>(counter), static_cast<unsigned long long>(total));
}

}  // namespace edp

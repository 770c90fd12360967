// Rank stage: certified patch connectivity (over the contour-segment grid),
// canonical samples, shared query groups with certified rectangles, ray hit
// gathering (over the source grid, or the source hierarchy with its
// continuation), the per-group hit order, per-polygon rank assignment and the
// optional convex merge (warp_peel/events.py:291-635, components.py, beams.py,
// event_kernels.py:28-385).
#include "../../include/edp.h"
#include "edp_filtered.cuh"
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kBlock = 128;
// Persistent continuation grid: 8 blocks of 256 threads on each of the 148 SMs
// (the reference launches 8192 workers, events.py:510,564, sized for a smaller part).
constexpr int kHeavyBlock = 256;
constexpr int kHeavyBlocks = 148 * 8;
constexpr int kCells = 1024;         // 32 x 32 image buckets (beams.py:18-22)

__device__ inline int64_t tid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ inline int64_t stride() { return int64_t(gridDim.x) * blockDim.x; }
__device__ inline void add_metric(const Dev &d, int m, long long v) { count_add(&d.metrics[m], v); }
__device__ inline int live_polygons(const Dev &d) { return d.sc[kLivePolygons]; }
__device__ inline float lower_f(double x) { return __double2float_rd(x); }
__device__ inline float upper_f(double x) { return __double2float_ru(x); }

__global__ void k_rank_begin(Dev d) {
  d.sc[kLivePolygons] = int(min(int64_t(d.status[kPolygons]), d.cap.regions));
}

// counts[k] is the edge count of the k-th polygon in spatial order, so that
// the patch edges are laid out, matched and connected in that order.
__global__ void k_polygon_init(Dev d) {
  const int live = live_polygons(d);
  for (int64_t i = tid(); i < live; i += stride()) {
    d.counts[i] = d.out_n[d.order[i]];
    d.parents[i] = int(i);
    d.group_counts[i] = 0;
  }
}

__global__ void k_check_edges(Dev d) {
  int total = d.sc[kPatchEdges];
  if (int64_t(total) > d.cap.vertices) {
    set_error(d.status, kErrVertices);
    d.sc[kPatchEdges] = int(d.cap.vertices);
  }
}

// Owner of each patch edge: the welded mesh edge when the patch edge lies on
// an internal (non-contour) edge of its unclipped source, else the source
// itself (components.py:287-327).
__global__ void k_patch_edges(Dev d) {
  const int live = live_polygons(d);
  for (int64_t o = tid(); o < live; o += stride()) {
    if (d.status[kError] != 0) return;
    const int i = d.order[o];
    const V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    const int n = d.out_n[i], source = d.out_src[i];
    const V2 *q = d.src_v + int64_t(kSourceVertices) * source;
    const int qn = d.src_n[source];
    for (int k = 0; k < n; ++k) {
      int64_t slot = int64_t(d.offsets[o]) + k;
      if (slot >= d.cap.vertices) break;
      V2 a = p[k], b = p[(k + 1) % n];
      unsigned long long owner = 0x8000000000000000ull | static_cast<unsigned>(source);
      if (d.clipped[source] == 0) {
        for (int j = 0; j < qn; ++j) {
          int edge = d.facing[source] < 0 ? (4 - j) % 3 : j;
          if (d.masks[3 * int64_t(source) + edge] == 0) {
            V2 u = q[j], v = q[(j + 1) % qn];
            if ((a == u || a == v || cross(u, v, a) == 0.0) &&
                (b == u || b == v || cross(u, v, b) == 0.0)) {
              owner = d.edge_keys[3 * int64_t(source) + edge];
              break;
            }
          }
        }
      }
      d.owners[slot] = owner;
      d.starts[slot] = a;
      d.ends[slot] = b;
      d.tasks[slot] = make_int2(i, k);
      d.partners[slot] = -1;
    }
  }
}

__device__ inline uint64_t point_key(V2 x) {
  return mix64(key_bits(x.x)) ^ mix64(key_bits(x.y) + 19ull);
}

// A bounded open-addressing table pairs each patch edge with the reversed edge
// of another patch that has the same owner (components.py:330-366).  The key
// is symmetric in the endpoints so both directions probe the same chain.
__global__ void k_match_edges(Dev d) {
  const int total = d.sc[kPatchEdges];
  for (int64_t i = tid(); i < total; i += stride()) {
    if (d.status[kError] != 0) return;
    V2 a = d.starts[i], b = d.ends[i];
    if (a == b) continue;
    const unsigned long long owner = d.owners[i];
    uint64_t key = mix64(owner) ^ point_key(a) ^ point_key(b);
    uint32_t slot = uint32_t(key) & uint32_t(d.edge_hash_mask);
    bool placed = false;
    for (int attempt = 0; attempt < 64; ++attempt) {
      int other = atomicCAS(&d.edge_hash[slot], -1, int(i));
      if (other < 0) {
        placed = true;
        break;
      }
      if (d.owners[other] == owner && d.tasks[i].x != d.tasks[other].x && a == d.ends[other] &&
          b == d.starts[other]) {
        d.partners[i] = other;
        d.partners[other] = int(i);
        add_metric(d, kMatchedPatchEdges, 1);
        placed = true;
        break;
      }
      slot = (slot + 1) & uint32_t(d.edge_hash_mask);
    }
    if (!placed) add_metric(d, kEdgeHashMisses, 1);  // loses only the optimisation
  }
}

__device__ inline int uf_read(int *p, int i) { return *reinterpret_cast<volatile int *>(p + i); }

// Lock-free union-find with atomic-min links (components.py:369-390).
__device__ inline int uf_root(int *parents, int i) {
  int node = i;
  while (true) {
    int parent = uf_read(parents, node);
    if (parent == node) break;
    int grand = uf_read(parents, parent);
    atomicMin(&parents[node], grand);
    node = grand;
  }
  return node;
}

__device__ inline void uf_unite(int *parents, int a, int b) {
  int ra = uf_root(parents, a), rb = uf_root(parents, b);
  while (ra != rb) {
    int high = max(ra, rb), low = min(ra, rb);
    int old = atomicMin(&parents[high], low);
    if (old == high) break;
    ra = uf_root(parents, old);
    rb = uf_root(parents, low);
  }
}

// Contour-segment grid (the same cells as the source grid): each distinct
// segment whose box, grown by 1e-6, meets at most kSegCells cells is listed
// in them; longer ones go to a list every query reads.
__device__ inline int seg_grid_cell(double v, int g) {
  const double c = floor(v * double(g));
  return c < 0.0 ? 0 : c > double(g - 1) ? g - 1 : int(c);
}

__device__ inline bool segment_cells(const Dev &d, int c, int &cx0, int &cx1, int &cy0, int &cy1) {
  const float4 lo = d.seg_lo[c], hi = d.seg_hi[c];
  if (!(lo.x <= hi.x && lo.y <= hi.y)) return false;
  const int g = d.grid_size;
  cx0 = seg_grid_cell(double(lo.x) - 1.0e-6, g);
  cx1 = seg_grid_cell(double(hi.x) + 1.0e-6, g);
  cy0 = seg_grid_cell(double(lo.y) - 1.0e-6, g);
  cy1 = seg_grid_cell(double(hi.y) + 1.0e-6, g);
  return true;
}

__global__ void k_seg_grid_count(Dev d) {
  const int total = d.sc[kSegmentCount];
  for (int64_t c = tid(); c < total; c += stride()) {
    int cx0, cx1, cy0, cy1;
    if (!segment_cells(d, int(c), cx0, cx1, cy0, cy1)) continue;
    if ((cx1 - cx0 + 1) * (cy1 - cy0 + 1) > kSegCells) {
      d.seg_big[reserve(&d.sc[kSegBig], 1)] = int(c);
      continue;
    }
    for (int cy = cy0; cy <= cy1; ++cy)
      for (int cx = cx0; cx <= cx1; ++cx) atomicAdd(&d.seg_count[cy * d.grid_size + cx], 1);
  }
}

__global__ void k_seg_grid_fill(Dev d) {
  if (tid() == 0) d.sc[kSegGridOn] = d.sc[kSegBig] <= 64 ? 1 : 0;
  const int total = d.sc[kSegmentCount];
  for (int64_t c = tid(); c < total; c += stride()) {
    int cx0, cx1, cy0, cy1;
    if (!segment_cells(d, int(c), cx0, cx1, cy0, cy1)) continue;
    if ((cx1 - cx0 + 1) * (cy1 - cy0 + 1) > kSegCells) continue;
    for (int cy = cy0; cy <= cy1; ++cy)
      for (int cx = cx0; cx <= cx1; ++cx) {
        const int cell = cy * d.grid_size + cx;
        d.seg_entries[d.seg_start[cell] + atomicSub(&d.seg_count[cell], 1) - 1] = int(c);
      }
  }
}

// Matched edges are connected when no nearer-or-equal contour passes through
// the edge midpoint (components.py:393-450).  Candidate segments are those
// whose box meets the query box: from the segment grid's cell of the midpoint
// (every such segment is listed there or among the long ones), else from the
// contour hierarchy.  Any blocking segment decides, so the order does not
// matter; the visit counter counts segments met until the first blocker.
__global__ void k_connect(Dev d) {
  const int total = d.sc[kPatchEdges];
  const int leaves = *d.seg_tree.size;
  for (int64_t i = tid(); i < total; i += stride()) {
    if (d.status[kError] != 0) return;
    int other = d.partners[i];
    if (other <= i) continue;
    int2 task = d.tasks[i];
    V2 a = d.starts[i], b = d.ends[i];
    if (length(b - a) <= 16.0 * kEps) continue;
    V2 x = 0.5 * (a + b);
    double z = value(d.scores[d.out_src[task.x]], x);
    double pad = 2.0e-7 * fmax(1.0, fabs(z));
    float4 lo = make_float4(lower_f(x.x - 2.0e-7), lower_f(x.y - 2.0e-7), -1.0e30f, 0.f);
    float4 hi = make_float4(upper_f(x.x + 2.0e-7), upper_f(x.y + 2.0e-7), upper_f(z + pad), 0.f);
    int visits = 0;
    bool safe = true;
    // Does segment c pass through x at or in front of the patch?
    auto blocks = [&](int c) {
      ++visits;
      V2 u = d.seg_a[c], v = d.seg_b[c], dv = v - u;
      double len = length(dv);
      if (len > 0.0) {
        double t = dot(x - u, dv) / dot(dv, dv);
        if (fabs(cross(u, v, x)) <= kEps * len && t >= -kEps / len && t <= 1.0 + kEps / len) {
          V2 near = d.seg_near[c];
          double depth = near.x + t * (near.y - near.x);
          if (depth <= z + pad) return true;
        }
      }
      return false;
    };
    if (d.sc[kSegGridOn]) {
      const int g = d.grid_size;
      const int cell = seg_grid_cell(x.y, g) * g + seg_grid_cell(x.x, g);
      const int begin = d.seg_start[cell], end = d.seg_start[cell + 1], big = d.sc[kSegBig];
      for (int e = begin; e < end + big; ++e) {
        const int c = e < end ? d.seg_entries[e] : d.seg_big[e - end];
        if (!overlaps(d.seg_lo[c], d.seg_hi[c], lo, hi)) continue;
        if (blocks(c)) {
          safe = false;
          break;
        }
      }
    } else {
      int node = 1;
      while (node > 0) {
        int c;
        node = query_next(d.seg_tree, leaves, lo, hi, node, 0, c);
        if (c < 0) break;
        if (blocks(c)) {
          safe = false;
          break;
        }
      }
    }
    add_metric(d, kConnectionContourTests, visits);
    if (safe) {
      uf_unite(d.parents, task.x, d.tasks[other].x);
      add_metric(d, kRankConnections, 1);
    }
  }
}

__global__ void k_roots(Dev d, int connected) {
  const int live = live_polygons(d);
  int components = 0;
  for (int64_t i = tid(); i < live; i += stride()) {
    int r = connected ? uf_root(d.parents, int(i)) : int(i);
    d.reps[i] = r;
    components += r == int(i);
  }
  if (components) add_metric(d, kRankComponents, d.propagate_ranks ? components : 0);
}

// Canonical interior sample of each polygon's representative: the vertex mean
// accumulated from the lexicographically smallest vertex, so that rotated
// copies of one footprint share bit-identical samples (event_kernels.py:28-48).
__global__ void k_samples(Dev d) {
  const int live = live_polygons(d);
  for (int64_t i = tid(); i < live; i += stride()) {
    int r = d.reps[i];
    const V2 *p = d.out_v + int64_t(kMaxVertices) * r;
    int n = d.out_n[r];
    int anchor = 0;
    for (int j = 1; j < n; ++j)
      if (less(p[j], p[anchor])) anchor = j;
    V2 x = v2(0.0, 0.0);
    for (int j = 0; j < n; ++j) x = x + p[(anchor + j) % n] / double(n);
    d.samples[i] = x;
  }
}

__device__ inline int cell_of(V2 x) {
  int cx = int(fmin(fmax(x.x * 32.0, 0.0), 31.0)), cy = int(fmin(fmax(x.y * 32.0, 0.0), 31.0));
  return cx * 32 + cy;
}

// Identical samples form one query group, whose id is the smallest polygon
// index in it (the reference groups by sorted position, event_kernels.py:71-92).
// Each 32x32 image cell also gathers its samples' bounding rectangle as a
// sharing proposal (beams.py:49-86).  Samples are taken in spatial order, so
// the lanes of a warp mostly share cells: lanes with one cell combine their
// minimum index and rectangle first (exact min / max) and one of them updates
// the cell.
__global__ void k_group_insert(Dev d) {
  namespace cg = cooperative_groups;
  const int live = live_polygons(d);
  for (int64_t k = tid(); k < live; k += stride()) {
    const int i = d.order[k];
    V2 x = d.samples[i];
    uint32_t slot = uint32_t(point_key(x)) & uint32_t(d.sample_mask);
    for (int probe = 0; probe <= d.sample_mask; ++probe) {
      int cur = atomicCAS(&d.sample_table[slot], -1, int(i));
      if (cur == -1 || d.samples[cur] == x) break;
      slot = (slot + 1) & uint32_t(d.sample_mask);
    }
    atomicMin(&d.sample_min[slot], int(i));
    d.sample_slot[i] = int(slot);
    if (d.share_regions) {
      const int c = cell_of(x);
      cg::coalesced_group cell = cg::labeled_partition(cg::coalesced_threads(), c);
      const int first = cg::reduce(cell, i, cg::less<int>());
      const double lx = cg::reduce(cell, x.x, cg::less<double>());
      const double ly = cg::reduce(cell, x.y, cg::less<double>());
      const double hx = cg::reduce(cell, x.x, cg::greater<double>());
      const double hy = cg::reduce(cell, x.y, cg::greater<double>());
      if (cell.thread_rank() == 0) {
        atomicMin(&d.cell_min[c], first);
        atomic_min_double(&d.cell_bounds[4 * c + 0], lx);
        atomic_min_double(&d.cell_bounds[4 * c + 1], ly);
        atomic_max_double(&d.cell_bounds[4 * c + 2], hx);
        atomic_max_double(&d.cell_bounds[4 * c + 3], hy);
      }
    }
  }
}

__global__ void k_group_resolve(Dev d) {
  const int live = live_polygons(d);
  for (int64_t i = tid(); i < live; i += stride()) d.groups[i] = d.sample_min[d.sample_slot[i]];
}

__global__ void k_cells_reset(Dev d) {
  int c = int(tid());
  if (c < kCells) {
    d.cell_min[c] = 0x7fffffff;
    d.cell_valid[c] = 0;
    d.cell_bounds[4 * c + 0] = 1.0e30;
    d.cell_bounds[4 * c + 1] = 1.0e30;
    d.cell_bounds[4 * c + 2] = -1.0e30;
    d.cell_bounds[4 * c + 3] = -1.0e30;
  }
}

// Source polygon strictly covers the four corners of cell c's rectangle with
// an edge-length margin (beams.py:89-98).
__device__ inline bool covers(const Dev &d, int source, int c) {
  const V2 *p = d.src_v + int64_t(kSourceVertices) * source;
  const int n = d.src_n[source];
  const double *b = d.cell_bounds + 4 * c;
  for (int j = 0; j < n; ++j) {
    V2 u = p[j], v = p[(j + 1) % n];
    double margin = kEps * length(v - u);
    for (int k = 0; k < 4; ++k) {
      V2 x = v2(b[2 * (k % 2)], b[1 + 2 * (k / 2)]);
      if (cross(u, v, x) <= margin) return false;
    }
  }
  return n > 0;
}

__device__ inline void cell_box(const Dev &d, int c, float4 &lo, float4 &hi) {
  const double *b = d.cell_bounds + 4 * c;
  lo = make_float4(lower_f(b[0] - 2.0e-7), lower_f(b[1] - 2.0e-7), -1.0e30f, 0.f);
  hi = make_float4(upper_f(b[2] + 2.0e-7), upper_f(b[3] + 2.0e-7), 1.0e30f, 0.f);
}

// Certified rectangles: a cell's samples may share one ray group only if
// every source candidate strictly covers the cell's sample rectangle; on
// intersection-resolved input the covering set and its depth order are then
// constant over the rectangle (beams.py:109-146).
__global__ void __launch_bounds__(kBlock) k_certify(Dev d) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int c = int(tid() >> 5);  // one warp per cell
  if (c >= kCells || d.status[kError] != 0 || d.cell_min[c] == 0x7fffffff) return;
  const double *b = d.cell_bounds + 4 * c;
  if (b[0] == b[2] && b[1] == b[3]) return;  // identical samples already share
  float4 lo, hi;
  cell_box(d, c, lo, hi);
  const int leaves = *d.source_tree.size;
  // Up to kCandidatesPerPass candidates in leaf order, a candidate per lane;
  // the first one that does not cover the cell rejects it.
  WarpWalk w;
  walk_begin(w, d.source_tree, leaves, lo, hi, 0);
  int budget = 0x7fffffff, first, resume, met = 0, accepted = 1, last = -1;
  unsigned batch;
  while (met < kCandidatesPerPass &&
         walk_next(w, d.source_tree, leaves, lo, hi, 0, budget, batch, first, resume)) {
    unsigned take = batch;
    for (int extra = __popc(take) - (kCandidatesPerPass - met); extra > 0; --extra)
      take &= ~(1u << (31 - __clz(take)));  // drop the highest leaves past the budget
    const bool bad = ((take >> lane) & 1u) && !covers(d, __ldg(&d.source_tree.ids[first + lane]), c);
    const unsigned bads = __ballot_sync(full, bad);
    if (bads) {
      const int k = __ffs(int(bads)) - 1;
      met += __popc(take & (full >> (31 - k)));  // met up to the rejecting one
      accepted = 0;
      break;
    }
    met += __popc(take);
    last = first + 31 - __clz(take);
  }
  if (lane != 0) return;
  add_metric(d, kBeamAttempts, 1);
  add_metric(d, kBeamCandidateTests, met);
  d.cell_valid[c] = accepted;
  // The binary walk would stop after its 32nd candidate with the rest of the
  // hierarchy still to walk unless that candidate was the last leaf.
  if (accepted && met == kCandidatesPerPass && last != leaves - 1) {
    int slot = int(atomicAdd(reinterpret_cast<unsigned long long *>(&d.metrics[kHeavyBeams]), 1ull));
    d.heavy_beams[slot] = make_int2(c, leaves + last + 1);
  }
}

// Disjoint-subtree partition of the unvisited traversal suffixes of long
// queries (event_kernels.py:248-298, beams.py:149-188).
__device__ inline void heavy_partition(int leaves, long long jobs, int &parts, int &width) {
  parts = min(8192, leaves);
  while (parts > 16 && (long long)parts * jobs > 65536) parts /= 2;
  width = leaves / parts;
}

__global__ void k_certify_heavy(Dev d) {
  if (d.status[kError] != 0) return;
  const int leaves = *d.source_tree.size;
  const long long jobs = d.metrics[kHeavyBeams];
  int parts, width;
  heavy_partition(leaves, jobs, parts, width);
  for (long long task = tid(); task < jobs * parts; task += stride()) {
    int2 job = d.heavy_beams[task / parts];
    int part = int(task % parts), c = job.x;
    int first = leaves + part * width;
    if (job.y >= first + width || atomicAdd(&d.cell_valid[c], 0) == 0) continue;
    int root = parts + part, node = job.y > first ? job.y : root, end = successor(root);
    float4 lo, hi;
    cell_box(d, c, lo, hi);
    int visits = 0;
    while (node > 0 && node != end) {
      int s;
      node = query_next(d.source_tree, leaves, lo, hi, node, end, s);
      if (s < 0) break;
      ++visits;
      if (!covers(d, s, c)) {
        atomicMin(&d.cell_valid[c], 0);
        break;
      }
    }
    add_metric(d, kBeamCandidateTests, visits);
  }
}

__global__ void k_apply_cells(Dev d) {
  const int live = live_polygons(d);
  for (int64_t i = tid(); i < live; i += stride()) {
    int c = cell_of(d.samples[i]);
    if (d.cell_valid[c] != 0) {
      int root = d.cell_min[c];
      d.groups[i] = root;
      if (root == int(i)) add_metric(d, kCertifiedBeams, 1);
    }
  }
}

// Half-open containment: a point on an edge belongs to the polygon only if the
// edge is "owned" (rising, or horizontal running in -x), so a tessellated
// sheet counts once on shared edges (event_kernels.py:95-148).
// F is the predicate form (edp_filtered.cuh): the side of x against each
// edge is the binary64 sign (0) or the exact one (1, 2; tallied in t by 2).
template <int F>
__device__ inline bool contains_flat(const Dev &d, int source, V2 x, Tally &t) {
  const V2 *p = d.src_v + int64_t(kSourceVertices) * source;
  const int n = d.src_n[source];
  for (int j = 0; j < n; ++j) {
    V2 a = p[j], b = p[(j + 1) % n];
    int stage = 0;
    const int s = side_sign<F>(a, b, x, stage);
    if constexpr (F == 2) t.add(stage);
    bool owned = b.y > a.y || (b.y == a.y && b.x < a.x);
    if (s < 0 || (s == 0 && !owned)) return false;
  }
  return n > 0;
}

// contains_flat's answer (0 or 1) in forms 0-3; in the filter-only form 4,
// pred::kUndecided when no edge's filtered sign excludes x and some edge's
// filter left its sign undecided (the exact pass then decides: the answer is
// the AND over the edges, so the order of the tests does not matter).
template <int F>
__device__ inline int contains_form(const Dev &d, int source, V2 x, Tally &t) {
  if constexpr (F != 4) {
    return contains_flat<F>(d, source, x, t) ? 1 : 0;
  } else {
    const V2 *p = d.src_v + int64_t(kSourceVertices) * source;
    const int n = d.src_n[source];
    bool undecided = false;
    for (int j = 0; j < n; ++j) {
      V2 a = p[j], b = p[(j + 1) % n];
      int stage = 0;
      const int s = side_sign<F>(a, b, x, stage);
      if (s == pred::kUndecided) {
        undecided = true;
        continue;
      }
      bool owned = b.y > a.y || (b.y == a.y && b.x < a.x);
      if (s < 0 || (s == 0 && !owned)) return 0;
    }
    return undecided ? pred::kUndecided : (n > 0 ? 1 : 0);
  }
}

// Leave a containment test of ray group `group` against `source` to the exact
// pass (k_ray_exact); the pool's overflow is a hit-pool overflow.
__device__ inline void defer_contains(const Dev &d, int group, int source) {
  const int k = atomicAdd(&d.sc[kRayDeferred], 1);
  if (k < d.ray_defer_cap)
    d.ray_defer[k] = make_int2(group, source);
  else
    set_error(d.status, kErrHits);
}

// ---------------------------------------------------------------- source grid
// Grid column (or row) of a window coordinate: floor(v G) clamped to the grid.
__device__ inline int ray_cell(double v, int g) {
  const double c = floor(v * double(g));
  return c < 0.0 ? 0 : c > double(g - 1) ? g - 1 : int(c);
}

// Cells of a source's box grown by 1e-6 (a ray's query box, x +- 2e-7 in
// binary32, meets the box only if the ray's point lies in this range); false
// for an empty box.
__device__ inline bool source_cells(const Dev &d, int s, int &cx0, int &cx1, int &cy0, int &cy1) {
  const float4 lo = d.src_lo[s], hi = d.src_hi[s];
  if (!(lo.x <= hi.x && lo.y <= hi.y)) return false;
  const int g = d.grid_size;
  cx0 = ray_cell(double(lo.x) - 1.0e-6, g);
  cx1 = ray_cell(double(hi.x) + 1.0e-6, g);
  cy0 = ray_cell(double(lo.y) - 1.0e-6, g);
  cy1 = ray_cell(double(hi.y) + 1.0e-6, g);
  return true;
}

__global__ void k_ray_grid_count(Dev d) {
  for (int64_t s = tid(); s < d.n; s += stride()) {
    int cx0, cx1, cy0, cy1;
    if (!source_cells(d, int(s), cx0, cx1, cy0, cy1)) continue;
    if ((cx1 - cx0 + 1) * (cy1 - cy0 + 1) > kRayCells) {
      d.ray_big[reserve(&d.sc[kRayBig], 1)] = int(s);
      continue;
    }
    for (int cy = cy0; cy <= cy1; ++cy)
      for (int cx = cx0; cx <= cx1; ++cx) atomicAdd(&d.ray_count[cy * d.grid_size + cx], 1);
  }
}

// Counting sort: ray_start is the scan of the counts; each listing takes a
// slot of its cell.  The grid serves the rays when few sources are big.
__global__ void k_ray_grid_fill(Dev d) {
  if (tid() == 0) d.sc[kRayGridOn] = d.sc[kRayBig] <= 64 ? 1 : 0;
  for (int64_t s = tid(); s < d.n; s += stride()) {
    int cx0, cx1, cy0, cy1;
    if (!source_cells(d, int(s), cx0, cx1, cy0, cy1)) continue;
    if ((cx1 - cx0 + 1) * (cy1 - cy0 + 1) > kRayCells) continue;
    for (int cy = cy0; cy <= cy1; ++cy)
      for (int cx = cx0; cx <= cx1; ++cx) {
        const int c = cy * d.grid_size + cx;
        d.ray_entries[d.ray_start[c] + atomicSub(&d.ray_count[c], 1) - 1] = int(s);
      }
  }
}

// Each source's leaf in the source hierarchy (the order of its binary walk).
__global__ void k_leaf_of(Dev d) {
  const int count = d.n;
  const int leaves = *d.source_tree.size;
  for (int64_t leaf = tid(); leaf < leaves; leaf += stride()) {
    const int s = d.source_tree.ids[leaf];
    if (s < count) d.leaf_of[s] = int(leaf);
  }
}

// Hits found by one thread, flushed to the shared pool with one reservation.
struct HitBuffer {
  static constexpr int kSize = kCandidatesPerPass;
  int source[kSize];
  double depth[kSize];
  int count = 0;

  __device__ void flush(const Dev &d, int group) {
    long long slot = reserve(&d.metrics[kRayHits], count);
    if (slot + count > d.cap.hits) {
      set_error(d.status, kErrHits);
    } else {
      for (int k = 0; k < count; ++k) {
        d.hit_depth[slot + k] = depth[k];
        d.hit_src[slot + k] = source[k];
        d.hit_group[slot + k] = group;
      }
    }
    count = 0;
  }
};

// One ray per group leader: up to kCandidatesPerPass sources, the rest of the
// traversal is queued for the persistent continuation (event_kernels.py:196-245).
template <int F>
__global__ void k_ray_hits(Dev d) {
  const int live = live_polygons(d);
  const int leaves = *d.source_tree.size;
  const bool grid = d.sc[kRayGridOn] != 0;
  long long groups = 0, tests = 0, heavy_rays = 0;
  HitBuffer hits;
  Tally contain;
  for (int64_t k = tid(); k < live; k += stride()) {
    if (d.status[kError] != 0) return;
    const int i = d.order[k];  // spatial order: neighbouring rays read neighbouring data
    if (d.groups[i] != i) continue;
    V2 x = d.samples[i];
    float4 lo = make_float4(lower_f(x.x - 2.0e-7), lower_f(x.y - 2.0e-7), -1.0e30f, 0.f);
    float4 hi = make_float4(upper_f(x.x + 2.0e-7), upper_f(x.y + 2.0e-7), 1.0e30f, 0.f);
    ++groups;
    if (grid) {
      // Every source whose box meets the query box is listed in the point's
      // cell (or among the big ones); the box test keeps exactly the
      // hierarchy's candidates, the whole ray in one pass.
      const int g = d.grid_size, c = ray_cell(x.y, g) * g + ray_cell(x.x, g);
      const int begin = d.ray_start[c], end = d.ray_start[c + 1], big = d.sc[kRayBig];
      int met = 0, last = -1, found = 0;
      for (int e = begin; e < end + big; ++e) {
        const int s = e < end ? d.ray_entries[e] : d.ray_big[e - end];
        if (!overlaps(d.src_lo[s], d.src_hi[s], lo, hi)) continue;
        ++met;
        last = max(last, d.leaf_of[s]);
        const int inside = contains_form<F>(d, s, x, contain);
        if (F == 4 && inside == pred::kUndecided) {
          defer_contains(d, i, s);
        } else if (inside) {
          hits.source[hits.count] = s;
          hits.depth[hits.count] = value(d.scores[s], x);
          ++found;
          if (++hits.count == HitBuffer::kSize) hits.flush(d, i);
        }
      }
      if (hits.count) hits.flush(d, i);
      d.group_counts[i] = found;
      tests += met;
      // The binary walk's primary pass would leave this ray unfinished.
      heavy_rays += met > kCandidatesPerPass || (met == kCandidatesPerPass && last != leaves - 1);
      continue;
    }
    int node = 1;
    for (int step = 0; step < kCandidatesPerPass; ++step) {
      int s;
      node = query_next(d.source_tree, leaves, lo, hi, node, 0, s);
      if (s < 0) break;
      ++tests;
      const int inside = contains_form<F>(d, s, x, contain);
      if (F == 4 && inside == pred::kUndecided) {
        defer_contains(d, i, s);
      } else if (inside) {
        hits.source[hits.count] = s;
        hits.depth[hits.count] = value(d.scores[s], x);
        ++hits.count;
      }
      if (node == 0) break;
    }
    d.group_counts[i] = hits.count;
    hits.flush(d, i);
    const bool heavy = node > 0;
    if (heavy)
      while (node < leaves) node *= 2;
    heavy_rays += heavy;
    int slot = reserve(&d.sc[kHeavyJobs], heavy ? 1 : 0);
    if (heavy) d.heavy_queries[slot] = make_int2(i, node);
  }
  count_add(&d.metrics[kRayGroups], groups);
  count_add(&d.metrics[kRayCandidateTests], tests);
  count_add(&d.metrics[kHeavyRayGroups], heavy_rays);
  if constexpr (F == 2) contain.flush(d, kPredContain);
}

// The continuation of the rays whose primary pass did not finish, one warp
// per ray (event_kernels.py:248-298).  The warp resumes the walk at the first
// leaf the primary pass did not reach and walks the rest of the source
// hierarchy 32 nodes at a time; each lane of a leaf batch takes one candidate,
// and the batch's hits go to the shared pool with one reservation.  The
// candidates, and so the hits, are those of the reference's disjoint-subtree
// continuation.
template <int F>
__global__ void __launch_bounds__(kBlock) k_heavy_hits(Dev d) {
  const unsigned full = 0xffffffffu;
  if (d.status[kError] != 0) return;
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int leaves = *d.source_tree.size;
  const long long jobs = d.sc[kHeavyJobs];
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  // Few rays share the GPU: split each one's rest into `parts` ranges of
  // whole leaf groups, about 32K warp tasks in all (event_kernels.py:248-298).
  int parts = 1;
  while (parts * 2LL * jobs <= 32768 && parts * 2 * 32 <= leaves) parts *= 2;
  const int width = leaves / parts;
  long long tests = 0;  // lane 0's tally
  Tally contain;
  for (int64_t task = tid() >> 5; task < jobs * parts; task += warps) {
    const int2 job = d.heavy_queries[task / parts];
    const int part = int(task % parts), end = (part + 1) * width;
    const int i = job.x;
    int cursor = job.y - leaves;  // job.y: the first leaf node left
    if (cursor >= end) continue;
    cursor = max(cursor, part * width);
    const V2 x = d.samples[i];
    const float4 lo = make_float4(lower_f(x.x - 2.0e-7), lower_f(x.y - 2.0e-7), -1.0e30f, 0.f);
    const float4 hi = make_float4(upper_f(x.x + 2.0e-7), upper_f(x.y + 2.0e-7), 1.0e30f, 0.f);
    WarpWalk w;
    walk_begin(w, d.source_tree, leaves, lo, hi, cursor, end);
    int budget = 0x7fffffff, first, resume, found = 0;
    unsigned batch;
    bool overflow = false;
    while (walk_next(w, d.source_tree, leaves, lo, hi, cursor, budget, batch, first, resume)) {
      tests += __popc(batch);
      bool hit = false;
      int s = 0;
      double depth = 0.0;
      if ((batch >> lane) & 1u) {
        s = __ldg(&d.source_tree.ids[first + lane]);
        const int inside = contains_form<F>(d, s, x, contain);
        if (F == 4 && inside == pred::kUndecided) {
          defer_contains(d, i, s);
        } else {
          hit = inside != 0;
        }
        if (hit) depth = value(d.scores[s], x);
      }
      const unsigned hits = __ballot_sync(full, hit);
      if (!hits) continue;
      const int count = __popc(hits);
      long long slot = 0;
      if (lane == 0)
        slot = static_cast<long long>(atomicAdd(
            reinterpret_cast<unsigned long long *>(&d.metrics[kRayHits]), (unsigned long long)count));
      slot = __shfl_sync(full, slot, 0);
      if (slot + count > d.cap.hits) {
        overflow = true;
      } else if (hit) {
        const long long at = slot + __popc(hits & below);
        d.hit_depth[at] = depth;
        d.hit_src[at] = s;
        d.hit_group[at] = i;
      }
      found += count;
    }
    if (lane == 0) {
      if (overflow) set_error(d.status, kErrHits);
      if (found) atomicAdd(&d.group_counts[i], found);
    }
  }
  if (lane == 0) add_metric(d, kRayCandidateTests, tests);
  if constexpr (F == 2) contain.flush(d, kPredContain);
}

// The exact pass over the containment tests the filter-only ray kernels left
// undecided: each hit joins its group's pool like the others (the group sort
// orders a group's hits whatever their slots).
__global__ void k_ray_exact(Dev d) {
  if (d.status[kError] != 0) return;
  const long long total = min(int64_t(d.sc[kRayDeferred]), d.ray_defer_cap);
  if (tid() == 0) d.metrics[kDeferredContainTests] = d.sc[kRayDeferred];
  Tally contain;
  for (int64_t k = tid(); k < total; k += stride()) {
    const int2 job = d.ray_defer[k];
    const V2 x = d.samples[job.x];
    if (!contains_flat<3>(d, job.y, x, contain)) continue;
    const long long slot = static_cast<long long>(atomicAdd(
        reinterpret_cast<unsigned long long *>(&d.metrics[kRayHits]), 1ull));
    if (slot < d.cap.hits) {
      d.hit_depth[slot] = value(d.scores[job.y], x);
      d.hit_src[slot] = job.y;
      d.hit_group[slot] = job.x;
    }
    atomicAdd(&d.group_counts[job.x], 1);
  }
}

__global__ void k_check_hits(Dev d) {
  long long total = d.metrics[kRayHits];
  if (total > d.cap.hits) set_error(d.status, kErrHits);
  d.sc[kLiveHits] = int(min(total, (long long)d.cap.hits));
  d.sc[kSortHits] = 0;
}

// Hits of one ray group are ordered by (depth, source) within the group.  A
// group holds one hit per source along its ray, so groups are as deep as the
// scene's depth complexity: up to kGroupSort hits are sorted by one thread in
// place; if any group is larger, every hit goes through the global stable
// radix passes instead (the order is the same either way).
constexpr int kGroupSort = 128;
// Groups deeper than this are sorted a warp each (k_group_sort_deep): one
// thread's insertion sort of a deep group held its warp's other lanes.
constexpr int kWarpSort = 32;

__global__ void k_group_sizes(Dev d) {
  const int live = live_polygons(d);
  bool large = false;
  for (int64_t i = tid(); i < live; i += stride()) large |= d.group_counts[i] > kGroupSort;
  if (__any_sync(0xffffffffu, large) && (threadIdx.x & 31) == 0) d.sc[kSortHits] = d.sc[kLiveHits];
}

// The condition of the global hit passes: some group is too deep for
// k_group_sort.
__global__ void k_sort_switch(Dev d, cudaGraphConditionalHandle handle) {
  cudaGraphSetConditional(handle, d.sc[kSortHits] != 0 ? 1u : 0u);
}

// Place each hit in its group's range (group_offsets is the scan of
// group_counts); the order inside a group is fixed by k_group_sort.
__global__ void k_hit_place(Dev d) {
  if (d.sc[kSortHits] != 0 || d.status[kError] != 0) return;
  const int live = d.sc[kLiveHits];
  for (int64_t h = tid(); h < live; h += stride()) {
    const int g = d.hit_group[h];
    d.hit_ids[d.group_offsets[g] + atomicAdd(&d.group_fill[g], 1)] = int(h);
  }
}

// Order each group's hits by (ordered depth bits, source): the order of the
// three stable radix passes below, whose keys are the same (a source is hit
// at most once per group, so no two hits of a group tie).
// The filtered forms (F > 0) order two hits by the exact sign of the
// difference of their sources' depth planes at the group's sample, equal
// depths by source: the order the binary64 keys give wherever rounding does
// not decide it.
// With filtered binary64 predicates the filter-only form (F = 4) sorts every
// group whose comparisons its filters decide and lists the others; form 3
// then sorts the listed groups (`deferred_pass`).
template <int F>
__global__ void k_group_sort(Dev d, int deferred_pass) {
  // After a hit-pool overflow the groups' counts exceed the hits stored.
  if (d.sc[kSortHits] != 0 || d.status[kError] != 0) return;
  const int live = deferred_pass ? d.sc[kSortDeferred] : live_polygons(d);
  if (deferred_pass && tid() == 0) d.metrics[kDeferredHitGroups] = live;
  Tally order;
  for (int64_t t = tid(); t < live; t += stride()) {
    const int64_t g = deferred_pass ? d.rank_defer[t] : t;
    const int k = d.group_counts[g];
    if (k < 2) continue;
    if (!deferred_pass && k > kWarpSort) {  // sorted a warp each by k_group_sort_deep
      d.deep_groups[atomicAdd(&d.sc[kDeepGroups], 1)] = int(g);
      continue;
    }
    int *ids = d.hit_ids + d.group_offsets[g];
    int src[kGroupSort], id[kGroupSort];
    if constexpr (F == 0) {
      unsigned long long key[kGroupSort];
      for (int j = 0; j < k; ++j) {
        const int h = ids[j];
        const unsigned long long kj = ordered_bits(d.hit_depth[h]);
        const int sj = d.hit_src[h];
        int m = j - 1;
        while (m >= 0 && (key[m] > kj || (key[m] == kj && src[m] > sj))) {
          key[m + 1] = key[m];
          src[m + 1] = src[m];
          id[m + 1] = id[m];
          --m;
        }
        key[m + 1] = kj;
        src[m + 1] = sj;
        id[m + 1] = h;
      }
    } else {
      const V2 x = d.samples[g];
      double depth[kGroupSort];
      // First the order of the binary64 keys (cheap comparisons), which the
      // exact order differs from only where rounding decides: the exact
      // insertion sort below then meets an almost sorted sequence and makes
      // about k exact comparisons instead of k^2 / 4.  Its result is the
      // exact order whatever the starting sequence.
      for (int j = 0; j < k; ++j) {
        const int h = ids[j];
        const double zj = d.hit_depth[h];
        const int sj = d.hit_src[h];
        int m = j - 1;
        while (m >= 0 && (depth[m] > zj || (depth[m] == zj && src[m] > sj))) {
          depth[m + 1] = depth[m];
          src[m + 1] = src[m];
          id[m + 1] = id[m];
          --m;
        }
        depth[m + 1] = zj;
        src[m + 1] = sj;
        id[m + 1] = h;
      }
      bool undecided = false;
      for (int j = 1; j < k && !undecided; ++j) {
        const double zj = depth[j];
        const int sj = src[j], h = id[j];
        const Plane pj = d.scores[sj];
        int m = j - 1;
        while (m >= 0) {
          int stage = 0;
          const int o = order_sign<F>(d.scores[src[m]], depth[m], pj, zj, x, stage);
          if constexpr (F == 2) order.add(stage);
          if (F == 4 && o == pred::kUndecided) {
            undecided = true;
            break;
          }
          if (!(o > 0 || (o == 0 && src[m] > sj))) break;
          depth[m + 1] = depth[m];
          src[m + 1] = src[m];
          id[m + 1] = id[m];
          --m;
        }
        depth[m + 1] = zj;
        src[m + 1] = sj;
        id[m + 1] = h;
      }
      if (undecided) {  // form 4: the exact pass sorts this group
        d.rank_defer[atomicAdd(&d.sc[kSortDeferred], 1)] = int(g);
        continue;
      }
    }
    for (int j = 0; j < k; ++j) ids[j] = id[j];
  }
  if constexpr (F == 2) order.flush(d, kPredOrder);
}

// The groups of more than kWarpSort (and at most kGroupSort) hits, a warp
// each.  The group's hits and their sources' planes go to shared memory; each
// lane counts, for each of its hits, the hits whose (ordered binary64 depth
// bits, source) key comes first, which is the hit's place in key order (the
// keys are distinct: one hit per source).  That is the plain form's order.
// The filtered forms order by the exact sign of the plane difference at the
// group's sample, then by source; they check the key order's neighbours with
// that comparison (a total order is sorted when its neighbours are), and a
// group that fails the check, or meets an undecided filter (F = 4), is sorted
// by insertion on lane 0 (forms 1-3) or goes to the exact pass's list (4).
template <int F>
__global__ void __launch_bounds__(kBlock) k_group_sort_deep(Dev d) {
  if (d.sc[kSortHits] != 0 || d.status[kError] != 0) return;
  constexpr int kWarpsPerBlock = kBlock / 32;
  __shared__ double s_depth[kWarpsPerBlock][kGroupSort];
  __shared__ Plane s_plane[kWarpsPerBlock][kGroupSort];
  __shared__ int s_src[kWarpsPerBlock][kGroupSort], s_id[kWarpsPerBlock][kGroupSort];
  __shared__ unsigned char s_order[kWarpsPerBlock][kGroupSort];  // key order -> hit
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int deep = d.sc[kDeepGroups];
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  Tally order;
  for (int64_t t = tid() >> 5; t < deep; t += warps) {
    const int g = d.deep_groups[t];
    const int k = d.group_counts[g];
    int *ids = d.hit_ids + d.group_offsets[g];
    for (int j = lane; j < k; j += 32) {
      const int h = ids[j];
      s_depth[w][j] = d.hit_depth[h];
      s_src[w][j] = d.hit_src[h];
      if constexpr (F != 0) s_plane[w][j] = d.scores[s_src[w][j]];
      s_id[w][j] = h;
    }
    __syncwarp();
    for (int j = lane; j < k; j += 32) {
      const unsigned long long kj = ordered_bits(s_depth[w][j]);
      const int sj = s_src[w][j];
      int before = 0;
      for (int i = 0; i < k; ++i) {
        const unsigned long long ki = ordered_bits(s_depth[w][i]);
        before += ki < kj || (ki == kj && s_src[w][i] < sj);
      }
      s_order[w][before] = (unsigned char)j;
    }
    __syncwarp();
    bool sorted = true, undecided = false;
    if constexpr (F != 0) {
      const V2 x = d.samples[g];
      for (int m = lane; m + 1 < k; m += 32) {
        const int a = s_order[w][m], b = s_order[w][m + 1];
        int stage = 0;
        const int o = order_sign<F>(s_plane[w][a], s_depth[w][a], s_plane[w][b], s_depth[w][b],
                                    x, stage);
        if constexpr (F == 2) order.add(stage);
        if (F == 4 && o == pred::kUndecided)
          undecided = true;
        else if (!(o < 0 || (o == 0 && s_src[w][a] < s_src[w][b])))
          sorted = false;
      }
      undecided = __any_sync(0xffffffffu, undecided);
      sorted = __all_sync(0xffffffffu, sorted);
    }
    if constexpr (F == 4) {
      if (undecided || !sorted) {  // the exact pass sorts this group
        if (lane == 0) d.rank_defer[atomicAdd(&d.sc[kSortDeferred], 1)] = g;
        __syncwarp();
        continue;
      }
    } else if constexpr (F != 0) {
      if (!sorted && lane == 0) {  // rare: lane 0 sorts the key order exactly
        const V2 x = d.samples[g];
        unsigned char *o = s_order[w];
        for (int j = 1; j < k; ++j) {
          const int b = o[j];
          int m = j - 1;
          while (m >= 0) {
            const int a = o[m];
            int stage = 0;
            const int c = order_sign<F>(s_plane[w][a], s_depth[w][a], s_plane[w][b],
                                        s_depth[w][b], x, stage);
            if constexpr (F == 2) order.add(stage);
            if (!(c > 0 || (c == 0 && s_src[w][a] > s_src[w][b]))) break;
            o[m + 1] = o[m];
            --m;
          }
          o[m + 1] = (unsigned char)b;
        }
      }
      __syncwarp();
    }
    for (int m = lane; m < k; m += 32) ids[m] = s_id[w][s_order[w][m]];
    __syncwarp();
  }
  if constexpr (F == 2) order.flush(d, kPredOrder);
}

// Keys of the three stable passes that order hits by (group, depth, source)
// (event_kernels.py:313-339, events.py:701-718).
__global__ void k_hit_keys(Dev d, int stage) {
  const int live = d.sc[kSortHits];
  for (int64_t i = tid(); i < live; i += stride()) {
    int h = stage == 0 ? int(i) : d.hit_ids[i];
    if (stage == 0) d.hit_ids[i] = int(i);
    unsigned long long key;
    if (stage == 0)
      key = static_cast<unsigned>(d.hit_src[h]);
    else if (stage == 1)
      key = ordered_bits(d.hit_depth[h]);
    else
      key = static_cast<unsigned>(d.hit_group[h]);
    d.hkeys[i] = key;
  }
}

// Rank = number of the group's hits nearer than the representative's source
// at this polygon's sample, equal depths ordered by source index
// (event_kernels.py:342-385).
// The filtered forms search with the exact order of k_group_sort when the
// groups were sorted there, and with the binary64 order after the radix
// passes (groups deeper than kGroupSort), matching the order searched.
// With filtered binary64 predicates the filter-only form (F = 4) places every
// polygon whose search its filters decide and lists the others; form 3 then
// places the listed ones (`deferred_pass`).
template <int F>
__global__ void k_assign(Dev d, int deferred_pass) {
  const int live = deferred_pass ? d.sc[kAssignDeferred] : live_polygons(d);
  if (deferred_pass && tid() == 0) d.metrics[kDeferredPolygons] = live;
  const bool exact = F != 0 && d.sc[kSortHits] == 0;
  Tally order;
  for (int64_t t = tid(); t < live; t += stride()) {
    if (d.status[kError] != 0) return;
    const int64_t i = deferred_pass ? d.rank_defer[t] : t;
    int source = d.out_src[d.reps[i]];
    V2 x = d.samples[i];
    const Plane ps = d.scores[source];
    double z = value(ps, x);
    int g = d.groups[i];
    int low = 0, high = d.group_counts[g];
    const int *ids = d.hit_ids + d.group_offsets[g];
    bool undecided = false;
    while (low < high) {
      int mid = (low + high) / 2;
      int h = ids[mid];
      int hs = d.hit_src[h];
      const Plane ph = d.scores[hs];
      double hz = value(ph, x);
      bool nearer;
      if (exact) {
        int stage = 0;
        const int o = order_sign<F>(ph, hz, ps, z, x, stage);
        if constexpr (F == 2) order.add(stage);
        if (F == 4 && o == pred::kUndecided) {
          undecided = true;
          break;
        }
        nearer = o < 0 || (o == 0 && hs < source);
      } else {
        nearer = hz < z || (hz == z && hs < source);
      }
      if (nearer)
        low = mid + 1;
      else
        high = mid;
    }
    if (undecided) {  // form 4: the exact pass places this polygon
      d.rank_defer[atomicAdd(&d.sc[kAssignDeferred], 1)] = int(i);
      continue;
    }
    d.out_layer[i] = low;
    if (low >= d.limit) {
      if (d.all_layers)
        set_error(d.status, kErrLayers);
      else
        d.out_n[i] = 0;
    } else {
      atomicMax(&d.status[kLayers], low + 1);
    }
  }
  if constexpr (F == 2) order.flush(d, kPredOrder);
}

__global__ void k_layers_reset(Dev d) { d.status[kLayers] = 0; }

// ---------------------------------------------------------------- merging
// Optional convex coalescing (components.py:274-395).  A matched pair of
// patch edges whose polygons share source and layer proposes a merge when the
// union stays convex at both joint vertices; every polygon keeps the smallest
// proposing edge, and a pair merges when both of its polygons chose it.  Each
// polygon is in at most one merge, so merges never touch the same slot.
__global__ void k_merge_propose(Dev d) {
  const int total = d.sc[kPatchEdges];
  for (int64_t t = tid(); t < total; t += stride()) {
    if (d.status[kError] != 0) return;
    const int other = d.partners[t];
    if (other <= t) continue;
    const int2 ta = d.tasks[t], tb = d.tasks[other];
    if (d.out_src[ta.x] != d.out_src[tb.x] || d.out_layer[ta.x] != d.out_layer[tb.x]) continue;
    const int na = d.out_n[ta.x], nb = d.out_n[tb.x];
    if (na < 3 || nb < 3 || na + nb - 2 > kMaxVertices) continue;
    const V2 *a = d.out_v + int64_t(kMaxVertices) * ta.x;
    const V2 *b = d.out_v + int64_t(kMaxVertices) * tb.x;
    const V2 u = a[ta.y], v = b[tb.y];
    if (cross(a[(ta.y + na - 1) % na], u, b[(tb.y + 2) % nb]) >= 0.0 &&
        cross(b[(tb.y + nb - 1) % nb], v, a[(ta.y + 2) % na]) >= 0.0) {
      atomicMin(&d.merge_choice[ta.x], int(t));
      atomicMin(&d.merge_choice[tb.x], int(t));
    }
  }
}

// The joined ring runs over all of a's vertices from the end of the shared
// edge, then b's vertices but the shared two; exactly collinear vertices are
// dropped.  The merged polygon replaces a, and b is emptied.
__global__ void k_merge(Dev d) {
  const int total = d.sc[kPatchEdges];
  long long merged = 0;
  for (int64_t t = tid(); t < total; t += stride()) {
    if (d.status[kError] != 0) break;
    const int other = d.partners[t];
    if (other <= t) continue;
    const int2 ta = d.tasks[t], tb = d.tasks[other];
    if (d.merge_choice[ta.x] != t || d.merge_choice[tb.x] != t) continue;
    V2 *a = d.out_v + int64_t(kMaxVertices) * ta.x;
    const V2 *b = d.out_v + int64_t(kMaxVertices) * tb.x;
    const int na = d.out_n[ta.x], nb = d.out_n[tb.x];
    V2 joined[kMaxVertices];
    int m = 0;
    for (int j = 0; j < na; ++j) joined[m++] = a[(ta.y + 1 + j) % na];
    for (int j = 0; j < nb - 2; ++j) joined[m++] = b[(tb.y + 2 + j) % nb];
    int kept = 0;
    V2 q[kMaxVertices];
    for (int j = 0; j < m; ++j) {
      const V2 x = joined[j];
      if (cross(joined[(j + m - 1) % m], x, joined[(j + 1) % m]) != 0.0) q[kept++] = x;
    }
    if (kept < 3) continue;
    for (int j = 0; j < kept; ++j) a[j] = q[j];
    d.out_n[ta.x] = kept;
    d.out_n[tb.x] = 0;
    ++merged;
  }
  count_add(&d.metrics[kMergedPolygons], merged);
}

__global__ void k_merge_counts(Dev d) {
  const int live = live_polygons(d);
  for (int64_t i = tid(); i < live; i += stride())
    d.counts[i] = d.status[kError] == 0 && d.out_n[i] > 0 ? 1 : 0;
}

// Live polygons, compacted in slot order into the copy and back
// (components.py:356-395).
__global__ void k_merge_compact(Dev d) {
  const int live = live_polygons(d);
  for (int64_t i = tid(); i < live; i += stride()) {
    if (d.status[kError] != 0 || d.out_n[i] <= 0) continue;
    const int slot = d.offsets[i], n = d.out_n[i];
    const V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    V2 *q = d.merged_v + int64_t(kMaxVertices) * slot;
    for (int j = 0; j < n; ++j) q[j] = p[j];
    d.merged_n[slot] = n;
    d.merged_src[slot] = d.out_src[i];
    d.merged_layer[slot] = d.out_layer[i];
  }
}

__global__ void k_merge_restore(Dev d) {
  if (d.status[kError] != 0) return;
  const int kept = d.sc[kMergedLive];
  for (int64_t i = tid(); i < kept; i += stride()) {
    const int n = d.merged_n[i];
    const V2 *q = d.merged_v + int64_t(kMaxVertices) * i;
    V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    for (int j = 0; j < n; ++j) p[j] = q[j];
    d.out_n[i] = n;
    d.out_src[i] = d.merged_src[i];
    d.out_layer[i] = d.merged_layer[i];
  }
}

__global__ void k_merge_finish(Dev d) {
  if (d.status[kError] != 0) return;
  d.status[kPolygons] = d.sc[kMergedLive];
  d.sc[kLivePolygons] = d.sc[kMergedLive];
}

unsigned blocks(int64_t n) {
  int64_t g = ceil_div(n > 0 ? n : 1, kBlock);
  return unsigned(g < 148 * 16 ? g : 148 * 16);
}

int bits_for(int64_t n) {
  int b = 1;
  while ((int64_t(1) << b) < n + 1) ++b;
  return b;
}

}  // namespace

cudaError_t stage_rank(const Dev &d, SortScratch &s, cudaStream_t st) {
  const int64_t R = d.cap.regions, E = d.cap.vertices;
  k_rank_begin<<<1, 1, 0, st>>>(d);
  note_launch();
  EDP_CHECK(order_polygons(d, false, s, st));
  k_polygon_init<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_ORDER, st));
  const bool connected = d.propagate_ranks || d.merge_regions;
  if (connected) {
    EDP_CHECK(scan_exclusive(d.counts, d.offsets, d.sc + kLivePolygons, R, d.sc + kPatchEdges, s, st));
    k_check_edges<<<1, 1, 0, st>>>(d);
    note_launch();
    k_patch_edges<<<blocks(R), kBlock, 0, st>>>(d);
    note_launch();
    EDP_CHECK(cudaMemsetAsync(d.edge_hash, 0xff, sizeof(int) * (int64_t(d.edge_hash_mask) + 1), st));
    k_match_edges<<<blocks(E), kBlock, 0, st>>>(d);
    note_launch();
    if (d.propagate_ranks) {
      const int64_t cells = int64_t(d.grid_size) * d.grid_size;
      EDP_CHECK(cudaMemsetAsync(d.seg_count, 0, sizeof(int) * cells, st));
      k_seg_grid_count<<<blocks(kSourceVertices * int64_t(d.n)), kBlock, 0, st>>>(d);
      note_launch();
      EDP_CHECK(scan_exclusive(d.seg_count, d.seg_start, d.sc + kRayGridCells, cells,
                               d.seg_start + cells, s, st));
      k_seg_grid_fill<<<blocks(kSourceVertices * int64_t(d.n)), kBlock, 0, st>>>(d);
      note_launch();
      k_connect<<<blocks(E), kBlock, 0, st>>>(d);
    }
    note_launch();
  }
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_CONNECTIVITY, st));
  k_roots<<<blocks(R), kBlock, 0, st>>>(d, d.propagate_ranks ? 1 : 0);
  note_launch();
  k_samples<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_SAMPLES, st));
  EDP_CHECK(cudaMemsetAsync(d.sample_table, 0xff, sizeof(int) * (int64_t(d.sample_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.sample_min, 0x7f, sizeof(int) * (int64_t(d.sample_mask) + 1), st));
  k_cells_reset<<<kCells / 128, 128, 0, st>>>(d);
  note_launch();
  k_group_insert<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  k_group_resolve<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_QUERY_GROUPS, st));
  if (d.share_regions) {
    k_certify<<<kCells * 32 / kBlock, kBlock, 0, st>>>(d);
    note_launch();
    k_certify_heavy<<<kHeavyBlocks, kHeavyBlock, 0, st>>>(d);
    note_launch();
    k_apply_cells<<<blocks(R), kBlock, 0, st>>>(d);
    note_launch();
  }
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_CERTIFY, st));
  {
    const int64_t cells = int64_t(d.grid_size) * d.grid_size;
    EDP_CHECK(cudaMemsetAsync(d.ray_count, 0, sizeof(int) * cells, st));
    k_leaf_of<<<blocks(d.n), kBlock, 0, st>>>(d);
    note_launch();
    k_ray_grid_count<<<blocks(d.n), kBlock, 0, st>>>(d);
    note_launch();
    EDP_CHECK(scan_exclusive(d.ray_count, d.ray_start, d.sc + kRayGridCells, cells,
                             d.ray_start + cells, s, st));
    k_ray_grid_fill<<<blocks(d.n), kBlock, 0, st>>>(d);
    note_launch();
  }
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_RAY_GRID, st));
  // Filtered binary64 predicates: the filter-only kernels, then exact passes
  // over what their filters left undecided (same results as form 3 alone).
  const bool split_exact = d.predicates == 3;
  if (split_exact) {
    k_ray_hits<4><<<blocks(R), kBlock, 0, st>>>(d);
  } else {
    EDP_LAUNCH_FORM(d.predicates, k_ray_hits, blocks(R), kBlock, st, d);
  }
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_RAY_PRIMARY, st));
  if (split_exact) {
    k_heavy_hits<4><<<148 * 16, kBlock, 0, st>>>(d);
    note_launch();
    k_ray_exact<<<148 * 4, kBlock, 0, st>>>(d);
  } else {
    EDP_LAUNCH_FORM(d.predicates, k_heavy_hits, 148 * 16, kBlock, st, d);
  }
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_RAY_HEAVY, st));
  EDP_CHECK(scan_exclusive(d.group_counts, d.group_offsets, d.sc + kLivePolygons, R, nullptr, s, st));
  k_check_hits<<<1, 1, 0, st>>>(d);
  note_launch();
  k_group_sizes<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  // Global passes: over all hits when some group is large, else over none.
  // In a captured graph they sit in a conditional IF node, so an extraction
  // whose groups all sort in k_group_sort launches none of their 40-odd
  // kernels; run eagerly, they take their count (zero) from the device.
  cudaStream_t radix = st;
  const bool branch = d.use_handle && d.aux_stream;
  if (branch) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    EDP_CHECK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphConditionalHandle handle;
    EDP_CHECK(cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
    k_sort_switch<<<1, 1, 0, st>>>(d, handle);
    note_launch();
    EDP_CHECK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams &params = *reinterpret_cast<cudaGraphNodeParams *>(raw);
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeIf;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    EDP_CHECK(cudaGraphAddNode(&node, g, deps, ndeps, &params));
    EDP_CHECK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    EDP_CHECK(cudaStreamBeginCaptureToGraph(d.aux_stream, params.conditional.phGraph_out[0],
                                            nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    radix = d.aux_stream;
  }
  const int pass_bits[3] = {bits_for(d.n), 64, bits_for(R)};
  const int64_t body_first = launch_count();
  cudaError_t sorted = cudaSuccess;
  for (int stage = 0; stage < 3 && sorted == cudaSuccess; ++stage) {
    k_hit_keys<<<blocks(d.cap.hits), kBlock, 0, radix>>>(d, stage);
    note_launch();
    sorted = sort_pairs_u64(reinterpret_cast<uint64_t *>(d.hkeys),
                            reinterpret_cast<uint64_t *>(d.hkeys_tmp), d.hit_ids, d.hit_ids_tmp,
                            d.sc + kSortHits, d.cap.hits, pass_bits[stage], s, radix);
  }
  if (branch) {
    cudaGraph_t body = nullptr;
    cudaError_t end = cudaStreamEndCapture(d.aux_stream, &body);
    EDP_CHECK(sorted);
    EDP_CHECK(end);
    forget_launches(launch_count() - body_first);
  }
  EDP_CHECK(sorted);
  EDP_CHECK(cudaMemsetAsync(d.group_fill, 0, sizeof(int) * R, st));
  k_hit_place<<<blocks(d.cap.hits), kBlock, 0, st>>>(d);
  note_launch();
  if (split_exact) {
    k_group_sort<4><<<blocks(R), kBlock, 0, st>>>(d, 0);
    note_launch();
    k_group_sort_deep<4><<<148 * 8, kBlock, 0, st>>>(d);
    note_launch();
    k_group_sort<3><<<148 * 4, kBlock, 0, st>>>(d, 1);
  } else {
    EDP_LAUNCH_FORM(d.predicates, k_group_sort, blocks(R), kBlock, st, d, 0);
    note_launch();
    EDP_LAUNCH_FORM(d.predicates, k_group_sort_deep, 148 * 8, kBlock, st, d);
  }
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_HIT_SORT, st));
  k_layers_reset<<<1, 1, 0, st>>>(d);
  note_launch();
  if (split_exact) {
    k_assign<4><<<blocks(R), kBlock, 0, st>>>(d, 0);
    note_launch();
    k_assign<3><<<148 * 4, kBlock, 0, st>>>(d, 1);
  } else {
    EDP_LAUNCH_FORM(d.predicates, k_assign, blocks(R), kBlock, st, d, 0);
  }
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_ASSIGN, st));
  if (d.merge_regions) {
    EDP_CHECK(cudaMemsetAsync(d.merge_choice, 0x7f, sizeof(int) * R, st));
    k_merge_propose<<<blocks(E), kBlock, 0, st>>>(d);
    note_launch();
    k_merge<<<blocks(E), kBlock, 0, st>>>(d);
    note_launch();
    k_merge_counts<<<blocks(R), kBlock, 0, st>>>(d);
    note_launch();
    EDP_CHECK(scan_exclusive(d.counts, d.offsets, d.sc + kLivePolygons, R, d.sc + kMergedLive, s, st));
    k_merge_compact<<<blocks(R), kBlock, 0, st>>>(d);
    note_launch();
    k_merge_restore<<<blocks(R), kBlock, 0, st>>>(d);
    note_launch();
    k_merge_finish<<<1, 1, 0, st>>>(d);
    note_launch();
  }
  EDP_CHECK(stage_mark(EDP_STAGE_RANK_MERGE, st));
  return cudaGetLastError();
}

}  // namespace edp

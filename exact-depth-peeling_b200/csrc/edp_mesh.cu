// Mesh stage: boundary vertex gathering and deduplication, the layered point
// grid (or, for very deep scenes, the layered point hierarchy), per-polygon
// noding, centroid-fan triangulation and world lifting
// (warp_peel/kernels.py:941-1204, events.py:720-780).
#include "../../include/edp.h"
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kBlock = 128;
constexpr int kMaxEdgeVertices = 128;  // edge noding capacity (solver.py:140-143)

__device__ inline int64_t tid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ inline int64_t stride() { return int64_t(gridDim.x) * blockDim.x; }

// Boundary vertex slots follow the polygons' (layer, Morton) order, so the
// copies of one point, which neighbouring polygons share, meet the point table
// close together in time.
__global__ void k_mesh_counts(Dev d) {
  const int live = d.sc[kLivePolygons];
  for (int64_t k = tid(); k < live; k += stride())
    d.counts[k] = d.status[kError] == 0 ? d.out_n[d.order[k]] : 0;
}

__global__ void k_mesh_check(Dev d) {
  d.sc[kUniqueVertices] = 0;
  int total = d.sc[kLiveVertices];
  d.status[kBoundaryVertices] = total;
  if (int64_t(total) > d.cap.vertices) {
    set_error(d.status, kErrVertices);
    d.sc[kLiveVertices] = int(d.cap.vertices);
  }
}

// Boundary vertices with their layer, one slot per polygon vertex
// (kernels.py:953-991, event_kernels.py:504-516).
__global__ void k_scatter(Dev d) {
  const int live = d.sc[kLivePolygons];
  for (int64_t k = tid(); k < live; k += stride()) {
    if (d.status[kError] != 0) return;
    const int i = d.order[k];
    const V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    const int layer = d.out_layer[i];
    const int64_t base = d.offsets[k];
    const int n = int(min(int64_t(d.out_n[i]), d.cap.vertices - base));
    for (int j = 0; j < n; ++j) {
      d.bverts[base + j] = p[j];
      d.blayers[base + j] = layer;
    }
  }
}

// Grid column (or row) of a window coordinate: floor(v G) clamped to the
// grid.  Monotone in v, so a query interval's cells hold every point inside it.
__device__ inline int grid_cell(double v, int g) {
  const double c = floor(v * double(g));
  return c < 0.0 ? 0 : c > double(g - 1) ? g - 1 : int(c);
}

// The grid serves this extraction when it has a row for every layer;
// otherwise the point hierarchy does.
__global__ void k_grid_begin(Dev d) {
  const int layers = d.status[kLayers];
  const bool on = d.status[kError] == 0 && layers <= d.grid_layers;
  d.sc[kGridOn] = on ? 1 : 0;
  d.sc[kGridCells] = on ? int(int64_t(layers) * d.point_grid * d.point_grid) : 0;
}

// Zero the point counts of the cells this extraction uses.
__global__ void k_grid_clear(Dev d) {
  const int cells = d.sc[kGridCells];
  for (int64_t c = tid(); c < cells; c += stride()) d.cell_count[c] = 0;
}

__global__ void k_tree_points(Dev d) {
  d.sc[kTreePoints] = d.sc[kGridOn] ? 0 : d.sc[kUniqueVertices];
}

// Counting sort of the distinct points by (layer, cell): the scan of the
// counts gives each cell's start, and each point takes a slot of its cell.
__global__ void k_grid_scatter(Dev d) {
  if (!d.sc[kGridOn] || d.status[kError] != 0) return;
  const int total = d.sc[kUniqueVertices], g = d.point_grid;
  if (tid() == 0) d.cell_start[d.sc[kGridCells]] = total;
  for (int64_t u = tid(); u < total; u += stride()) {
    const V2 x = d.uverts[u];
    const int layer = int(d.pt_lo[u].z);
    const int64_t cell = (int64_t(layer) * g + grid_cell(x.y, g)) * g + grid_cell(x.x, g);
    const int slot = atomicSub(&d.cell_count[cell], 1) - 1;
    d.grid_pts[d.cell_start[cell] + slot] = x;
  }
}

// Each distinct (layer, point) enters the point hierarchy once: a vertex
// shared by several patches would otherwise be a candidate of every query
// several times over.  One thread per boundary vertex inserts it into an
// open-addressing table keyed by its bits and layer; the first slot to claim
// an entry adds the point.
__global__ void k_unique_points(Dev d) {
  if (d.status[kError] != 0) return;
  const int total = d.sc[kLiveVertices];
  for (int64_t slot = tid(); slot < total; slot += stride()) {
    const V2 x = d.bverts[slot];
    const int layer = d.blayers[slot];
    uint64_t h = mix64(mix64(key_bits(x.x)) ^ key_bits(x.y)) ^ mix64(uint64_t(layer) + 7ull);
    uint32_t probe = uint32_t(h) & uint32_t(d.point_mask);
    bool fresh = false;
    for (int k = 0; k <= d.point_mask; ++k) {
      const int cur = atomicCAS(&d.point_table[probe], -1, int(slot));
      if (cur == -1) {
        fresh = true;
        break;
      }
      if (d.bverts[cur] == x && d.blayers[cur] == layer) break;
      probe = (probe + 1) & uint32_t(d.point_mask);
    }
    const int u = reserve(&d.sc[kUniqueVertices], fresh ? 1 : 0);
    if (fresh && d.sc[kGridOn]) {
      const int g = d.point_grid;
      atomicAdd(&d.cell_count[(int64_t(layer) * g + grid_cell(x.y, g)) * g + grid_cell(x.x, g)], 1);
    }
    if (fresh) {
      d.uverts[u] = x;
      d.pt_lo[u] = make_float4(__double2float_rd(x.x - 2.0e-7), __double2float_rd(x.y - 2.0e-7),
                               float(layer), 0.f);
      d.pt_hi[u] = make_float4(__double2float_ru(x.x + 2.0e-7), __double2float_ru(x.y + 2.0e-7),
                               float(layer), 0.f);
    }
  }
}

// Sort key of each live output polygon: the Morton code of its box centre
// (the 15-bit-per-axis code of the hierarchies, kernels.py:67-91, cut to 12
// bits per axis), below its layer when `layered`.
__global__ void k_order_keys(Dev d, int layered) {
  const int live = d.sc[kLivePolygons];
  for (int64_t i = tid(); i < live; i += stride()) {
    const V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    const int n = min(max(d.out_n[i], 1), kMaxVertices);
    double lx = p[0].x, ly = p[0].y, hx = p[0].x, hy = p[0].y;
    for (int j = 1; j < n; ++j) {
      lx = fmin(lx, p[j].x); ly = fmin(ly, p[j].y);
      hx = fmax(hx, p[j].x); hy = fmax(hy, p[j].y);
    }
    const float cx = fminf(fmaxf(float(0.5 * (lx + hx)), 0.f), 1.f);
    const float cy = fminf(fmaxf(float(0.5 * (ly + hy)), 0.f), 1.f);
    const uint32_t x = uint32_t(int(cx * 32767.0f)), y = uint32_t(int(cy * 32767.0f));
    // 12 bits per axis (a 4096 x 4096 grid) are plenty for locality.
    uint64_t key = (part1by1(x) | (part1by1(y) << 1)) >> 6;
    if (layered) key |= uint64_t(uint32_t(d.out_layer[i]) & 0xffffu) << 24;
    d.order_keys[i] = key;
    d.order[i] = int(i);
  }
}

// World position of a window point on a source plane (kernels.py:994-1006).
__device__ inline void lift(const Dev &d, V2 x, const Plane &s, double *w) {
  const double *st = d.settings, *m = d.inverse;
  double u = st[0] + x.x * (st[2] - st[0]);
  double v = st[1] + x.y * (st[3] - st[1]);
  double z = value(s, x);
  if (st[4] != 0.0) {
    z = -1.0 / z;
    u *= z;
    v *= z;
  }
  for (int r = 0; r < 3; ++r) w[r] = m[4 * r] * u + m[4 * r + 1] * v + m[4 * r + 2] * z + m[4 * r + 3];
}

// Node every edge of one output polygon against the same-layer boundary
// vertices lying on it (collinear within EPS, strictly inside the edge), then
// emit the polygon's centroid fan with the split points, lifted to world
// space (kernels.py:1009-1125).  One point-hierarchy query per polygon (its
// box contains every edge's box) replaces the reference's query per edge; the
// acceptance test and therefore the triangles are the same.
constexpr int kPolygonSplits = 256;  // split points buffered per polygon
// Candidate points x edges above which a polygon is noded by a whole warp
// (k_mesh_heavy) rather than by one thread, so that a few large polygons in
// dense cells do not hold 31 idle lanes of a warp: Dev::heavy_noding_work
// (1024 unless tuned).

// The centroid fan of polygon p (n vertices, centroid `center`) through its
// split points sorted by (edge, parameter).  Counts the fan triangles (signed
// doubled area above EPS^2: noded points 1e-13 apart can otherwise give
// slivers of area ~1e-19 whose orientation rounding decides; the reference
// tests |area|, kernels.py:1105), reserves their slots at once, then writes
// them with their world positions.
__device__ inline void emit_fan(const Dev &d, const V2 *p, int n, V2 center, int layer,
                                int source, const double *split_t,
                                const unsigned char *split_edge, int count) {
  int emitted = 0;
  for (int e = 0, k = 0; e < n; ++e) {
    const V2 a = p[e], dir = p[(e + 1) % n] - a;
    double previous = 0.0;
    V2 cursor = a;
    for (;;) {
      const bool last = !(k < count && split_edge[k] == e);
      const double following = last ? 1.0 : split_t[k++];
      if (following > previous + kEps) {
        const V2 next = a + following * dir;
        if (cross(center, cursor, next) > kEps * kEps) ++emitted;
        cursor = next;
        previous = following;
      }
      if (last) break;
    }
  }
  int slot = reserve(&d.status[kTriangles], emitted);
  if (int64_t(slot) + emitted > d.cap.triangles) {
    set_error(d.status, kErrTriangles);
    return;
  }
  const Plane sc = d.scores[source];
  double w_center[3];
  lift(d, center, sc, w_center);
  for (int e = 0, k = 0; e < n; ++e) {
    const V2 a = p[e], dir = p[(e + 1) % n] - a;
    double previous = 0.0;
    V2 cursor = a;
    double w_cursor[3];
    lift(d, cursor, sc, w_cursor);
    for (;;) {
      const bool last = !(k < count && split_edge[k] == e);
      const double following = last ? 1.0 : split_t[k++];
      if (following > previous + kEps) {
        const V2 next = a + following * dir;
        double w_next[3];
        lift(d, next, sc, w_next);
        if (cross(center, cursor, next) > kEps * kEps) {
          V2 *uv = d.tri_uv + 3 * int64_t(slot);
          double *w = d.tri_world + 9 * int64_t(slot);
          uv[0] = center;
          uv[1] = cursor;
          uv[2] = next;
          for (int c = 0; c < 3; ++c) {
            w[c] = w_center[c];
            w[3 + c] = w_cursor[c];
            w[6 + c] = w_next[c];
          }
          d.tri_src[slot] = source;
          d.tri_layer[slot] = layer;
          ++slot;
        }
        cursor = next;
        for (int c = 0; c < 3; ++c) w_cursor[c] = w_next[c];
        previous = following;
      }
      if (last) break;
    }
  }
}

__global__ void __launch_bounds__(kBlock, 8) k_mesh_polygons(Dev d, int edge_capacity) {
  const int live = d.sc[kLivePolygons];
  const int leaves = *d.point_tree.size;
  double split_t[kPolygonSplits];
  unsigned char split_edge[kPolygonSplits];
  for (int64_t k = tid(); k < live; k += stride()) {
    if (d.status[kError] != 0) return;
    const int64_t i = d.order[k];
    const V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    const int n = d.out_n[i];
    if (n < 3) continue;
    const int layer = d.out_layer[i], source = d.out_src[i];
    double lx = 1.0e30, ly = 1.0e30, hx = -1.0e30, hy = -1.0e30;
    V2 center = v2(0.0, 0.0);
    for (int j = 0; j < n; ++j) {
      lx = fmin(lx, p[j].x); ly = fmin(ly, p[j].y);
      hx = fmax(hx, p[j].x); hy = fmax(hy, p[j].y);
      center = center + p[j] / double(n);
    }
    const float4 lo = make_float4(__double2float_rd(lx - 2.0e-7), __double2float_rd(ly - 2.0e-7),
                                  float(layer), 0.f);
    const float4 hi = make_float4(__double2float_ru(hx + 2.0e-7), __double2float_ru(hy + 2.0e-7),
                                  float(layer), 0.f);
    // The grid cells meeting the polygon's box grown by 1e-9 hold every
    // same-layer point within 1e-10 of its boundary, hence every split point.
    const bool grid = d.sc[kGridOn] != 0;
    const int g = d.point_grid;
    const double qlx = lx - 1.0e-9, qly = ly - 1.0e-9, qhx = hx + 1.0e-9, qhy = hy + 1.0e-9;
    const int cx0 = grid_cell(qlx, g), cx1 = grid_cell(qhx, g);
    const int cy0 = grid_cell(qly, g), cy1 = grid_cell(qhy, g);
    if (grid) {
      int64_t candidates = 0;
      for (int cy = cy0; cy <= cy1; ++cy) {
        const int64_t row = (int64_t(layer) * g + cy) * g;
        candidates += d.cell_start[row + cx1 + 1] - d.cell_start[row + cx0];
      }
      if (candidates * n > d.heavy_noding_work) {
        d.heavy_polygons[atomicAdd(&d.sc[kHeavyPolygons], 1)] = int(i);
        continue;
      }
    }
    int count = 0, per_edge[kMaxVertices];
    for (int e = 0; e < n; ++e) per_edge[e] = 0;
    bool overflow = false;
    // Test one candidate point against every edge: a split point lies on the
    // edge's line within EPS, strictly inside the edge.
    auto node_point = [&](const V2 x) {
      for (int e = 0; e < n; ++e) {
        const V2 a = p[e], b = p[(e + 1) % n];
        // An edge's own end point has parameter 0 or 1 exactly: never a split.
        if (x == a || x == b) continue;
        const V2 dir = b - a;
        const double length2 = dot(dir, dir);
        if (!(length2 > 0.0)) continue;
        // Division-free rejection of points off the edge's line (4x slack over
        // the exact test below, which alone decides).
        const double off = cross(a, b, x);
        if (off * off > 4.0 * kEps * kEps * length2) continue;
        const double tt = dot(x - a, dir) / length2;
        if (tt > kEps && tt < 1.0 - kEps && fabs(cross(a, b, x)) <= kEps * sqrt(length2)) {
          if (++per_edge[e] > edge_capacity || count == kPolygonSplits) {
            overflow = true;
            return;
          }
          split_t[count] = tt;
          split_edge[count] = (unsigned char)e;
          ++count;
        }
      }
    };
    if (grid) {
      for (int cy = cy0; cy <= cy1 && !overflow; ++cy) {
        const int64_t row = (int64_t(layer) * g + cy) * g;
        const int end = d.cell_start[row + cx1 + 1];
        for (int j = d.cell_start[row + cx0]; j < end && !overflow; ++j) {
          const V2 x = d.grid_pts[j];
          if (x.x < qlx || x.x > qhx || x.y < qly || x.y > qhy) continue;
          node_point(x);
        }
      }
    } else {
      int node = 1;
      while (node > 0 && !overflow) {
        int j;
        node = query_next(d.point_tree, leaves, lo, hi, node, 0, j);
        if (j < 0) break;
        node_point(d.uverts[j]);
      }
    }
    if (overflow) {
      set_error(d.status, kErrEdgeNoding);
      return;
    }
    // Order the split points by (edge, parameter).
    for (int k = 1; k < count; ++k) {
      const double t = split_t[k];
      const unsigned char e = split_edge[k];
      int m = k - 1;
      while (m >= 0 && (split_edge[m] > e || (split_edge[m] == e && split_t[m] > t))) {
        split_t[m + 1] = split_t[m];
        split_edge[m + 1] = split_edge[m];
        --m;
      }
      split_t[m + 1] = t;
      split_edge[m + 1] = e;
    }
    emit_fan(d, p, n, center, layer, source, split_t, split_edge, count);
  }
}

// One polygon edge as the split-point test of k_mesh_polygons uses it, with
// the quantities that test derives from the edge computed once.
struct NodeEdge {
  V2 a, b, dir;
  double length2, slack, tol;
};

constexpr int kHeavyWarps = kBlock / 32;

// Noding and emission of the polygons k_mesh_polygons queued as heavy, one
// polygon per warp.  Lanes take the polygon's grid candidates 32 at a time
// and test each against every edge with the thread kernel's expressions, so
// the split points are the same.  Each split point is placed by its edge and
// its rank along the edge, and the fan is written with a lane per edge.
__global__ void __launch_bounds__(kBlock, 5) k_mesh_heavy(Dev d, int edge_capacity) {
  __shared__ NodeEdge s_edge[kHeavyWarps][kMaxVertices];
  __shared__ double s_t[kHeavyWarps][kPolygonSplits], s_sorted_t[kHeavyWarps][kPolygonSplits];
  __shared__ unsigned char s_e[kHeavyWarps][kPolygonSplits];
  __shared__ int s_count[kHeavyWarps], s_per_edge[kHeavyWarps][kMaxVertices];
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int heavy = d.sc[kHeavyPolygons];
  if (tid() == 0) d.metrics[kHeavyNodedPolygons] = heavy;
  const int g = d.point_grid;
  NodeEdge *edges = s_edge[warp];
  int *per_edge = s_per_edge[warp];
  double *split_t = s_t[warp], *sorted_t = s_sorted_t[warp];
  unsigned char *split_edge = s_e[warp];
  for (int64_t h = tid() >> 5; h < heavy; h += stride() >> 5) {
    int failed = 0;
    if (lane == 0) failed = *(volatile int *)&d.status[kError];
    if (__shfl_sync(kFull, failed, 0) != 0) return;
    const int i = d.heavy_polygons[h];
    const V2 *p = d.out_v + int64_t(kMaxVertices) * i;
    const int n = d.out_n[i];
    const int layer = d.out_layer[i], source = d.out_src[i];
    // Box and centroid in the thread kernel's order (every lane alike).
    double lx = 1.0e30, ly = 1.0e30, hx = -1.0e30, hy = -1.0e30;
    V2 center = v2(0.0, 0.0);
    for (int j = 0; j < n; ++j) {
      const V2 x = p[j];
      lx = fmin(lx, x.x); ly = fmin(ly, x.y);
      hx = fmax(hx, x.x); hy = fmax(hy, x.y);
      center = center + x / double(n);
    }
    if (lane < n) {
      NodeEdge e;
      e.a = p[lane];
      e.b = p[(lane + 1) % n];
      e.dir = e.b - e.a;
      e.length2 = dot(e.dir, e.dir);
      e.slack = 4.0 * kEps * kEps * e.length2;
      e.tol = kEps * sqrt(e.length2);
      edges[lane] = e;
      per_edge[lane] = 0;
    }
    if (lane == 0) s_count[warp] = 0;
    __syncwarp();
    const double qlx = lx - 1.0e-9, qly = ly - 1.0e-9, qhx = hx + 1.0e-9, qhy = hy + 1.0e-9;
    const int cx0 = grid_cell(qlx, g), cx1 = grid_cell(qhx, g);
    const int cy0 = grid_cell(qly, g), cy1 = grid_cell(qhy, g);
    for (int cy = cy0; cy <= cy1; ++cy) {
      const int64_t row = (int64_t(layer) * g + cy) * g;
      const int begin = d.cell_start[row + cx0], end = d.cell_start[row + cx1 + 1];
      for (int j = begin + lane; j < end; j += 32) {
        const V2 x = d.grid_pts[j];
        if (x.x < qlx || x.x > qhx || x.y < qly || x.y > qhy) continue;
        for (int e = 0; e < n; ++e) {
          const NodeEdge &E = edges[e];
          if (x == E.a || x == E.b) continue;
          if (!(E.length2 > 0.0)) continue;
          const double off = cross(E.a, E.b, x);
          if (off * off > E.slack) continue;
          const double tt = dot(x - E.a, E.dir) / E.length2;
          if (tt > kEps && tt < 1.0 - kEps && fabs(off) <= E.tol) {
            const int at = atomicAdd(&s_count[warp], 1);
            atomicAdd(&per_edge[e], 1);
            if (at < kPolygonSplits) {
              split_t[at] = tt;
              split_edge[at] = (unsigned char)e;
            }
          }
        }
      }
    }
    __syncwarp();
    // The thread kernel's overflow rule on the totals: more split points
    // than the buffer, or more on one edge than edge_capacity.
    const int count = s_count[warp];
    if (__any_sync(kFull, lane < n && per_edge[lane] > edge_capacity) || count > kPolygonSplits) {
      if (lane == 0) set_error(d.status, kErrEdgeNoding);
      return;
    }
    // Edge e's split points take places [first_e, first_e + count_e) of the
    // order by (edge, parameter): an exclusive scan of the per-edge counts.
    const int mine = lane < n ? per_edge[lane] : 0;
    int first = mine;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(kFull, first, off);
      if (lane >= off) first += y;
    }
    first -= mine;
    __syncwarp();
    if (lane < n) per_edge[lane] = first;
    __syncwarp();
    // A split point's place: its edge's first place plus its rank among the
    // edge's points by parameter, ties by arrival (equal parameters give the
    // same triangles in either order).
    for (int k = lane; k < count; k += 32) {
      const double t = split_t[k];
      const int e = split_edge[k];
      int rank = per_edge[e];
      for (int m = 0; m < count; ++m) {
        const double tm = split_t[m];
        rank += (split_edge[m] == e && (tm < t || (tm == t && m < k))) ? 1 : 0;
      }
      sorted_t[rank] = t;
    }
    __syncwarp();
    // The fan of emit_fan() with a lane per edge: lane e walks its edge's
    // split points, and the lanes' triangle counts are scanned in edge order,
    // so the triangles and their order within the polygon are emit_fan()'s.
    V2 a = v2(0.0, 0.0), dir = a;
    int emitted = 0;
    if (lane < n) {
      a = edges[lane].a;
      dir = edges[lane].dir;
      double previous = 0.0;
      V2 cursor = a;
      for (int k = first;;) {
        const bool last = k == first + mine;
        const double following = last ? 1.0 : sorted_t[k++];
        if (following > previous + kEps) {
          const V2 next = a + following * dir;
          if (cross(center, cursor, next) > kEps * kEps) ++emitted;
          cursor = next;
          previous = following;
        }
        if (last) break;
      }
    }
    int offset = emitted;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(kFull, offset, off);
      if (lane >= off) offset += y;
    }
    const int total = __shfl_sync(kFull, offset, 31);
    offset -= emitted;
    int base = 0;
    if (lane == 0 && total) base = atomicAdd(&d.status[kTriangles], total);
    base = __shfl_sync(kFull, base, 0);
    if (int64_t(base) + total > d.cap.triangles) {
      if (lane == 0) set_error(d.status, kErrTriangles);
      __syncwarp();
      continue;
    }
    if (lane < n) {
      const Plane sc = d.scores[source];
      double w_center[3];
      lift(d, center, sc, w_center);
      int slot = base + offset;
      double previous = 0.0;
      V2 cursor = a;
      double w_cursor[3];
      lift(d, cursor, sc, w_cursor);
      for (int k = first;;) {
        const bool last = k == first + mine;
        const double following = last ? 1.0 : sorted_t[k++];
        if (following > previous + kEps) {
          const V2 next = a + following * dir;
          double w_next[3];
          lift(d, next, sc, w_next);
          if (cross(center, cursor, next) > kEps * kEps) {
            V2 *uv = d.tri_uv + 3 * int64_t(slot);
            double *w = d.tri_world + 9 * int64_t(slot);
            uv[0] = center;
            uv[1] = cursor;
            uv[2] = next;
            for (int c = 0; c < 3; ++c) {
              w[c] = w_center[c];
              w[3 + c] = w_cursor[c];
              w[6 + c] = w_next[c];
            }
            d.tri_src[slot] = source;
            d.tri_layer[slot] = layer;
            ++slot;
          }
          cursor = next;
          for (int c = 0; c < 3; ++c) w_cursor[c] = w_next[c];
          previous = following;
        }
        if (last) break;
      }
    }
    __syncwarp();
  }
}
unsigned blocks(int64_t n) {
  int64_t g = ceil_div(n > 0 ? n : 1, kBlock);
  return unsigned(g < 148 * 16 ? g : 148 * 16);
}

}  // namespace

cudaError_t order_polygons(const Dev &d, bool layered, SortScratch &s, cudaStream_t st) {
  const int64_t R = d.cap.regions;
  k_order_keys<<<blocks(R), kBlock, 0, st>>>(d, layered ? 1 : 0);
  note_launch();
  // 16 layer bits above 24 Morton bits.
  return sort_pairs_u64(d.order_keys, d.order_keys_tmp, d.order, d.order_tmp,
                        d.sc + kLivePolygons, R, layered ? 40 : 24, s, st);
}

cudaError_t stage_mesh_index(const Dev &d, SortScratch &s, TreeBuffers &point_tree,
                             cudaStream_t st) {
  const int64_t R = d.cap.regions, E = d.cap.vertices;
  EDP_CHECK(order_polygons(d, true, s, st));
  k_mesh_counts<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(scan_exclusive(d.counts, d.offsets, d.sc + kLivePolygons, R, d.sc + kLiveVertices, s, st));
  k_mesh_check<<<1, 1, 0, st>>>(d);
  note_launch();
  EDP_CHECK(cudaMemsetAsync(d.point_table, 0xff, sizeof(int) * (int64_t(d.point_mask) + 1), st));
  const int64_t cells = int64_t(d.grid_layers) * d.point_grid * d.point_grid;
  k_grid_begin<<<1, 1, 0, st>>>(d);
  note_launch();
  k_grid_clear<<<blocks(cells), kBlock, 0, st>>>(d);
  note_launch();
  k_scatter<<<blocks(R), kBlock, 0, st>>>(d);
  note_launch();
  k_unique_points<<<blocks(E), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_MESH_VERTICES, st));
  EDP_CHECK(scan_exclusive(d.cell_count, d.cell_start, d.sc + kGridCells, cells, nullptr, s, st));
  k_grid_scatter<<<blocks(E), kBlock, 0, st>>>(d);
  note_launch();
  k_tree_points<<<1, 1, 0, st>>>(d);
  note_launch();
  EDP_CHECK(tree_build(point_tree, d.pt_lo, d.pt_hi, d.sc + kTreePoints, 0, true, s, st));
  EDP_CHECK(stage_mark(EDP_STAGE_MESH_INDEX, st));
  return cudaGetLastError();
}

cudaError_t stage_mesh_emit(const Dev &d, cudaStream_t st) {
  int cap = int(d.cap.edge_vertices < kMaxEdgeVertices ? d.cap.edge_vertices : kMaxEdgeVertices);
  EDP_CHECK(cudaMemsetAsync(d.sc + kHeavyPolygons, 0, sizeof(int), st));
  k_mesh_polygons<<<blocks(d.cap.regions), kBlock, 0, st>>>(d, cap);
  note_launch();
  k_mesh_heavy<<<148 * 5, kBlock, 0, st>>>(d, cap);
  note_launch();
  EDP_CHECK(stage_mark(EDP_STAGE_MESH_EMIT, st));
  return cudaGetLastError();
}

cudaError_t stage_mesh(const Dev &d, SortScratch &s, TreeBuffers &point_tree, cudaStream_t st) {
  EDP_CHECK(stage_mesh_index(d, s, point_tree, st));
  return stage_mesh_emit(d, st);
}

}  // namespace edp

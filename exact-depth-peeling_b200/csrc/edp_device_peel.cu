// DevicePeeler: whole-source ranks, then iterative per-layer clipping
// (warp_peel/solver.py:217-379, kernels.py:539-938).
//
// Each layer pass: sources whose whole-face rank is below the current layer
// retire from the source hierarchy (a refit, no re-sort), the residual
// hierarchy is rebuilt over the patches still unresolved, and persistent
// workers subtract every candidate that can be in front of a target patch.
// Pieces that stay visible are output for this layer; hidden pieces form the
// next pass's residual.  The loop is the graph's conditional WHILE node.
#include "../../include/edp.h"
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kBlock = 128;

__device__ inline int64_t tid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ inline int64_t stride() { return int64_t(gridDim.x) * blockDim.x; }

unsigned blocks(int64_t n) {
  int64_t g = ceil_div(n > 0 ? n : 1, kBlock);
  return unsigned(g < 148 * 16 ? g : 148 * 16);
}

// Bounds of a source's contour edges, xy only (kernels.py:539-559).
__global__ void k_contour_bounds(Dev d) {
  for (int64_t i = tid(); i < d.n; i += stride()) {
    const V2 *p = d.src_v + int64_t(kSourceVertices) * i;
    const int n = d.status[kError] == 0 ? d.src_n[i] : 0;
    double lx = 1.0e30, ly = 1.0e30, hx = -1.0e30, hy = -1.0e30;
    for (int j = 0; j < n; ++j) {
      if (!contour_edge(d, i, j)) continue;
      V2 a = p[j], b = p[(j + 1) % n];
      lx = fmin(lx, fmin(a.x, b.x)); ly = fmin(ly, fmin(a.y, b.y));
      hx = fmax(hx, fmax(a.x, b.x)); hy = fmax(hy, fmax(a.y, b.y));
    }
    if (lx <= hx) {
      d.contour_lo[i] = make_float4(__double2float_rd(lx - 2.0e-7), __double2float_rd(ly - 2.0e-7),
                                    -2.0e-7f, 0.f);
      d.contour_hi[i] = make_float4(__double2float_ru(hx + 2.0e-7), __double2float_ru(hy + 2.0e-7),
                                    2.0e-7f, 0.f);
    } else {
      d.contour_lo[i] = empty_lo();
      d.contour_hi[i] = empty_hi();
    }
  }
}

// Segment a-b touches convex polygon p, conservatively by EPS (kernels.py:562-576).
__device__ inline bool touches(const V2 *p, int n, V2 a, V2 b) {
  bool hit = true;
  for (int j = 0; j < n; ++j)
    if (cross(p[j], p[(j + 1) % n], a) < -kEps && cross(p[j], p[(j + 1) % n], b) < -kEps)
      hit = false;
  bool positive = false, negative = false;
  for (int j = 0; j < n; ++j) {
    double v = cross(a, b, p[j]);
    positive = positive || v >= -kEps;
    negative = negative || v <= kEps;
  }
  return hit && positive && negative;
}

__device__ inline void save_polygon(const Dev &d, const V2 *p, int n, int source, int layer) {
  int slot = reserve(&d.status[kPolygons], 1);
  if (slot < d.cap.regions) {
    V2 *dst = d.out_v + int64_t(kMaxVertices) * slot;
    for (int j = 0; j < n; ++j) dst[j] = p[j];
    d.out_n[slot] = n;
    d.out_src[slot] = source;
    d.out_layer[slot] = layer;
    atomicMax(&d.status[kLayers], layer + 1);
  } else {
    set_error(d.status, kErrOutput);
  }
}

// Whole-source rank where no contour touches the source: count the sources
// strictly nearer at its centroid; ambiguous samples (on an edge, or a depth
// tie within 1e-12) go to clipping instead (kernels.py:599-690).
__global__ void k_classify(Dev d) {
  const int contour_leaves = *d.contour_tree.size, source_leaves = *d.source_tree.size;
  for (int64_t i = tid(); i < d.n; i += stride()) {
    const V2 *p = d.src_v + int64_t(kSourceVertices) * i;
    const int n = d.status[kError] == 0 ? d.src_n[i] : 0;
    int rank = -1;
    if (n > 0) {
      float4 lo, hi;
      polygon_bounds(p, n, Plane{0, 0, 0, 0}, lo, hi);
      lo.z = -1.0e-6f;
      hi.z = 1.0e-6f;
      bool boundary = false;
      int node = 1;
      while (node > 0 && !boundary) {
        int j;
        node = query_next(d.contour_tree, contour_leaves, lo, hi, node, 0, j);
        if (j < 0) break;
        const V2 *q = d.src_v + int64_t(kSourceVertices) * j;
        const int qn = d.src_n[j];
        for (int e = 0; e < qn && !boundary; ++e)
          if (contour_edge(d, j, e) && touches(p, n, q[e], q[(e + 1) % qn])) boundary = true;
      }
      if (!boundary) {
        V2 sample = v2(0.0, 0.0);
        for (int e = 0; e < n; ++e) sample = sample + p[e] / double(n);
        double z = value(d.scores[i], sample);
        float4 qlo = make_float4(__double2float_rd(sample.x - 2.0e-7),
                                 __double2float_rd(sample.y - 2.0e-7), -1.0e30f, 0.f);
        float4 qhi = make_float4(__double2float_ru(sample.x + 2.0e-7),
                                 __double2float_ru(sample.y + 2.0e-7),
                                 __double2float_ru(z + 2.0e-7 * fmax(1.0, fabs(z))), 0.f);
        rank = 0;
        bool ambiguous = false;
        int node2 = 1;
        while (node2 > 0) {
          int j;
          node2 = query_next(d.source_tree, source_leaves, qlo, qhi, node2, 0, j);
          if (j < 0) break;
          if (j == int(i)) continue;
          const V2 *q = d.src_v + int64_t(kSourceVertices) * j;
          const int qn = d.src_n[j];
          bool inside = qn > 0, edge = false;
          for (int e = 0; e < qn; ++e) {
            double s = cross(q[e], q[(e + 1) % qn], sample);
            inside = inside && s >= 0.0;
            edge = edge || fabs(s) <= kEps;
          }
          if (inside) {
            double delta = z - value(d.scores[j], sample);
            if (edge || fabs(delta) <= 1.0e-12 * fmax(1.0, fabs(z)))
              ambiguous = true;
            else if (delta > 0.0)
              ++rank;
          }
        }
        if (ambiguous) rank = -1;
      }
      if (rank < 0) {
        int slot = reserve(&d.status[kResidual], 1);
        if (slot < d.cap.frontier) {
          V2 *dst = d.res_v[0] + int64_t(kMaxVertices) * slot;
          for (int e = 0; e < n; ++e) dst[e] = p[e];
          d.res_n[0][slot] = n;
          d.res_src[0][slot] = int(i);
        } else {
          set_error(d.status, kErrResidual);
        }
      } else if (rank < d.limit) {
        save_polygon(d, p, n, int(i), rank);
      } else if (d.all_layers) {
        set_error(d.status, kErrLayers);
      }
    }
    d.ranks[i] = rank;
  }
}

__global__ void k_start_loop(Dev d) {
  d.status[kPeakResidual] = d.status[kResidual];
  *d.parity = 0;
  int c = d.status[kResidual] > 0 && d.status[kError] == 0;
  *d.condition = c;
  if (d.use_handle) cudaGraphSetConditional(d.cond_handle, unsigned(c));
}

// Source boxes with ranks below the current layer retire (kernels.py:717-732).
__global__ void k_retire_bounds(Dev d) {
  const int layer = d.status[kPass];
  for (int64_t i = tid(); i < d.n; i += stride()) {
    float4 lo = empty_lo(), hi = empty_hi();
    if (d.ranks[i] >= layer)
      polygon_bounds(d.src_v + int64_t(kSourceVertices) * i, d.src_n[i], d.scores[i], lo, hi);
    d.src_lo[i] = lo;
    d.src_hi[i] = hi;
  }
}

// Boxes of the current residual patches (kernels.py:699-714).
__global__ void k_active_bounds(Dev d) {
  const int par = *d.parity;
  const int live = int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  for (int64_t i = tid(); i < live; i += stride()) {
    float4 lo = empty_lo(), hi = empty_hi();
    if (d.status[kError] == 0)
      polygon_bounds(d.res_v[par] + int64_t(kMaxVertices) * i, d.res_n[par][i],
                     d.scores[d.res_src[par][i]], lo, hi);
    d.res_lo[i] = lo;
    d.res_hi[i] = hi;
  }
  if (tid() == 0) d.sc[kFrontierLive] = live;
}

// A worker's pool slot k of kind (0 visible, 1 temporary, 2 hidden).
struct Pools {
  const Dev &d;
  int worker;
  __device__ V2 *v(int kind, int k) const {
    return d.pool_v[kind] + (int64_t(worker) * d.pieces + k) * kMaxVertices;
  }
  __device__ int &n(int kind, int k) const { return d.pool_n[kind][int64_t(worker) * d.pieces + k]; }
  __device__ void put(int kind, int k, const V2 *p, int pn) const {
    if (k >= d.pieces) return;
    V2 *dst = v(kind, k);
    for (int j = 0; j < pn; ++j) dst[j] = p[j];
    n(kind, k) = pn;
  }
};

// Subtract `candidate` from the worker's visible pieces where the target is
// behind it (delta = target - candidate depth > 0): split by the depth
// equality line, then by the candidate's edges; the covered part becomes a
// hidden piece.  Equal-depth overlap uses the lower source index as nearer.
// Returns the new visible count, or -1 after setting an error bit
// (kernels.py:735-812).
__device__ int cut(const Pools &pool, int nv, int &nh, const V2 *cand, int cn, Plane delta,
                   int target_source, int other_source) {
  const Dev &d = pool.d;
  const int cap = d.pieces;
  int count = 0;
  V2 p[kMaxVertices], inside[kMaxVertices], outside[kMaxVertices], rest[kMaxVertices];
  for (int k = 0; k < nv; ++k) {
    const int pn = pool.n(0, k);
    {
      const V2 *src = pool.v(0, k);
      for (int j = 0; j < pn; ++j) p[j] = src[j];
    }
    if (separated(p, pn, cand, cn) || separated(cand, cn, p, pn)) {
      pool.put(1, count++, p, pn);
    } else {
      bool positive = false, negative = false;
      for (int e = 0; e < pn; ++e) {
        double v = value(delta, p[e]);
        positive = positive || v > 0.0;
        negative = negative || v < 0.0;
      }
      if (!positive && !negative) {
        positive = target_source > other_source;
        atomicAdd(&d.status[kDepthTies], 1);
      }
      if (!positive) {
        pool.put(1, count++, p, pn);
      } else {
        int in_n = pn;
        for (int j = 0; j < pn; ++j) inside[j] = p[j];
        const int base = count;
        if (negative) {
          int out_n;
          split_at(p, pn, delta, v2(0.0, 0.0), inside, in_n, outside, out_n);
          if (in_n > kMaxVertices || out_n > kMaxVertices) {
            set_error(d.status, kErrPolygon);
            return -1;
          }
          if (out_n > 0) pool.put(1, count++, outside, out_n);
        }
        for (int e = 0; e < cn && in_n > 0; ++e) {
          int next_n, out_n;
          split_edge(inside, in_n, cand[e], cand[(e + 1) % cn], rest, next_n, outside, out_n);
          if (next_n > kMaxVertices || out_n > kMaxVertices) {
            set_error(d.status, kErrPolygon);
            return -1;
          }
          for (int j = 0; j < next_n; ++j) inside[j] = rest[j];
          in_n = next_n;
          if (out_n > 0) pool.put(1, count++, outside, out_n);
        }
        if (in_n == 0) {
          count = base;
          pool.put(1, count++, p, pn);
        } else {
          pool.put(2, nh++, inside, in_n);
        }
      }
    }
    if (count > cap || nh > cap) {
      set_error(d.status, kErrWorker);
      return -1;
    }
  }
  for (int k = 0; k < count; ++k) pool.put(0, k, pool.v(1, k), pool.n(1, k));
  return count;
}

// One layer pass: persistent workers own targets in turn (kernels.py:815-908).
__global__ void k_peel(Dev d) {
  const int par = *d.parity;
  const V2 *res_v = d.res_v[par];
  const int *res_n = d.res_n[par], *res_src = d.res_src[par];
  V2 *next_v = d.res_v[par ^ 1];
  int *next_n = d.res_n[par ^ 1], *next_src = d.res_src[par ^ 1];
  const int layer = d.status[kPass];
  const int live = int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  const int source_leaves = *d.source_tree.size, residual_leaves = *d.residual_tree.size;
  const int worker = int(tid());
  if (worker >= d.workers) return;
  Pools pool{d, worker};
  long long targets = 0, tested_all = 0, restored = 0;
  int max_hidden = 0;
  for (int target = worker; target < live; target += d.workers) {
    if (d.status[kError] != 0) break;
    const V2 *p = res_v + int64_t(kMaxVertices) * target;
    const int pn = res_n[target], source = res_src[target];
    int nv = 1, nh = 0;
    pool.put(0, 0, p, pn);
    const Plane score = d.scores[source];
    float4 lo, hi;
    polygon_bounds(p, pn, score, lo, hi);
    lo.z = -1.0e30f;
    long long tested = 0;
    for (int tree = 0; tree < 2 && nv > 0; ++tree) {
      const Tree &t = tree == 0 ? d.source_tree : d.residual_tree;
      const int leaves = tree == 0 ? source_leaves : residual_leaves;
      int node = 1;
      while (node > 0 && nv > 0) {
        int c;
        node = query_next(t, leaves, lo, hi, node, 0, c);
        if (c < 0) break;
        int other = c;
        const V2 *cand;
        int cn;
        bool eligible = true;
        if (tree == 0) {
          cand = d.src_v + int64_t(kSourceVertices) * c;
          cn = d.src_n[c];
          eligible = d.ranks[c] >= layer;
        } else {
          cand = res_v + int64_t(kMaxVertices) * c;
          cn = res_n[c];
          other = res_src[c];
        }
        if (eligible && other != source) {
          ++tested;
          const Plane so = d.scores[other];
          Plane delta{score.a - so.a, score.b - so.b, score.c - so.c, 0.0};
          nv = cut(pool, nv, nh, cand, cn, delta, source, other);
        }
      }
    }
    ++targets;
    tested_all += tested;
    max_hidden = max(max_hidden, nh);
    if (nv == 0) {
      pool.put(2, 0, p, pn);
      nh = 1;
      ++restored;
    }
    if (nv >= 0 && d.status[kError] == 0) {
      for (int k = 0; k < nv; ++k) save_polygon(d, pool.v(0, k), pool.n(0, k), source, layer);
      int offset = reserve(&d.status[kNextResidual], nh);
      if (int64_t(offset) + nh > d.cap.frontier) {
        set_error(d.status, kErrResidual);
      } else {
        for (int k = 0; k < nh; ++k) {
          const V2 *src = pool.v(2, k);
          const int hn = pool.n(2, k);
          V2 *dst = next_v + int64_t(kMaxVertices) * (offset + k);
          for (int j = 0; j < hn; ++j) dst[j] = src[j];
          next_n[offset + k] = hn;
          next_src[offset + k] = source;
        }
      }
    }
  }
  if (layer < d.cap.layers) {
    long long *row = d.stats + 3 * int64_t(layer);
    count_add(&row[0], targets);
    count_add(&row[1], tested_all);
    count_add(&row[2], restored);
  }
  if (max_hidden) atomicMax(&d.status[kMaxHidden], max_hidden);
}

// Next pass, or stop (kernels.py:925-938).
__global__ void k_advance_layer(Dev d) {
  int next = d.status[kNextResidual];
  d.status[kResidual] = next;
  d.status[kPeakResidual] = max(d.status[kPeakResidual], next);
  d.status[kNextResidual] = 0;
  int layer = ++d.status[kPass];
  *d.parity ^= 1;
  if (next > 0 && layer >= d.limit && d.all_layers) set_error(d.status, kErrLayers);
  int c = next > 0 && layer < d.limit && d.status[kError] == 0;
  *d.condition = c;
  if (d.use_handle) cudaGraphSetConditional(d.cond_handle, unsigned(c));
}

__global__ void k_device_finish(Dev d) {
  d.sc[kLivePolygons] = int(min(int64_t(d.status[kPolygons]), d.cap.regions));
}

}  // namespace

cudaError_t stage_device_finish(const Dev &d, cudaStream_t st) {
  k_device_finish<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t stage_device_prepare(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                                 TreeBuffers &contour_tree, cudaStream_t st) {
  EDP_CHECK(stage_prepare_common(d, s, source_tree, st));
  EDP_CHECK(cudaMemsetAsync(d.stats, 0, sizeof(long long) * 3 * d.cap.layers, st));
  k_contour_bounds<<<blocks(d.n), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(tree_build(contour_tree, d.contour_lo, d.contour_hi, nullptr, d.n, false, s, st));
  k_classify<<<blocks(d.n), kBlock, 0, st>>>(d);
  note_launch();
  k_start_loop<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

cudaError_t stage_device_layer(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                               TreeBuffers &residual_tree, cudaStream_t st) {
  k_retire_bounds<<<blocks(d.n), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(tree_refit(source_tree, d.src_lo, d.src_hi, st));
  k_active_bounds<<<blocks(d.cap.frontier), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(tree_build(residual_tree, d.res_lo, d.res_hi, d.sc + kFrontierLive, 0, false, s, st));
  k_peel<<<unsigned(ceil_div(d.workers, kBlock)), kBlock, 0, st>>>(d);
  note_launch();
  k_advance_layer<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

}  // namespace edp

// DevicePeeler: whole-source ranks, then iterative per-layer clipping
// (warp_peel/solver.py:217-379, kernels.py:539-938).
//
// Each layer pass: sources whose whole-face rank is below the current layer
// retire from the source hierarchy (a refit, no re-sort), the residual
// hierarchy is rebuilt over the patches still unresolved, and a queue of
// pieces is clipped round by round against every candidate that can be in
// front of its target (below).  Pieces that stay visible are output for this
// layer; hidden pieces form the next pass's residual.  The layer loop is the
// graph's conditional WHILE node, the clipping rounds a WHILE node nested in
// its body.
#include "../../include/edp.h"
#include "edp_filtered.cuh"
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

// ---------------------------------------------------------------- clipping
// A layer pass subtracts, from every residual patch (a target), each
// candidate that can lie in front of it: original sources of rank >= layer
// from the source hierarchy, then the other residual patches from the
// residual hierarchy (src/peel_common.h:169-199).  The work is a queue of
// pieces: a piece is a convex part of a target with the position of its
// candidate walk (which hierarchy, and the node the stackless walk resumes
// at).  Each clipping round runs every queued piece against its next
// Dev::clip_budget candidates.  A candidate that cuts a piece ends the piece's
// round: the parts of the piece outside the candidate (or nearer than it)
// are queued for the next round with the walk position past the candidate,
// and the part the candidate hides goes to the layer's hidden pool.  A piece
// that meets no more candidates is visible in this layer.  Rounds repeat
// (a conditional WHILE node inside the layer loop) until the queue is empty;
// then a target none of whose pieces stayed visible is hidden whole, as the
// exact route restores it (src/bvh_peel.cpp:141-199), and the hidden pieces
// form the next layer's residual.  The work and hidden pools are shared by
// all targets and compacted by atomic appends, so their size follows the
// pieces alive, not a per-thread reservation.

constexpr int kCursorTree = 29;   // walk position: hierarchy << 29 | node
constexpr int kCursorNode = (1 << kCursorTree) - 1;

__device__ inline V2 *piece_at(V2 *base, int64_t slot) { return base + kMaxVertices * slot; }

// Queues a piece for the next round; false (and the worker-pool error) when
// the pool is full.
__device__ inline bool queue_piece(const Dev &d, int next, const V2 *v, int n, int target,
                                   int cursor) {
  const int slot = atomicAdd(&d.sc[kClipNext], 1);
  if (slot >= d.work_cap) {
    set_error(d.status, kErrWorker);
    return false;
  }
  V2 *dst = piece_at(d.work_v[next], slot);
  for (int j = 0; j < n; ++j) dst[j] = v[j];
  d.work_n[next][slot] = n;
  d.work_target[next][slot] = target;
  d.work_cursor[next][slot] = cursor;
  return true;
}

__device__ inline void hide_piece(const Dev &d, const V2 *v, int n, int target) {
  if (atomicAdd(&d.target_hidden[target], 1) >= d.pieces) set_error(d.status, kErrWorker);
  const int slot = atomicAdd(&d.sc[kClipHidden], 1);
  if (slot >= d.hidden_cap) {
    set_error(d.status, kErrResidual);
    return;
  }
  V2 *dst = piece_at(d.hid_v, slot);
  for (int j = 0; j < n; ++j) dst[j] = v[j];
  d.hid_n[slot] = n;
  d.hid_target[slot] = target;
}

// Split convex p by per-vertex signs (>= 0 goes to `in`, <= 0 to `out`), the
// crossing points placed with the binary64 values `val` (the signed
// distances the signs belong to), then clean both (kernels.py:184-203).
__device__ inline void split_signed(const V2 *p, int n, const int *sgn, const double *val, V2 *in,
                                    int &ni, V2 *out, int &no) {
  ni = 0;
  no = 0;
  for (int j = 0; j < n; ++j) {
    const int k = (j + 1) % n;
    if (sgn[j] >= 0) ni = append(in, ni, p[j]);
    if (sgn[j] <= 0) no = append(out, no, p[j]);
    if ((sgn[j] > 0 && sgn[k] < 0) || (sgn[j] < 0 && sgn[k] > 0)) {
      const V2 x = p[j] + crossing(val[j], val[k]) * (p[k] - p[j]);
      ni = append(in, ni, x);
      no = append(out, no, x);
    }
  }
  ni = clean(in, ni);
  no = clean(out, no);
}

// Some edge of a has no vertex of b strictly on its left (kernels.py:219-232),
// with the form's side predicate.
template <int F>
__device__ inline bool separated_form(const V2 *a, int na, const V2 *b, int nb, Tally &t) {
  for (int j = 0; j < na; ++j) {
    bool positive = false;
    for (int k = 0; k < nb && !positive; ++k) {
      int stage = 0;
      positive = side_sign<F>(a[j], a[(j + 1) % na], b[k], stage) > 0;
      if constexpr (F == 2) t.add(stage);
    }
    if (!positive) return true;
  }
  return false;
}

enum CutResult : int { kKept = 0, kCut = 1, kFailed = 2 };

// Split `in` by the supporting line of a->b: the left part (inside a
// counter-clockwise candidate) to `left`, the right part to `right`.
template <int F>
__device__ inline void clip_edge(const V2 *in, int n, V2 a, V2 b, V2 *left, int &nl, V2 *right,
                                 int &nr, Tally &t) {
  if constexpr (F == 0) {
    split_edge(in, n, a, b, left, nl, right, nr);
  } else {
    int sgn[kMaxVertices];
    double val[kMaxVertices];
    const V2 dir = b - a;
    const Plane line{-dir.y, dir.x, 0.0, 0.0};
    for (int j = 0; j < n; ++j) {
      int stage = 0;
      val[j] = value(line, in[j] - a);
      sgn[j] = side_sign<F>(a, b, in[j], stage);
      if constexpr (F == 2) t.add(stage);
    }
    split_signed(in, n, sgn, val, left, nl, right, nr);
  }
}

// One candidate against one piece (the semantics of src/bvh_peel.cpp:141-199):
// where the piece lies behind the candidate (its depth plane st above the
// candidate's so), the part inside the candidate is hidden and the rest of
// the piece is queued with walk position `cursor`.  A piece the candidate
// cannot cover, or whose covered part clips away to nothing, is kept
// unchanged (kKept).  Equal-depth overlap counts the lower source index as
// nearer.  The covered part is found first without queuing anything, so a
// cut that hides nothing leaves no parts behind; the splits are then redone
// (same operations, same results) to queue the uncovered parts.
template <int F>
__device__ int cut_piece(const Dev &d, const V2 *p, int pn, const V2 *cand, int cn,
                         const Plane &st, const Plane &so, int target_source, int other_source,
                         int target, int next, int cursor, Tally &t) {
  if (separated_form<F>(p, pn, cand, cn, t) || separated_form<F>(cand, cn, p, pn, t))
    return kKept;
  const Plane delta{st.a - so.a, st.b - so.b, st.c - so.c, 0.0};
  int sgn[kMaxVertices];
  double val[kMaxVertices];
  bool positive = false, negative = false;
  for (int e = 0; e < pn; ++e) {
    val[e] = value(delta, p[e]);
    if constexpr (F == 0) {
      sgn[e] = sign_of(val[e]);
    } else {
      int stage = 0;
      sgn[e] = order_sign<F>(st, value(st, p[e]), so, value(so, p[e]), p[e], stage);
      if constexpr (F == 2) t.add(stage);
    }
    positive = positive || sgn[e] > 0;
    negative = negative || sgn[e] < 0;
  }
  if (!positive && !negative) {
    positive = target_source > other_source;
    atomicAdd(&d.status[kDepthTies], 1);
  }
  if (!positive) return kKept;
  V2 behind[kMaxVertices], nearer[kMaxVertices], inside[kMaxVertices], rest[kMaxVertices];
  V2 out[kMaxVertices];
  int behind_n = pn, nearer_n = 0;
  if (negative) {
    if constexpr (F == 0)
      split_at(p, pn, delta, v2(0.0, 0.0), behind, behind_n, nearer, nearer_n);
    else
      split_signed(p, pn, sgn, val, behind, behind_n, nearer, nearer_n);
  } else {
    for (int j = 0; j < pn; ++j) behind[j] = p[j];
  }
  if (behind_n > kMaxVertices || nearer_n > kMaxVertices) {
    set_error(d.status, kErrPolygon);
    return kFailed;
  }
  for (int pass = 0; pass < 2; ++pass) {
    // Pass 0 finds the covered part; pass 1 queues the uncovered parts.
    if (pass == 1 && nearer_n > 0 && !queue_piece(d, next, nearer, nearer_n, target, cursor))
      return kFailed;
    int in_n = behind_n;
    for (int j = 0; j < in_n; ++j) inside[j] = behind[j];
    for (int e = 0; e < cn && in_n > 0; ++e) {
      int rest_n, out_n;
      clip_edge<F>(inside, in_n, cand[e], cand[(e + 1) % cn], rest, rest_n, out, out_n, t);
      if (rest_n > kMaxVertices || out_n > kMaxVertices) {
        set_error(d.status, kErrPolygon);
        return kFailed;
      }
      if (pass == 1 && out_n > 0 && !queue_piece(d, next, out, out_n, target, cursor))
        return kFailed;
      for (int j = 0; j < rest_n; ++j) inside[j] = rest[j];
      in_n = rest_n;
    }
    if (pass == 0 && in_n == 0) return kKept;  // nothing covered after all
    if (pass == 1) hide_piece(d, inside, in_n, target);
  }
  return kCut;
}

// Seed the clipping queue with this layer's targets, each a whole residual
// patch at the start of its walk.
__global__ void k_clip_begin(Dev d) {
  const int par = *d.parity;
  const int live = int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  for (int64_t i = tid(); i < live; i += stride()) {
    const int n = d.status[kError] == 0 ? d.res_n[par][i] : 0;
    V2 *dst = piece_at(d.work_v[0], i);
    const V2 *src = piece_at(d.res_v[par], i);
    for (int j = 0; j < n; ++j) dst[j] = src[j];
    d.work_n[0][i] = n;
    d.work_target[0][i] = int(i);
    d.work_cursor[0][i] = 1;  // the source hierarchy's root
    d.target_visible[i] = 0;
    d.target_hidden[i] = 0;
  }
  if (tid() == 0) {
    const int queued = live <= d.work_cap ? live : 0;
    if (live > d.work_cap) set_error(d.status, kErrWorker);
    d.sc[kClipLive] = queued;
    d.sc[kClipNext] = 0;
    d.sc[kClipHidden] = 0;
    d.sc[kClipParity] = 0;
    const int c = queued > 0 && d.status[kError] == 0;
    d.sc[kClipCondition] = c;
    if (d.use_inner) cudaGraphSetConditional(d.inner_handle, unsigned(c));
  }
}

// One clipping round over the queued pieces.  F is the predicate form.
template <int F>
__global__ void k_clip_round(Dev d) {
  const int wpar = d.sc[kClipParity], next = wpar ^ 1;
  const int live = min(d.sc[kClipLive], d.work_cap);
  const int rpar = *d.parity;
  const int layer = d.status[kPass];
  const int source_leaves = *d.source_tree.size, residual_leaves = *d.residual_tree.size;
  long long tested = 0;
  Tally clip;
  V2 p[kMaxVertices];
  for (int64_t i = tid(); i < live; i += stride()) {
    if (d.status[kError] != 0) break;
    const int pn = d.work_n[wpar][i];
    if (pn < 3) continue;
    const int target = d.work_target[wpar][i];
    int cursor = d.work_cursor[wpar][i];
    {
      const V2 *src = piece_at(d.work_v[wpar], i);
      for (int j = 0; j < pn; ++j) p[j] = src[j];
    }
    const int source = d.res_src[rpar][target];
    const Plane st = d.scores[source];
    float4 lo, hi;
    polygon_bounds(p, pn, st, lo, hi);
    lo.z = -1.0e30f;
    int budget = d.clip_budget;
    int result = kKept;
    while (budget > 0) {
      const int tree = cursor >> kCursorTree;
      int node = cursor & kCursorNode;
      if (tree >= 2) break;  // both walks done
      const Tree &t = tree == 0 ? d.source_tree : d.residual_tree;
      const int leaves = tree == 0 ? source_leaves : residual_leaves;
      int c = -1;
      node = node > 0 ? query_next(t, leaves, lo, hi, node, 0, c) : 0;
      cursor = node > 0 ? (tree << kCursorTree) | node : (tree + 1) << kCursorTree | 1;
      if (c < 0) continue;
      const V2 *cand;
      int cn, other;
      bool eligible;
      if (tree == 0) {
        cand = d.src_v + int64_t(kSourceVertices) * c;
        cn = d.src_n[c];
        other = c;
        eligible = d.ranks[c] >= layer;
      } else {
        cand = piece_at(d.res_v[rpar], c);
        cn = d.res_n[rpar][c];
        other = d.res_src[rpar][c];
        eligible = true;
      }
      if (!eligible || other == source) continue;
      --budget;
      ++tested;
      result = cut_piece<F>(d, p, pn, cand, cn, st, d.scores[other], source, other, target,
                            next, cursor, clip);
      if (result != kKept) break;
    }
    if (result == kFailed) break;
    if (result == kCut) {
      // cut_piece queued the uncovered parts; the covered part is hidden.
      continue;
    }
    if ((cursor >> kCursorTree) >= 2) {
      if (atomicAdd(&d.target_visible[target], 1) >= d.pieces) set_error(d.status, kErrWorker);
      save_polygon(d, p, pn, source, layer);
    } else {
      queue_piece(d, next, p, pn, target, cursor);
    }
  }
  if (layer < d.cap.layers && tested) count_add(&d.stats[3 * int64_t(layer) + 1], tested);
  if constexpr (F == 2) clip.flush(d, kPredClip);
}

// Between rounds: the appended pieces become the queue; stop when it is
// empty.
__global__ void k_clip_advance(Dev d) {
  const int queued = d.sc[kClipNext];
  d.sc[kClipLive] = min(queued, d.work_cap);
  d.sc[kClipNext] = 0;
  d.sc[kClipParity] ^= 1;
  const int c = queued > 0 && d.status[kError] == 0;
  d.sc[kClipCondition] = c;
  if (d.use_inner) cudaGraphSetConditional(d.inner_handle, unsigned(c));
}

// After the last round: a target with no visible piece is hidden whole (its
// hidden pieces are dropped); every other target's hidden pieces go to the
// next layer's residual.  Threads run over targets and hidden pieces alike.
__global__ void k_clip_finish(Dev d) {
  const int rpar = *d.parity;
  const int targets = int(min(int64_t(d.status[kResidual]), d.cap.frontier));
  const int hidden = min(d.sc[kClipHidden], d.hidden_cap);
  const int layer = d.status[kPass];
  V2 *next_v = d.res_v[rpar ^ 1];
  int *next_n = d.res_n[rpar ^ 1], *next_src = d.res_src[rpar ^ 1];
  long long restored = 0;
  int most_hidden = 0;
  for (int64_t i = tid(); i < int64_t(targets) + hidden; i += stride()) {
    if (d.status[kError] != 0) break;
    const V2 *src;
    int n, source;
    if (i < targets) {
      most_hidden = max(most_hidden, d.target_hidden[i]);
      if (d.target_visible[i] > 0) continue;
      src = piece_at(d.res_v[rpar], i);
      n = d.res_n[rpar][i];
      source = d.res_src[rpar][i];
      ++restored;
    } else {
      const int h = int(i - targets), target = d.hid_target[h];
      if (d.target_visible[target] == 0) continue;
      src = piece_at(d.hid_v, h);
      n = d.hid_n[h];
      source = d.res_src[rpar][target];
    }
    const int slot = reserve(&d.status[kNextResidual], 1);
    if (slot >= d.cap.frontier) {
      set_error(d.status, kErrResidual);
      continue;
    }
    V2 *dst = piece_at(next_v, slot);
    for (int j = 0; j < n; ++j) dst[j] = src[j];
    next_n[slot] = n;
    next_src[slot] = source;
  }
  if (layer < d.cap.layers) {
    if (tid() == 0) count_add(&d.stats[3 * int64_t(layer)], targets);
    if (restored) count_add(&d.stats[3 * int64_t(layer) + 2], restored);
  }
  if (most_hidden) atomicMax(&d.status[kMaxHidden], most_hidden);
}

// The next layer's residual becomes current; the layer loop goes on while
// patches remain and the layer limit allows.
__global__ void k_layer_next(Dev d) {
  const int remaining = d.status[kNextResidual];
  d.status[kResidual] = remaining;
  d.status[kNextResidual] = 0;
  d.status[kPeakResidual] = max(d.status[kPeakResidual], remaining);
  *d.parity ^= 1;
  const int layer = ++d.status[kPass];
  if (remaining > 0 && layer >= d.limit && d.all_layers) set_error(d.status, kErrLayers);
  const int c = remaining > 0 && layer < d.limit && d.status[kError] == 0;
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

cudaError_t stage_device_layer(const Dev &layer_dev, SortScratch &s, TreeBuffers &source_tree,
                               TreeBuffers &residual_tree, cudaStream_t st, cudaStream_t rounds) {
  Dev d = layer_dev;
  k_retire_bounds<<<blocks(d.n), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(tree_refit(source_tree, d.src_lo, d.src_hi, st));
  k_active_bounds<<<blocks(d.cap.frontier), kBlock, 0, st>>>(d);
  note_launch();
  EDP_CHECK(tree_build(residual_tree, d.res_lo, d.res_hi, d.sc + kFrontierLive, 0, false, s, st));
  const unsigned clip_blocks = 148 * 8;
  if (d.use_handle) {
    // Inside a capture: the clipping rounds are a conditional WHILE node of
    // the graph being recorded on `st` (the layer loop's body), their body
    // recorded on `rounds`.
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    EDP_CHECK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphConditionalHandle handle;
    EDP_CHECK(cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
    d.use_inner = 1;
    d.inner_handle = handle;
    k_clip_begin<<<blocks(d.cap.frontier), kBlock, 0, st>>>(d);
    note_launch();
    EDP_CHECK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)] = {};
    cudaGraphNodeParams &params = *reinterpret_cast<cudaGraphNodeParams *>(raw);
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t loop;
    EDP_CHECK(cudaGraphAddNode(&loop, g, deps, ndeps, &params));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    EDP_CHECK(cudaStreamUpdateCaptureDependencies(st, &loop, 1, cudaStreamSetCaptureDependencies));
    EDP_CHECK(cudaStreamBeginCaptureToGraph(rounds, body, nullptr, nullptr, 0,
                                            cudaStreamCaptureModeRelaxed));
    EDP_LAUNCH_FORM(d.predicates, k_clip_round, clip_blocks, kBlock, rounds, d);
    note_launch();
    k_clip_advance<<<1, 1, 0, rounds>>>(d);
    note_launch();
    cudaError_t launched = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    cudaError_t end = cudaStreamEndCapture(rounds, &captured);
    EDP_CHECK(launched);
    EDP_CHECK(end);
  } else {
    // Eager (warm-up): the host drives the rounds.
    d.use_inner = 0;
    k_clip_begin<<<blocks(d.cap.frontier), kBlock, 0, st>>>(d);
    for (;;) {
      int more = 0;
      EDP_CHECK(cudaMemcpyAsync(&more, d.sc + kClipCondition, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
      EDP_CHECK(cudaStreamSynchronize(st));
      if (!more) break;
      EDP_LAUNCH_FORM(d.predicates, k_clip_round, clip_blocks, kBlock, st, d);
      k_clip_advance<<<1, 1, 0, st>>>(d);
      EDP_CHECK(cudaGetLastError());
    }
  }
  k_clip_finish<<<blocks(int64_t(d.cap.frontier) + d.hidden_cap), kBlock, 0, st>>>(d);
  note_launch();
  k_layer_next<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

}  // namespace edp

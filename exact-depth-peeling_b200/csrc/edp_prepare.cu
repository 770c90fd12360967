// Preparation stage: validation, welding, projection, mesh contours, contour
// segments and the source / segment hierarchies
// (warp_peel/solver.py:217-321, warp_peel/events.py:148-220).
#include "edp_internal.h"

namespace edp {
namespace {

constexpr int kBlock = 128;

__device__ inline int64_t tid() { return blockIdx.x * int64_t(blockDim.x) + threadIdx.x; }
__device__ inline int64_t stride() { return int64_t(gridDim.x) * blockDim.x; }

__global__ void k_reset(Dev d) {
  const int i = int(tid());
  if (i < kStatusSlots) d.status[i] = 0;
  if (i < kMetrics) d.metrics[i] = 0;
  if (i < kScalarCount) d.sc[i] = 0;
  if (i < kPredCounters) d.pred_counts[i] = 0;
  if (i == 0) {
    d.sc[kSourceCount] = d.n;
    d.sc[kSegmentSlots] = kSourceVertices * d.n;
    d.sc[kRayGridCells] = d.grid_size * d.grid_size;
    *d.parity = 0;
    *d.condition = 0;
  }
}

__device__ inline double det4(const double *m) {
  // Laplace expansion along the first row of a row-major 4x4 matrix.
  double s0 = m[10] * m[15] - m[11] * m[14], s1 = m[9] * m[15] - m[11] * m[13];
  double s2 = m[9] * m[14] - m[10] * m[13], s3 = m[8] * m[15] - m[11] * m[12];
  double s4 = m[8] * m[14] - m[10] * m[12], s5 = m[8] * m[13] - m[9] * m[12];
  double c0 = m[5] * s0 - m[6] * s1 + m[7] * s2;
  double c1 = m[4] * s0 - m[6] * s3 + m[7] * s4;
  double c2 = m[4] * s1 - m[5] * s3 + m[7] * s5;
  double c3 = m[4] * s2 - m[5] * s4 + m[6] * s5;
  return m[0] * c0 - m[1] * c1 + m[2] * c2 - m[3] * c3;
}

// Input validation (kernels.py:309-350): finite values, face indices in
// range, an invertible affine camera and a valid window and near plane.
__global__ void k_validate(Dev d) {
  for (int64_t i = tid(); i < max(max(d.nv, d.n), 1); i += stride()) {
    if (i < d.nv) {
      for (int j = 0; j < 3; ++j)
        if (!isfinite(d.vertices[3 * i + j])) set_error(d.status, kErrInput);
    }
    if (i < d.n) {
      for (int j = 0; j < 3; ++j) {
        int f = d.faces[3 * i + j];
        if (f < 0 || f >= d.nv) set_error(d.status, kErrInput);
      }
    }
    if (i == 0) {
      const double *m = d.camera;
      bool bad = false;
      for (int k = 0; k < 16; ++k) bad |= !isfinite(m[k]);
      for (int k = 0; k < 6; ++k) bad |= !isfinite(d.settings[k]);
      bad |= det4(m) == 0.0 || m[12] != 0.0 || m[13] != 0.0 || m[14] != 0.0 || m[15] != 1.0;
      const double *s = d.settings;
      bad |= s[2] <= s[0] || s[3] <= s[1] || s[5] <= 0.0 || (s[4] != 0.0 && s[4] != 1.0);
      if (bad) set_error(d.status, kErrInput);
      // Inverse camera by Gauss-Jordan elimination with partial pivoting.
      double a[4][8];
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c) a[r][c] = c < 4 ? m[4 * r + c] : double(c - 4 == r);
      for (int k = 0; k < 4; ++k) {
        int p = k;
        for (int r = k + 1; r < 4; ++r)
          if (fabs(a[r][k]) > fabs(a[p][k])) p = r;
        for (int c = 0; c < 8; ++c) {
          double t = a[k][c]; a[k][c] = a[p][c]; a[p][c] = t;
        }
        double piv = a[k][k];
        if (piv == 0.0) piv = 1.0;  // singular input is already flagged
        for (int c = 0; c < 8; ++c) a[k][c] /= piv;
        for (int r = 0; r < 4; ++r)
          if (r != k) {
            double f = a[r][k];
            for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
          }
      }
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) d.inverse[4 * r + c] = a[r][c + 4];
    }
  }
}

// Exact-position welding: the canonical id of a vertex is the smallest index
// with an equal position, signed zeros equal (kernels.py:269-306).  The
// reference sorts positions; an open-addressing table gives the same ids.
__device__ inline uint64_t position_hash(const double *v) {
  uint64_t h = mix64(key_bits(v[0]));
  h = mix64(h ^ key_bits(v[1]));
  return mix64(h ^ key_bits(v[2]));
}

__global__ void k_weld_insert(Dev d) {
  for (int64_t i = tid(); i < d.nv; i += stride()) {
    const double *v = d.vertices + 3 * i;
    uint32_t slot = uint32_t(position_hash(v)) & uint32_t(d.weld_mask);
    for (int probe = 0; probe <= d.weld_mask; ++probe) {
      int cur = atomicCAS(&d.weld_table[slot], -1, int(i));
      if (cur == -1) break;
      const double *w = d.vertices + 3 * int64_t(cur);
      if (w[0] == v[0] && w[1] == v[1] && w[2] == v[2]) break;
      slot = (slot + 1) & uint32_t(d.weld_mask);
    }
    atomicMin(&d.weld_min[slot], int(i));
    d.weld_slot[i] = int(slot);
  }
}

__global__ void k_weld_resolve(Dev d) {
  for (int64_t i = tid(); i < d.nv; i += stride()) d.canonical[i] = d.weld_min[d.weld_slot[i]];
}

// Camera transform, near clip, projection, depth plane, facing and window
// clip of one triangle (kernels.py:353-468).
__global__ void k_project(Dev d) {
  for (int64_t i = tid(); i < d.n; i += stride()) {
    V2 *out = d.src_v + kSourceVertices * i;
    if (d.status[kError] != 0) {
      d.src_n[i] = 0;
      d.src_lo[i] = empty_lo();
      d.src_hi[i] = empty_hi();
      d.scores[i] = Plane{0, 0, 0, 0};
      d.facing[i] = 0;
      d.clipped[i] = 0;
      continue;
    }
    const double *m = d.camera, *s = d.settings;
    double r[kSourceVertices][3];
    int count = 3;
    for (int j = 0; j < 3; ++j) {
      const double *w = d.vertices + 3 * int64_t(d.faces[3 * i + j]);
      for (int k = 0; k < 3; ++k)
        r[j][k] = m[4 * k] * w[0] + m[4 * k + 1] * w[1] + m[4 * k + 2] * w[2] + m[4 * k + 3];
      if (!isfinite(r[j][0]) || !isfinite(r[j][1]) || !isfinite(r[j][2]))
        set_error(d.status, kErrInput);
    }
    int was_clipped = 0;
    const bool persp = s[4] != 0.0;
    if (persp) {
      double ring[kSourceVertices][3];
      int c = 0;
      for (int j = 0; j < 3; ++j) {
        const double *a = r[j], *b = r[(j + 1) % 3];
        double da = a[2] - s[5], db = b[2] - s[5];
        if (da >= 0.0) {
          for (int k = 0; k < 3; ++k) ring[c][k] = a[k];
          ++c;
        } else {
          was_clipped = 1;
        }
        if ((da > 0.0 && db < 0.0) || (da < 0.0 && db > 0.0)) {
          double t = da / (da - db);
          for (int k = 0; k < 3; ++k) ring[c][k] = a[k] + t * (b[k] - a[k]);
          ++c;
        }
      }
      for (int j = 0; j < c; ++j)
        for (int k = 0; k < 3; ++k) r[j][k] = ring[j][k];
      count = c;
    }
    V2 p[kMaxVertices];
    double depth[kSourceVertices];
    int n = 0;
    for (int j = 0; j < count; ++j) {
      double invz = persp ? 1.0 / r[j][2] : 1.0;
      V2 x = v2((r[j][0] * invz - s[0]) / (s[2] - s[0]), (r[j][1] * invz - s[1]) / (s[3] - s[1]));
      n = append(p, n, x);
      depth[j] = persp ? -invz : r[j][2];
      if (x.x < 0.0 || x.x > 1.0 || x.y < 0.0 || x.y > 1.0) was_clipped = 1;
    }
    Plane score{0, 0, 0, 0};
    double det = 0.0;
    int index = 2;
    if (count >= 3) {
      for (int j = 2; j < count; ++j) {
        det = cross(p[0], p[1], p[j]);
        if (det != 0.0) {
          index = j;
          break;
        }
      }
    }
    int face = 0;
    if (det != 0.0) {
      V2 pa = p[1] - p[0], pb = p[index] - p[0];
      double s0 = ((depth[1] - depth[0]) * pb.y - (depth[index] - depth[0]) * pa.y) / det;
      double s1 = (pa.x * (depth[index] - depth[0]) - pb.x * (depth[1] - depth[0])) / det;
      score = Plane{s0, s1, depth[0] - s0 * p[0].x - s1 * p[0].y, 0.0};
      face = 1;
      if (det < 0.0) {
        face = -1;
        for (int j = 0; j < n / 2; ++j) {
          V2 t = p[j]; p[j] = p[n - 1 - j]; p[n - 1 - j] = t;
        }
      }
      const Plane window[4] = {{1.0, 0.0, 0.0, 0}, {-1.0, 0.0, 1.0, 0}, {0.0, 1.0, 0.0, 0},
                               {0.0, -1.0, 1.0, 0}};
      V2 q[kMaxVertices], rest[kMaxVertices];
      for (int w = 0; w < 4; ++w) {
        int nq, nr;
        split_at(p, n, window[w], v2(0.0, 0.0), q, nq, rest, nr);
        n = nq;
        for (int j = 0; j < n && j < kMaxVertices; ++j) p[j] = q[j];
      }
    } else {
      n = 0;
    }
    if (!isfinite(score.a) || !isfinite(score.b) || !isfinite(score.c) ||
        fabs(score.a) > 1.0e28 || fabs(score.b) > 1.0e28 || fabs(score.c) > 1.0e28)
      set_error(d.status, kErrInput);
    if (n > kSourceVertices) {
      set_error(d.status, kErrPolygon);
      n = 0;
    }
    for (int j = 0; j < n; ++j) out[j] = p[j];
    d.src_n[i] = n;
    d.scores[i] = score;
    d.facing[i] = face;
    d.clipped[i] = was_clipped;
    float4 lo, hi;
    polygon_bounds(p, n, score, lo, hi);
    d.src_lo[i] = lo;
    d.src_hi[i] = hi;
  }
}

// Undirected welded edge keys, grouped in an open-addressing table; the
// reference sorts them (kernels.py:471-492).
__global__ void k_edge_insert(Dev d) {
  for (int64_t e = tid(); e < 3 * int64_t(d.n); e += stride()) {
    d.masks[e] = 0;
    if (d.status[kError] != 0) {
      d.edge_slot[e] = -1;
      continue;
    }
    int64_t f = e / 3;
    int j = int(e % 3);
    int a = d.canonical[d.faces[3 * f + j]], b = d.canonical[d.faces[3 * f + (j + 1) % 3]];
    unsigned long long key =
        (static_cast<unsigned long long>(min(a, b)) << 32) | static_cast<unsigned>(max(a, b));
    d.edge_keys[e] = key;
    uint32_t slot = uint32_t(mix64(key)) & uint32_t(d.ekey_mask);
    for (int probe = 0; probe <= d.ekey_mask; ++probe) {
      unsigned long long cur = atomicCAS(&d.ekey_table[slot], ~0ull, key);
      if (cur == ~0ull || cur == key) break;
      slot = (slot + 1) & uint32_t(d.ekey_mask);
    }
    int k = atomicAdd(&d.ekey_count[slot], 1);
    if (k < 2) d.ekey_member[2 * slot + k] = int(e);
    d.edge_slot[e] = int(slot);
  }
}

// Contour = not exactly two oppositely directed incidences with the same
// facing: boundary, silhouette, non-manifold or inconsistent (kernels.py:495-520).
__global__ void k_edge_mark(Dev d) {
  for (int64_t e = tid(); e < 3 * int64_t(d.n); e += stride()) {
    int slot = d.edge_slot[e];
    if (slot < 0) continue;
    bool contour = true;
    if (d.ekey_count[slot] == 2) {
      int e0 = d.ekey_member[2 * slot], e1 = d.ekey_member[2 * slot + 1];
      int a = d.canonical[d.faces[3 * (e0 / 3) + e0 % 3]];
      int b = d.canonical[d.faces[3 * (e1 / 3) + e1 % 3]];
      if (a != b && d.facing[e0 / 3] == d.facing[e1 / 3]) contour = false;
    }
    d.masks[e] = contour ? 1 : 0;
  }
}

// Up to eight canonical contour segments per source with endpoint depths,
// deduplicated exactly; each group keeps its per-endpoint minimum depth
// (event_kernels.py:388-480).  Grouping uses a table instead of four sorts.
__global__ void k_segments(Dev d) {
  const int64_t total = int64_t(kSourceVertices) * d.n;
  for (int64_t i = tid(); i < total; i += stride()) {
    int64_t source = i / kSourceVertices;
    int edge = int(i % kSourceVertices);
    V2 a = v2(1.0e30, 1.0e30), b = a;
    double za = 1.0e30, zb = 1.0e30;
    d.seg_slot[i] = -1;
    int n = d.src_n[source];
    if (d.status[kError] == 0 && edge < n && contour_edge(d, source, edge)) {
      const V2 *p = d.src_v + kSourceVertices * source;
      a = p[edge];
      b = p[(edge + 1) % n];
      if (less(b, a)) {
        V2 t = a; a = b; b = t;
      }
      Plane sc = d.scores[source];
      za = value(sc, a);
      zb = value(sc, b);
      // Publish the endpoints before the slot can be seen by other threads.
      d.slot_a[i] = a;
      d.slot_b[i] = b;
      __threadfence();
      uint64_t h = mix64(key_bits(a.x));
      h = mix64(h ^ key_bits(a.y));
      h = mix64(h ^ key_bits(b.x));
      h = mix64(h ^ key_bits(b.y));
      uint32_t slot = uint32_t(h) & uint32_t(d.seg_mask);
      for (int probe = 0; probe <= d.seg_mask; ++probe) {
        int cur = atomicCAS(&d.seg_table[slot], -1, int(i));
        if (cur == -1) break;
        V2 ca = v2(__ldcg(&d.slot_a[cur].x), __ldcg(&d.slot_a[cur].y));
        V2 cb = v2(__ldcg(&d.slot_b[cur].x), __ldcg(&d.slot_b[cur].y));
        if (ca == a && cb == b) break;
        slot = (slot + 1) & uint32_t(d.seg_mask);
      }
      atomicMin(&d.seg_min[slot], int(i));
      atomic_min_double(&d.seg_za[slot], za);
      atomic_min_double(&d.seg_zb[slot], zb);
      d.seg_slot[i] = int(slot);
    } else {
      d.slot_a[i] = a;
      d.slot_b[i] = b;
    }
  }
}

// The first slot of each group represents it (event_kernels.py:440-501).
// Each member whose endpoint depth is the group's minimum offers its source,
// the smallest of which the exact depth tests evaluate.
__global__ void k_segment_flags(Dev d) {
  const int64_t total = int64_t(kSourceVertices) * d.n;
  for (int64_t i = tid(); i < total; i += stride()) {
    const int slot = d.seg_slot[i];
    if (slot >= 0) {
      const int source = int(i / kSourceVertices);
      const Plane sc = d.scores[source];
      if (value(sc, d.slot_a[i]) == d.seg_za[slot]) atomicMin(&d.seg_srca[slot], source);
      if (value(sc, d.slot_b[i]) == d.seg_zb[slot]) atomicMin(&d.seg_srcb[slot], source);
    }
    const bool first = slot >= 0 && d.seg_min[slot] == int(i);
    d.seg_flag[i] = first ? 1 : 0;
    count_add(&d.metrics[kUniqueContours], first ? 1 : 0);
  }
}

// Representatives, compacted in slot order (seg_pos is the scan of seg_flag),
// with their near depths and padded boxes.
__global__ void k_segment_compact(Dev d) {
  const int64_t total = int64_t(kSourceVertices) * d.n;
  for (int64_t i = tid(); i < total; i += stride()) {
    if (!d.seg_flag[i]) continue;
    const int c = d.seg_pos[i], slot = d.seg_slot[i];
    const V2 a = d.slot_a[i], b = d.slot_b[i];
    const double za = d.seg_za[slot], zb = d.seg_zb[slot];
    const double pz = 2.0e-7 * fmax(1.0, fmax(fabs(za), fabs(zb)));
    d.seg_a[c] = a;
    d.seg_b[c] = b;
    d.seg_near[c] = v2(za, zb);
    // Every group has a member attaining each minimum (the same binary64
    // expression is evaluated again); the representative's own source
    // stands in should none have been recorded.
    const int own = int(i / kSourceVertices);
    int2 near_src = make_int2(d.seg_srca[slot], d.seg_srcb[slot]);
    if (near_src.x < 0 || near_src.x >= d.n) near_src.x = own;
    if (near_src.y < 0 || near_src.y >= d.n) near_src.y = own;
    d.seg_near_src[c] = near_src;
    const Plane pa = d.scores[near_src.x], pb = d.scores[near_src.y];
    d.seg_near_mag[c] = v2(fabs(pa.a * a.x) + fabs(pa.b * a.y) + fabs(pa.c),
                           fabs(pb.a * b.x) + fabs(pb.b * b.y) + fabs(pb.c));
    // The welded mesh vertex at each end: the representative's polygon is its
    // triangle's projection (unclipped; reversed when back-facing), so its
    // vertex j is the face's vertex j, or 2 - j.
    int2 vid = make_int2(-1, -1);
    if (!d.clipped[own] && d.src_n[own] == 3) {
      const V2 *p = d.src_v + int64_t(kSourceVertices) * own;
      for (int j = 0; j < 3; ++j) {
        const int v = d.canonical[d.faces[3 * int64_t(own) + (d.facing[own] < 0 ? 2 - j : j)]];
        if (p[j] == a) vid.x = v;
        if (p[j] == b) vid.y = v;
      }
    }
    d.seg_vid[c] = vid;
    d.seg_lo[c] = make_float4(float(fmin(a.x, b.x) - 2.0e-7), float(fmin(a.y, b.y) - 2.0e-7),
                              float(fmin(za, zb) - pz), 0.f);
    d.seg_hi[c] = make_float4(float(fmax(a.x, b.x) + 2.0e-7), float(fmax(a.y, b.y) + 2.0e-7),
                              float(fmax(za, zb) + pz), 0.f);
  }
}

// Seed the frontier with every projected source, in source order; empty
// sources keep size 0 and are skipped by the subdivision (frontier.py:15-42).
__global__ void k_seed(Dev d) {
  const bool fits = int64_t(d.n) <= d.cap.frontier;
  for (int64_t i = tid(); fits && i < d.n; i += stride()) {
    int n = d.status[kError] == 0 ? d.src_n[i] : 0;
    V2 *dst = d.fv[0] + int64_t(kMaxVertices) * i;
    const V2 *src = d.src_v + kSourceVertices * i;
    for (int j = 0; j < n; ++j) dst[j] = src[j];
    d.fn[0][i] = n;
    d.fsrc[0][i] = int(i);
    d.fcur[0][i] = 0;  // first contour leaf not yet met
  }
  if (tid() == 0) {
    if (!fits) set_error(d.status, kErrResidual);
    d.status[kResidual] = fits ? d.n : 0;
    d.status[kPeakResidual] = d.status[kResidual];
    d.sc[kFrontierNext] = 0;
    d.sc[kDeferred] = 0;
    d.sc[kDeferredNext] = 0;
  }
}

__global__ void k_loop_condition(Dev d) {
  int c = d.status[kResidual] > 0 && d.status[kError] == 0;
  *d.condition = c;
  if (d.use_handle) cudaGraphSetConditional(d.cond_handle, unsigned(c));
}

unsigned blocks(int64_t n) {
  int64_t g = ceil_div(n > 0 ? n : 1, kBlock);
  return unsigned(g < 148 * 16 ? g : 148 * 16);
}

}  // namespace

cudaError_t stage_prepare_common(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                                 cudaStream_t st) {
  k_reset<<<1, 32, 0, st>>>(d);
  note_launch();
  EDP_CHECK(cudaMemsetAsync(d.weld_table, 0xff, sizeof(int) * (int64_t(d.weld_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.weld_min, 0x7f, sizeof(int) * (int64_t(d.weld_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.ekey_table, 0xff, sizeof(unsigned long long) * (int64_t(d.ekey_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.ekey_count, 0, sizeof(int) * (int64_t(d.ekey_mask) + 1), st));
  k_validate<<<blocks(std::max(d.nv, d.n)), kBlock, 0, st>>>(d);
  note_launch();
  if (d.nv > 0) {
    k_weld_insert<<<blocks(d.nv), kBlock, 0, st>>>(d);
    note_launch();
    k_weld_resolve<<<blocks(d.nv), kBlock, 0, st>>>(d);
    note_launch();
  }
  if (d.n > 0) {
    k_project<<<blocks(d.n), kBlock, 0, st>>>(d);
    note_launch();
    k_edge_insert<<<blocks(3 * int64_t(d.n)), kBlock, 0, st>>>(d);
    note_launch();
    k_edge_mark<<<blocks(3 * int64_t(d.n)), kBlock, 0, st>>>(d);
    note_launch();
  }
  EDP_CHECK(tree_build(source_tree, d.src_lo, d.src_hi, nullptr, d.n, false, s, st));
  return cudaGetLastError();
}

cudaError_t stage_prepare(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                          TreeBuffers &seg_tree, cudaStream_t st) {
  EDP_CHECK(stage_prepare_common(d, s, source_tree, st));
  EDP_CHECK(cudaMemsetAsync(d.seg_table, 0xff, sizeof(int) * (int64_t(d.seg_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.seg_min, 0x7f, sizeof(int) * (int64_t(d.seg_mask) + 1), st));
  // 0x7f bytes are 1.38e306 as binary64: above every finite depth we store.
  EDP_CHECK(cudaMemsetAsync(d.seg_za, 0x7f, sizeof(double) * (int64_t(d.seg_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.seg_zb, 0x7f, sizeof(double) * (int64_t(d.seg_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.seg_srca, 0x7f, sizeof(int) * (int64_t(d.seg_mask) + 1), st));
  EDP_CHECK(cudaMemsetAsync(d.seg_srcb, 0x7f, sizeof(int) * (int64_t(d.seg_mask) + 1), st));
  if (d.n > 0) {
    k_segments<<<blocks(kSourceVertices * int64_t(d.n)), kBlock, 0, st>>>(d);
    note_launch();
    k_segment_flags<<<blocks(kSourceVertices * int64_t(d.n)), kBlock, 0, st>>>(d);
    note_launch();
    EDP_CHECK(scan_exclusive(d.seg_flag, d.seg_pos, d.sc + kSegmentSlots, kSourceVertices * d.n,
                             d.sc + kSegmentCount, s, st));
    k_segment_compact<<<blocks(kSourceVertices * int64_t(d.n)), kBlock, 0, st>>>(d);
    note_launch();
  }
  EDP_CHECK(tree_build(seg_tree, d.seg_lo, d.seg_hi, d.sc + kSegmentCount, 0, false, s, st));
  k_seed<<<blocks(d.n), kBlock, 0, st>>>(d);
  note_launch();
  k_loop_condition<<<1, 1, 0, st>>>(d);
  note_launch();
  return cudaGetLastError();
}

}  // namespace edp

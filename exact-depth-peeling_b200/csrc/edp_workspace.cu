// Workspace lifetime, stage orchestration, CUDA graph capture with a device
// conditional loop, and the C ABI declared in include/edp.h.
#include <cstring>
#include <initializer_list>
#include <vector>

#include "../../include/edp.h"
#include "edp_internal.h"

#include <algorithm>
#include <cmath>

using namespace edp;

namespace {
// Stages that can be replayed alone after a full extraction, each from its own
// captured graph: preparation, boundary vertices + point hierarchy, and the
// noding / emission / lifting kernel.
constexpr int kStages = 3;
}  // namespace

struct edp_peeler {
  int method = 0;  // 0 = EventPeeler, 1 = DevicePeeler
  Dev d{};
  cudaStream_t stream = nullptr;
  cudaStream_t body_stream = nullptr;
  cudaStream_t round_stream = nullptr;  // records the DevicePeeler's clipping rounds
  SortScratch scratch;
  TreeBuffers source_tree, seg_tree, point_tree;  // seg_tree holds contours for DevicePeeler
  TreeBuffers residual_tree;
  std::vector<void *> allocations;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool warmed = false;
  int device = 0;
  cudaGraphExec_t stage_exec[kStages] = {};
  // Kernel nodes of the last capture: outside the subdivision loop, and in
  // one iteration of its body.
  int64_t kernels_outside = 0, kernels_per_round = 0;
  // Stage timing events recorded by the workspace's own graph (start, then
  // the end of each EDP_STAGE_*); created with the graph.
  cudaEvent_t marks[EDP_STAGE_COUNT + 1] = {};
  bool marked = false;
  int64_t bytes = 0;  // device bytes of the pools allocated through alloc()
};

namespace {

thread_local int g_last_cuda = 0;
thread_local const char *g_last_site = "";

int cuda_fail(cudaError_t e, const char *site) { return edp::record_cuda_failure(e, site); }

#define EDP_STR2(x) #x
#define EDP_STR(x) EDP_STR2(x)
#define EDP_TRY(call)                                                              \
  do {                                                                             \
    cudaError_t e__ = (call);                                                      \
    if (e__ != cudaSuccess) return cuda_fail(e__, __FILE__ ":" EDP_STR(__LINE__)); \
  } while (0)

template <class T>
cudaError_t alloc(edp_peeler *p, T **ptr, int64_t count) {
  if (count < 1) count = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(ptr), sizeof(T) * size_t(count));
  if (e == cudaSuccess) {
    p->allocations.push_back(*ptr);
    p->bytes += int64_t(sizeof(T)) * count;
    e = cudaMemset(*ptr, 0, sizeof(T) * size_t(count));
  }
  return e;
}

int table_mask(int64_t entries) { return int(pow2_at_least(2 * (entries > 0 ? entries : 1)) - 1); }

bool caps_valid(const Caps &c) {
  const int64_t v[] = {c.frontier, c.regions, c.hits, c.vertices, c.triangles, c.rounds, c.layers,
                       c.edge_vertices};
  for (int64_t x : v)
    if (x < 1 || x > (int64_t(1) << 30)) return false;
  return c.edge_vertices <= 128;
}

// Buffers both peelers use: control, welding, sources, mesh edges, output
// polygons, boundary noding, triangles, the source and point hierarchies.
cudaError_t allocate_shared(edp_peeler *p) {
  Dev &d = p->d;
  const int64_t n = d.n, nv = d.nv, R = d.cap.regions, E = d.cap.vertices, T = d.cap.triangles,
                S = int64_t(kSourceVertices) * n;
  EDP_CHECK(alloc(p, &d.status, kStatusSlots));
  EDP_CHECK(alloc(p, &d.metrics, kMetrics));
  EDP_CHECK(alloc(p, &d.pred_counts, kPredCounters));
  EDP_CHECK(alloc(p, &d.sc, kScalarCount));
  EDP_CHECK(alloc(p, &d.parity, 1));
  EDP_CHECK(alloc(p, &d.condition, 1));
  EDP_CHECK(alloc(p, &d.inverse, 16));
  d.weld_mask = table_mask(nv);
  EDP_CHECK(alloc(p, &d.canonical, nv));
  EDP_CHECK(alloc(p, &d.weld_slot, nv));
  EDP_CHECK(alloc(p, &d.weld_table, int64_t(d.weld_mask) + 1));
  EDP_CHECK(alloc(p, &d.weld_min, int64_t(d.weld_mask) + 1));
  EDP_CHECK(alloc(p, &d.src_v, S));
  EDP_CHECK(alloc(p, &d.src_n, n));
  EDP_CHECK(alloc(p, &d.scores, n));
  EDP_CHECK(alloc(p, &d.facing, n));
  EDP_CHECK(alloc(p, &d.clipped, n));
  EDP_CHECK(alloc(p, &d.src_lo, n));
  EDP_CHECK(alloc(p, &d.src_hi, n));
  d.ekey_mask = table_mask(3 * n);
  EDP_CHECK(alloc(p, &d.ekey_table, int64_t(d.ekey_mask) + 1));
  EDP_CHECK(alloc(p, &d.ekey_count, int64_t(d.ekey_mask) + 1));
  EDP_CHECK(alloc(p, &d.ekey_member, 2 * (int64_t(d.ekey_mask) + 1)));
  EDP_CHECK(alloc(p, &d.edge_slot, 3 * n));
  EDP_CHECK(alloc(p, &d.masks, 3 * n));
  EDP_CHECK(alloc(p, &d.edge_keys, 3 * n));
  EDP_CHECK(alloc(p, &d.out_v, R * kMaxVertices));
  EDP_CHECK(alloc(p, &d.out_n, R));
  EDP_CHECK(alloc(p, &d.out_src, R));
  EDP_CHECK(alloc(p, &d.out_layer, R));
  EDP_CHECK(alloc(p, &d.order_keys, R));
  EDP_CHECK(alloc(p, &d.order_keys_tmp, R));
  EDP_CHECK(alloc(p, &d.order, R));
  EDP_CHECK(alloc(p, &d.order_tmp, R));
  EDP_CHECK(alloc(p, &d.counts, R));
  EDP_CHECK(alloc(p, &d.offsets, R));
  EDP_CHECK(alloc(p, &d.bverts, E));
  EDP_CHECK(alloc(p, &d.blayers, E));
  EDP_CHECK(alloc(p, &d.uverts, E));
  d.point_mask = table_mask(E);
  EDP_CHECK(alloc(p, &d.point_table, int64_t(d.point_mask) + 1));
  // Source and segment grids: about sqrt(N) / 1.5 cells per axis (a power of
  // two in [32, 512]).  Layered point grid: about 2 sqrt(N) cells per axis (a
  // power of two in [32, 1024]; a front layer holds ~14 distinct boundary
  // points per face, so its cells hold a few each), rows for as many layers as
  // 256 N cells allow, at least 16M and at most 64M cells.
  {
    int g = 32;
    while (g < 512 && double(2 * g) * 1.5 <= std::sqrt(double(n > 0 ? n : 1))) g *= 2;
    d.grid_size = g;
    g = 32;
    while (g < 1024 && double(2 * g) <= 2.0 * std::sqrt(double(n > 0 ? n : 1))) g *= 2;
    d.point_grid = g;
    const int64_t per_layer = int64_t(g) * g;
    const int64_t budget =
        std::max(int64_t(1) << 24, std::min(int64_t(1) << 26, int64_t(256) * (n > 0 ? n : 1)));
    d.grid_layers = int(std::min<int64_t>(d.cap.layers, std::max<int64_t>(1, budget / per_layer)));
    EDP_CHECK(alloc(p, &d.cell_count, d.grid_layers * per_layer));
    EDP_CHECK(alloc(p, &d.cell_start, d.grid_layers * per_layer + 1));
    EDP_CHECK(alloc(p, &d.grid_pts, E));
    EDP_CHECK(alloc(p, &d.heavy_polygons, R));
  }
  EDP_CHECK(alloc(p, &d.pt_lo, E));
  EDP_CHECK(alloc(p, &d.pt_hi, E));
  EDP_CHECK(alloc(p, &d.tri_uv, 3 * T));
  EDP_CHECK(alloc(p, &d.tri_world, 9 * T));
  EDP_CHECK(alloc(p, &d.tri_src, T));
  EDP_CHECK(alloc(p, &d.tri_layer, T));
  EDP_CHECK(tree_alloc(p->source_tree, n));
  EDP_CHECK(tree_alloc(p->point_tree, E));
  d.source_tree = p->source_tree.tree();
  d.point_tree = p->point_tree.tree();
  return cudaSuccess;
}

cudaError_t allocate_scratch(edp_peeler *p, int64_t largest_sort, int64_t largest_scan) {
  p->scratch.tiles = ceil_div(largest_sort, kSortTile);
  p->scratch.scan_tiles = ceil_div(largest_scan, kScanTile);
  EDP_CHECK(alloc(p, &p->scratch.hist, 256 * p->scratch.tiles));
  EDP_CHECK(alloc(p, &p->scratch.totals, 256));
  EDP_CHECK(alloc(p, &p->scratch.partials, p->scratch.scan_tiles));
  return cudaSuccess;
}

cudaError_t allocate_event(edp_peeler *p) {
  Dev &d = p->d;
  const int64_t n = d.n, F = d.cap.frontier, R = d.cap.regions, H = d.cap.hits,
                E = d.cap.vertices, S = int64_t(kSourceVertices) * n;
  EDP_CHECK(allocate_shared(p));
  d.seg_mask = table_mask(S);
  EDP_CHECK(alloc(p, &d.slot_a, S));
  EDP_CHECK(alloc(p, &d.slot_b, S));
  EDP_CHECK(alloc(p, &d.seg_flag, S));
  EDP_CHECK(alloc(p, &d.seg_pos, S));
  EDP_CHECK(alloc(p, &d.seg_a, S));
  EDP_CHECK(alloc(p, &d.seg_b, S));
  EDP_CHECK(alloc(p, &d.seg_near, S));
  EDP_CHECK(alloc(p, &d.seg_near_src, S));
  EDP_CHECK(alloc(p, &d.seg_near_mag, S));
  EDP_CHECK(alloc(p, &d.seg_vid, S));
  EDP_CHECK(alloc(p, &d.seg_lo, S));
  EDP_CHECK(alloc(p, &d.seg_hi, S));
  EDP_CHECK(alloc(p, &d.seg_slot, S));
  EDP_CHECK(alloc(p, &d.seg_za, int64_t(d.seg_mask) + 1));
  EDP_CHECK(alloc(p, &d.seg_zb, int64_t(d.seg_mask) + 1));
  EDP_CHECK(alloc(p, &d.seg_srca, int64_t(d.seg_mask) + 1));
  EDP_CHECK(alloc(p, &d.seg_srcb, int64_t(d.seg_mask) + 1));
  EDP_CHECK(alloc(p, &d.seg_table, int64_t(d.seg_mask) + 1));
  EDP_CHECK(alloc(p, &d.seg_min, int64_t(d.seg_mask) + 1));
  for (int k = 0; k < 2; ++k) {
    EDP_CHECK(alloc(p, &d.fv[k], F * kMaxVertices));
    EDP_CHECK(alloc(p, &d.fn[k], F));
    EDP_CHECK(alloc(p, &d.fsrc[k], F));
    EDP_CHECK(alloc(p, &d.fcur[k], F));
  }
  EDP_CHECK(alloc(p, &d.parents, R));
  EDP_CHECK(alloc(p, &d.reps, R));
  EDP_CHECK(alloc(p, &d.samples, R));
  EDP_CHECK(alloc(p, &d.groups, R));
  EDP_CHECK(alloc(p, &d.sample_slot, R));
  d.sample_mask = table_mask(R);
  EDP_CHECK(alloc(p, &d.sample_table, int64_t(d.sample_mask) + 1));
  EDP_CHECK(alloc(p, &d.sample_min, int64_t(d.sample_mask) + 1));
  EDP_CHECK(alloc(p, &d.cell_bounds, 4 * 1024));
  EDP_CHECK(alloc(p, &d.cell_min, 1024));
  EDP_CHECK(alloc(p, &d.cell_valid, 1024));
  EDP_CHECK(alloc(p, &d.heavy_beams, 1024));
  EDP_CHECK(alloc(p, &d.heavy_queries, R));
  {
    const int64_t cells = int64_t(d.grid_size) * d.grid_size;
    EDP_CHECK(alloc(p, &d.ray_count, cells));
    EDP_CHECK(alloc(p, &d.ray_start, cells + 1));
    EDP_CHECK(alloc(p, &d.ray_entries, int64_t(kRayCells) * (n > 0 ? n : 1)));
    EDP_CHECK(alloc(p, &d.ray_big, n > 0 ? n : 1));
    EDP_CHECK(alloc(p, &d.leaf_of, n > 0 ? n : 1));
    EDP_CHECK(alloc(p, &d.seg_count, cells));
    EDP_CHECK(alloc(p, &d.seg_start, cells + 1));
    EDP_CHECK(alloc(p, &d.seg_entries, int64_t(kSegCells) * S));
    EDP_CHECK(alloc(p, &d.seg_big, S));
  }
  EDP_CHECK(alloc(p, &d.group_counts, R));
  EDP_CHECK(alloc(p, &d.group_offsets, R));
  EDP_CHECK(alloc(p, &d.group_fill, R));
  EDP_CHECK(alloc(p, &d.rank_defer, R));
  EDP_CHECK(alloc(p, &d.deep_groups, R));
  d.ray_defer_cap = H / 8 + 1024;
  EDP_CHECK(alloc(p, &d.ray_defer, d.ray_defer_cap));
  EDP_CHECK(alloc(p, &d.tasks, E));
  EDP_CHECK(alloc(p, &d.owners, E));
  EDP_CHECK(alloc(p, &d.starts, E));
  EDP_CHECK(alloc(p, &d.ends, E));
  EDP_CHECK(alloc(p, &d.partners, E));
  if (d.merge_regions) {
    EDP_CHECK(alloc(p, &d.merge_choice, R));
    EDP_CHECK(alloc(p, &d.merged_v, R * kMaxVertices));
    EDP_CHECK(alloc(p, &d.merged_n, R));
    EDP_CHECK(alloc(p, &d.merged_src, R));
    EDP_CHECK(alloc(p, &d.merged_layer, R));
  }
  d.edge_hash_mask = table_mask(E);
  EDP_CHECK(alloc(p, &d.edge_hash, int64_t(d.edge_hash_mask) + 1));
  EDP_CHECK(alloc(p, &d.hit_depth, H));
  EDP_CHECK(alloc(p, &d.hit_src, H));
  EDP_CHECK(alloc(p, &d.hit_group, H));
  EDP_CHECK(alloc(p, &d.hit_ids, H));
  EDP_CHECK(alloc(p, &d.hit_ids_tmp, H));
  EDP_CHECK(alloc(p, &d.hkeys, H));
  EDP_CHECK(alloc(p, &d.hkeys_tmp, H));
  EDP_CHECK(tree_alloc(p->seg_tree, S));
  d.seg_tree = p->seg_tree.tree();
  int64_t largest = H;
  for (int64_t v : {p->point_tree.leaves_cap, p->seg_tree.leaves_cap, p->source_tree.leaves_cap, R})
    largest = v > largest ? v : largest;
  int64_t scan = R > E ? R : E;
  scan = S > scan ? S : scan;  // the segment-slot compaction
  scan = std::max(scan, int64_t(d.grid_layers) * d.point_grid * d.point_grid);
  return allocate_scratch(p, largest, scan);
}

cudaError_t allocate_device(edp_peeler *p) {
  Dev &d = p->d;
  const int64_t n = d.n, F = d.cap.frontier, R = d.cap.regions, E = d.cap.vertices;
  // Live clipping pieces end as visible (at most R) or hidden pieces, so
  // R + F slots hold every round's queue.  The hidden pool also holds the
  // pieces of targets that end up hidden whole (dropped when the layer
  // finishes), so it takes R + F slots too.
  d.work_cap = int(std::min<int64_t>(R + F, (int64_t(1) << 31) - 1));
  d.hidden_cap = d.work_cap;
  EDP_CHECK(allocate_shared(p));
  EDP_CHECK(alloc(p, &d.contour_lo, n));
  EDP_CHECK(alloc(p, &d.contour_hi, n));
  EDP_CHECK(alloc(p, &d.ranks, n));
  for (int k = 0; k < 2; ++k) {
    EDP_CHECK(alloc(p, &d.res_v[k], F * kMaxVertices));
    EDP_CHECK(alloc(p, &d.res_n[k], F));
    EDP_CHECK(alloc(p, &d.res_src[k], F));
  }
  EDP_CHECK(alloc(p, &d.res_lo, F));
  EDP_CHECK(alloc(p, &d.res_hi, F));
  for (int k = 0; k < 2; ++k) {
    EDP_CHECK(alloc(p, &d.work_v[k], int64_t(d.work_cap) * kMaxVertices));
    EDP_CHECK(alloc(p, &d.work_n[k], d.work_cap));
    EDP_CHECK(alloc(p, &d.work_target[k], d.work_cap));
    EDP_CHECK(alloc(p, &d.work_cursor[k], d.work_cap));
  }
  EDP_CHECK(alloc(p, &d.hid_v, int64_t(d.hidden_cap) * kMaxVertices));
  EDP_CHECK(alloc(p, &d.hid_n, d.hidden_cap));
  EDP_CHECK(alloc(p, &d.hid_target, d.hidden_cap));
  EDP_CHECK(alloc(p, &d.target_visible, F));
  EDP_CHECK(alloc(p, &d.target_hidden, F));
  EDP_CHECK(alloc(p, &d.stats, 3 * d.cap.layers));
  EDP_CHECK(tree_alloc(p->seg_tree, n));  // the contour hierarchy
  EDP_CHECK(tree_alloc(p->residual_tree, F));
  d.contour_tree = p->seg_tree.tree();
  d.residual_tree = p->residual_tree.tree();
  int64_t largest = R;
  for (int64_t v : {p->point_tree.leaves_cap, p->seg_tree.leaves_cap, p->source_tree.leaves_cap,
                    p->residual_tree.leaves_cap})
    largest = v > largest ? v : largest;
  return allocate_scratch(p, largest,
                         std::max({R, E, int64_t(d.grid_layers) * d.point_grid * d.point_grid}));
}

// Stage sequence of each peeler.  The loop body runs while the device sets
// the condition: subdivision rounds (EventPeeler) or layer passes
// (DevicePeeler).
cudaError_t run_prepare(edp_peeler *p, const Dev &d, cudaStream_t st) {
  return p->method == 0 ? stage_prepare(d, p->scratch, p->source_tree, p->seg_tree, st)
                        : stage_device_prepare(d, p->scratch, p->source_tree, p->seg_tree, st);
}
cudaError_t run_body(edp_peeler *p, const Dev &d, cudaStream_t st) {
  return p->method == 0 ? stage_step(d, st)
                        : stage_device_layer(d, p->scratch, p->source_tree, p->residual_tree, st,
                                             p->round_stream);
}
cudaError_t run_finish(edp_peeler *p, const Dev &d, cudaStream_t st) {
  if (p->method == 0) {
    EDP_CHECK(stage_rank(d, p->scratch, st));
  } else {  // its finish is timed as the assignment stage
    EDP_CHECK(stage_mark(EDP_STAGE_RANK_HIT_SORT, st));
    EDP_CHECK(stage_device_finish(d, st));
    EDP_CHECK(stage_mark(EDP_STAGE_RANK_MERGE, st));
  }
  EDP_CHECK(stage_mesh_index(d, p->scratch, p->point_tree, st));
  EDP_CHECK(stage_mesh_emit(d, st));
  return stage_mark(EDP_STAGE_COUNT - 1, st);
}

// The whole extraction, recorded on `st`.  With `graph` the loop becomes a
// conditional WHILE node of the graph being captured on `st`; otherwise the
// host drives the loop (used by warm-up only).
int enqueue(edp_peeler *p, cudaStream_t st, bool graph) {
  Dev d = p->d;
  if (!graph) {
    d.use_handle = 0;
    EDP_TRY(run_prepare(p, d, st));
    while (true) {
      int cond = 0;
      EDP_TRY(cudaMemcpyAsync(&cond, d.condition, sizeof(int), cudaMemcpyDeviceToHost, st));
      EDP_TRY(cudaStreamSynchronize(st));
      if (!cond) break;
      EDP_TRY(run_body(p, d, st));
    }
    EDP_TRY(run_finish(p, d, st));
    return EDP_OK;
  }
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  EDP_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
  if (cs != cudaStreamCaptureStatusActive) return EDP_ERR_STATE;
  cudaGraphConditionalHandle handle;
  EDP_TRY(cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
  d.use_handle = 1;
  d.cond_handle = handle;
  const int64_t first_launch = launch_count();
  EDP_TRY(stage_mark(-1, st));
  EDP_TRY(run_prepare(p, d, st));
  EDP_TRY(stage_mark(EDP_STAGE_PREPARE, st));
  EDP_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)] = {};
  cudaGraphNodeParams &params = *reinterpret_cast<cudaGraphNodeParams *>(raw);
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = handle;
  params.conditional.type = cudaGraphCondTypeWhile;
  params.conditional.size = 1;
  cudaGraphNode_t loop;
  EDP_TRY(cudaGraphAddNode(&loop, g, deps, ndeps, &params));
  cudaGraph_t body = params.conditional.phGraph_out[0];
  EDP_TRY(cudaStreamUpdateCaptureDependencies(st, &loop, 1, cudaStreamSetCaptureDependencies));
  EDP_TRY(cudaStreamBeginCaptureToGraph(p->body_stream, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeRelaxed));
  const int64_t body_first = launch_count();
  cudaError_t step = run_body(p, d, p->body_stream);
  const int64_t per_round = launch_count() - body_first;
  cudaGraph_t captured = nullptr;
  cudaError_t end = cudaStreamEndCapture(p->body_stream, &captured);
  EDP_TRY(step);
  EDP_TRY(end);
  EDP_TRY(stage_mark(EDP_STAGE_SUBDIVIDE, st));
  EDP_TRY(run_finish(p, d, st));
  p->kernels_per_round = per_round;
  p->kernels_outside = launch_count() - first_launch - per_round;
  return EDP_OK;
}

int check_inputs(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                 const double *camera, const double *settings, void *stream) {
  if (nv < 0 || nf < 0 || nv >= (int64_t(1) << 31) || nf >= (int64_t(1) << 28))
    return EDP_ERR_ARGUMENT;
  if ((nv > 0 && !vertices) || (nf > 0 && !faces) || !camera || !settings || !stream)
    return EDP_ERR_ARGUMENT;
  return EDP_OK;
}

}  // namespace

int edp::record_cuda_failure(cudaError_t e, const char *site) {
  g_last_cuda = int(e);
  g_last_site = site;
  return EDP_ERR_CUDA;
}

extern "C" {

void edp_event_default_capacities(int64_t nf, edp_event_capacities *cap) {
  int64_t n = nf > 16 ? nf : 16;
  cap->frontier = 4 * n;
  cap->regions = 8 * n;
  cap->hits = 32 * n;
  cap->vertices = 32 * n;
  cap->triangles = 32 * n;
  cap->rounds = 4096;
  cap->layers = n;
  cap->edge_vertices = 128;
}

void edp_device_default_capacities(int64_t nf, edp_device_capacities *cap) {
  int64_t n = nf > 16 ? nf : 16;
  cap->residual = 4 * n;
  cap->polygons = 16 * n;
  cap->vertices = 96 * n;
  cap->triangles = 64 * n;
  cap->workers = n < 4096 ? n : 4096;
  cap->pieces_per_worker = n <= 8192 ? 512 : 2048;
  cap->layers = 128;
  cap->edge_vertices = 128;
}

int edp_event_create(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                     const double *camera, const double *settings,
                     const edp_event_capacities *cap, const edp_event_options *opt, void *stream,
                     edp_peeler **out) {
  if (!out) return EDP_ERR_ARGUMENT;
  *out = nullptr;
  int rc = check_inputs(vertices, nv, faces, nf, camera, settings, stream);
  if (rc) return rc;
  edp_event_capacities c;
  if (cap)
    c = *cap;
  else
    edp_event_default_capacities(nf, &c);
  edp_event_options o{0, 1, 1, 0};
  if (opt) o = *opt;
  Caps caps{c.frontier, c.regions, c.hits, c.vertices, c.triangles, c.rounds, c.layers,
            c.edge_vertices};
  if (!caps_valid(caps)) return EDP_ERR_ARGUMENT;
  if (o.layers < 0 || o.layers > c.layers) return EDP_ERR_ARGUMENT;
  edp_peeler *p = new edp_peeler();
  p->method = 0;
  p->stream = static_cast<cudaStream_t>(stream);
  Dev &d = p->d;
  d.vertices = vertices;
  d.faces = faces;
  d.camera = camera;
  d.settings = settings;
  d.nv = int(nv);
  d.n = int(nf);
  d.cap = caps;
  d.limit = o.layers ? o.layers : int(c.layers);
  d.all_layers = o.layers == 0;
  d.share_regions = o.share_regions != 0;
  d.propagate_ranks = o.propagate_ranks != 0;
  d.merge_regions = o.merge_regions != 0;
  d.predicates = EDP_PREDICATES_FILTERED64;
  d.aux_stream = nullptr;
  d.step_budget = 48;
  d.subdivide_blocks = 8;
  d.heavy_noding_work = 1024;
  d.clip_budget = 32;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->body_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->round_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) d.aux_stream = p->round_stream;
  if (e == cudaSuccess) e = allocate_event(p);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    edp_destroy(p);
    g_last_cuda = int(e);
    return e == cudaErrorMemoryAllocation ? EDP_ERR_MEMORY : EDP_ERR_CUDA;
  }
  *out = p;
  return EDP_OK;
}

int edp_device_create(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                      const double *camera, const double *settings,
                      const edp_device_capacities *cap, int32_t layers, void *stream,
                      edp_peeler **out) {
  if (!out) return EDP_ERR_ARGUMENT;
  *out = nullptr;
  int rc = check_inputs(vertices, nv, faces, nf, camera, settings, stream);
  if (rc) return rc;
  edp_device_capacities c;
  if (cap)
    c = *cap;
  else
    edp_device_default_capacities(nf, &c);
  // Residual patches use the frontier slot; no ray hits or round cap.
  Caps caps{c.residual, c.polygons, 1, c.vertices, c.triangles, 1, c.layers, c.edge_vertices};
  if (!caps_valid(caps) || c.workers < 1 || c.pieces_per_worker < 1 ||
      c.workers > (int64_t(1) << 24) || c.pieces_per_worker > (int64_t(1) << 20) ||
      c.workers * c.pieces_per_worker > (int64_t(1) << 30))
    return EDP_ERR_ARGUMENT;
  if (layers < 0 || layers > c.layers) return EDP_ERR_ARGUMENT;
  edp_peeler *p = new edp_peeler();
  p->method = 1;
  p->stream = static_cast<cudaStream_t>(stream);
  Dev &d = p->d;
  d.vertices = vertices;
  d.faces = faces;
  d.camera = camera;
  d.settings = settings;
  d.nv = int(nv);
  d.n = int(nf);
  d.cap = caps;
  d.limit = layers ? layers : int(c.layers);
  d.all_layers = layers == 0;
  d.workers = int(c.workers);
  d.pieces = int(c.pieces_per_worker);
  d.predicates = EDP_PREDICATES_FILTERED64;
  d.step_budget = 48;
  d.subdivide_blocks = 8;
  d.heavy_noding_work = 1024;
  d.clip_budget = 32;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->body_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->round_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = allocate_device(p);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    edp_destroy(p);
    g_last_cuda = int(e);
    return e == cudaErrorMemoryAllocation ? EDP_ERR_MEMORY : EDP_ERR_CUDA;
  }
  *out = p;
  return EDP_OK;
}

int edp_warmup(edp_peeler *p) {
  if (!p) return EDP_ERR_ARGUMENT;
  cudaStreamCaptureStatus cs;
  EDP_TRY(cudaStreamIsCapturing(p->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return EDP_ERR_STATE;
  int rc = enqueue(p, p->stream, false);
  if (rc) return rc;
  EDP_TRY(cudaStreamSynchronize(p->stream));
  p->warmed = true;
  return EDP_OK;
}

int edp_enqueue(edp_peeler *p, void *stream) {
  if (!p) return EDP_ERR_ARGUMENT;
  if (!p->warmed || static_cast<cudaStream_t>(stream) != p->stream) return EDP_ERR_STATE;
  cudaStreamCaptureStatus cs;
  EDP_TRY(cudaStreamIsCapturing(p->stream, &cs));
  if (cs != cudaStreamCaptureStatusActive) return EDP_ERR_STATE;
  return enqueue(p, p->stream, true);
}

int edp_capture(edp_peeler *p) {
  if (!p) return EDP_ERR_ARGUMENT;
  if (p->exec) return EDP_OK;
  if (!p->warmed) {
    int rc = edp_warmup(p);
    if (rc) return rc;
  }
  for (cudaEvent_t &ev : p->marks)
    if (!ev) EDP_TRY(cudaEventCreate(&ev));
  EDP_TRY(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
  set_stage_marks(p->marks);
  int rc = enqueue(p, p->stream, true);
  set_stage_marks(nullptr);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(p->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  EDP_TRY(e);
  p->graph = g;
  p->marked = true;
  EDP_TRY(cudaGraphInstantiate(&p->exec, g, 0));
  return EDP_OK;
}

int edp_run(edp_peeler *p) {
  if (!p) return EDP_ERR_ARGUMENT;
  if (!p->exec) {
    int rc = edp_capture(p);
    if (rc) return rc;
  }
  EDP_TRY(cudaGraphLaunch(p->exec, p->stream));
  return EDP_OK;
}

int edp_read_status(edp_peeler *p, int32_t *status, int64_t *metrics) {
  if (!p) return EDP_ERR_ARGUMENT;
  EDP_TRY(cudaStreamSynchronize(p->stream));
  if (status)
    EDP_TRY(cudaMemcpy(status, p->d.status, sizeof(int32_t) * kStatusSlots, cudaMemcpyDeviceToHost));
  if (metrics)
    EDP_TRY(cudaMemcpy(metrics, p->d.metrics, sizeof(int64_t) * kMetrics, cudaMemcpyDeviceToHost));
  return EDP_OK;
}

int edp_get_outputs(edp_peeler *p, edp_outputs *o) {
  if (!p || !o) return EDP_ERR_ARGUMENT;
  const Dev &d = p->d;
  o->status = d.status;
  o->metrics = reinterpret_cast<int64_t *>(d.metrics);
  o->output_vertices = reinterpret_cast<double *>(d.out_v);
  o->output_sizes = d.out_n;
  o->output_sources = d.out_src;
  o->output_layers = d.out_layer;
  o->triangles_uv = reinterpret_cast<double *>(d.tri_uv);
  o->triangles_world = d.tri_world;
  o->triangle_sources = d.tri_src;
  o->triangle_layers = d.tri_layer;
  o->canonical = d.canonical;
  o->regions = d.cap.regions;
  o->triangles = d.cap.triangles;
  o->vertices = d.cap.vertices;
  return EDP_OK;
}

void edp_destroy(edp_peeler *p) {
  if (!p) return;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  tree_free(p->source_tree);
  tree_free(p->seg_tree);
  tree_free(p->point_tree);
  tree_free(p->residual_tree);
  for (void *a : p->allocations) cudaFree(a);
  if (p->body_stream) cudaStreamDestroy(p->body_stream);
  if (p->round_stream) cudaStreamDestroy(p->round_stream);
  for (auto &e : p->stage_exec)
    if (e) cudaGraphExecDestroy(e);
  for (cudaEvent_t ev : p->marks)
    if (ev) cudaEventDestroy(ev);
  delete p;
}

const char *edp_status_string(int code) {
  switch (code) {
    case EDP_OK: return "ok";
    case EDP_ERR_ARGUMENT: return "invalid argument";
    case EDP_ERR_STATE: return "invalid call order or capture state";
    case EDP_ERR_CUDA: return "CUDA runtime error";
    case EDP_ERR_MEMORY: return "device memory allocation failed";
    default: return "unknown status";
  }
}

int edp_run_stage(edp_peeler *p, int32_t stage) {
  if (!p || stage < 0 || stage >= kStages) return EDP_ERR_ARGUMENT;
  if (!p->exec) return EDP_ERR_STATE;  // stages replay the state of a full run
  if (!p->stage_exec[stage]) {
    Dev d = p->d;
    d.use_handle = 0;
    EDP_TRY(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    if (stage == 0) {
      e = run_prepare(p, d, p->stream);
    } else if (stage == 1) {
      e = stage_mesh_index(d, p->scratch, p->point_tree, p->stream);
    } else {
      e = cudaMemsetAsync(d.status + kTriangles, 0, sizeof(int), p->stream);
      if (e == cudaSuccess) e = stage_mesh_emit(d, p->stream);
    }
    cudaGraph_t g = nullptr;
    cudaError_t end = cudaStreamEndCapture(p->stream, &g);
    EDP_TRY(e);
    EDP_TRY(end);
    e = cudaGraphInstantiate(&p->stage_exec[stage], g, 0);
    cudaGraphDestroy(g);
    EDP_TRY(e);
  }
  EDP_TRY(cudaGraphLaunch(p->stage_exec[stage], p->stream));
  return EDP_OK;
}

int edp_set_predicates(edp_peeler *p, int32_t mode) {
  if (!p || mode < EDP_PREDICATES_BINARY64 || mode > EDP_PREDICATES_FILTERED64)
    return EDP_ERR_ARGUMENT;
  if (p->exec) return EDP_ERR_STATE;  // the captured graph holds the mode it was made with
  p->d.predicates = mode;
  return EDP_OK;
}

int edp_set_tuning(edp_peeler *p, const edp_tuning *t) {
  if (!p || !t || t->step_budget < 0 || t->subdivide_blocks < 0 || t->subdivide_blocks > 64 ||
      t->heavy_noding_work < 0 || t->clip_budget < 0)
    return EDP_ERR_ARGUMENT;
  if (p->exec) {
    // The captured graphs hold the knobs they were made with: drop them, and
    // the next run records the extraction again.
    EDP_TRY(cudaStreamSynchronize(p->stream));
    EDP_TRY(cudaGraphExecDestroy(p->exec));
    EDP_TRY(cudaGraphDestroy(p->graph));
    p->exec = nullptr;
    p->graph = nullptr;
    p->marked = false;
    for (auto &e : p->stage_exec)
      if (e) {
        EDP_TRY(cudaGraphExecDestroy(e));
        e = nullptr;
      }
  }
  Dev &d = p->d;
  if (t->step_budget) d.step_budget = t->step_budget;
  if (t->subdivide_blocks) d.subdivide_blocks = t->subdivide_blocks;
  if (t->heavy_noding_work) d.heavy_noding_work = t->heavy_noding_work;
  if (t->clip_budget) d.clip_budget = t->clip_budget;
  return EDP_OK;
}

int edp_get_tuning(edp_peeler *p, edp_tuning *t) {
  if (!p || !t) return EDP_ERR_ARGUMENT;
  t->step_budget = p->d.step_budget;
  t->subdivide_blocks = p->d.subdivide_blocks;
  t->heavy_noding_work = p->d.heavy_noding_work;
  t->clip_budget = p->d.clip_budget;
  return EDP_OK;
}

int edp_predicate_counts(edp_peeler *p, int64_t *counts) {
  if (!p || !counts) return EDP_ERR_ARGUMENT;
  EDP_TRY(cudaStreamSynchronize(p->stream));
  EDP_TRY(cudaMemcpy(counts, p->d.pred_counts, sizeof(int64_t) * kPredCounters,
                     cudaMemcpyDeviceToHost));
  return EDP_OK;
}

int edp_workspace_bytes(edp_peeler *p, int64_t *bytes) {
  if (!p || !bytes) return EDP_ERR_ARGUMENT;
  int64_t total = p->bytes;
  for (const TreeBuffers *t : {&p->source_tree, &p->seg_tree, &p->point_tree, &p->residual_tree})
    if (t->nodes)  // nodes, ids (x2), keys (x2), flags and size
      total += int64_t(sizeof(float4) * 4 + 2 * sizeof(int) + 2 * sizeof(uint64_t)) *
                   t->leaves_cap + 3 * int64_t(sizeof(int));
  *bytes = total;
  return EDP_OK;
}

int edp_stage_times(edp_peeler *p, float *ms) {
  if (!p || !ms) return EDP_ERR_ARGUMENT;
  if (!p->marked) return EDP_ERR_STATE;  // no replay of the workspace's own graph yet
  EDP_TRY(cudaEventSynchronize(p->marks[EDP_STAGE_COUNT]));
  for (int k = 0; k < EDP_STAGE_COUNT; ++k)
    EDP_TRY(cudaEventElapsedTime(&ms[k], p->marks[k], p->marks[k + 1]));
  return EDP_OK;
}

int edp_graph_kernels(edp_peeler *p, int64_t *outside_loop, int64_t *per_round) {
  if (!p || !outside_loop || !per_round) return EDP_ERR_ARGUMENT;
  // Counted whenever the extraction was recorded into a graph: the
  // workspace's own (edp_capture) or a caller's (edp_enqueue).
  if (!p->exec && p->kernels_outside == 0) return EDP_ERR_STATE;
  *outside_loop = p->kernels_outside;
  *per_round = p->kernels_per_round;
  return EDP_OK;
}

int edp_last_cuda_error(void) { return g_last_cuda; }
const char *edp_last_error_site(void) { return g_last_site; }
int edp_abi_version(void) { return EDP_ABI_VERSION; }

}  // extern "C"

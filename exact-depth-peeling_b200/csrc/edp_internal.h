// Host-side declarations shared by the translation units of libedp_b200.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "edp_device.cuh"

namespace edp {

#define EDP_CHECK(call)                                  \
  do {                                                   \
    cudaError_t err__ = (call);                          \
    if (err__ != cudaSuccess) return err__;              \
  } while (0)

// Records a failed CUDA call (its code and "file:line") for edp_last_cuda_error
// and edp_last_error_site on this host thread; returns EDP_ERR_CUDA.
int record_cuda_failure(cudaError_t e, const char *site);

constexpr int kSortBlock = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortBlock * kSortItems;  // keys per radix tile
constexpr int kScanTile = 2048;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t pow2_at_least(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}
inline unsigned grid_for(int64_t n, int block) {
  int64_t g = ceil_div(n > 0 ? n : 1, block);
  return static_cast<unsigned>(g);
}

// ---------------------------------------------------------------- primitives
// Scratch for scans and radix sorts, sized once for the largest pool.
struct SortScratch {
  int *hist = nullptr;     // [256][tiles]
  int *totals = nullptr;   // [256]
  int *partials = nullptr; // scan tile sums
  int64_t tiles = 0;       // capacity in radix tiles
  int64_t scan_tiles = 0;  // capacity in scan tiles
};

// Exclusive scan of in[0, *count) into out; out[*count..capacity) untouched.
// The total is written to *total.  Counts are read on the device.
cudaError_t scan_exclusive(const int *in, int *out, const int *count, int64_t capacity,
                           int *total, SortScratch &s, cudaStream_t st);

// Stable LSD radix sort of (key, value) pairs over the first *count items
// (device scalar); items at and after *count are left untouched.  `bits` is
// the number of low key bits that can be non-zero.  The sorted pairs end in
// keys/vals; keys_tmp/vals_tmp are scratch of the same capacity.
cudaError_t sort_pairs_u64(uint64_t *keys, uint64_t *keys_tmp, int *vals, int *vals_tmp,
                           const int *count, int64_t capacity, int bits, SortScratch &s,
                           cudaStream_t st);
cudaError_t sort_pairs_u32(uint32_t *keys, uint32_t *keys_tmp, int *vals, int *vals_tmp,
                           const int *count, int64_t capacity, int bits, SortScratch &s,
                           cudaStream_t st);

// ---------------------------------------------------------------- hierarchy
struct TreeBuffers {
  int64_t capacity = 0;   // items
  int64_t leaves_cap = 0; // power of two >= capacity
  float4 *nodes = nullptr;  // [2 * leaves_cap][2]: lower, upper corner of each node
  int *ids = nullptr, *ids_tmp = nullptr;
  uint64_t *keys = nullptr, *keys_tmp = nullptr;
  int *flags = nullptr;   // [1]: blocks finished in the current fit
  int *size = nullptr;    // device scalar: leaves of the current build
  int *count = nullptr;   // device scalar: items of the current build
  Tree tree() const { return Tree{nodes, ids, size}; }
};

cudaError_t tree_alloc(TreeBuffers &t, int64_t capacity);
void tree_free(TreeBuffers &t);
// Build over item boxes [0, *count).  `count_ptr` null means `static_count`.
// `layered` adds lo.z (a layer number) above the Morton bits (kernels.py:89-90).
cudaError_t tree_build(TreeBuffers &t, const float4 *lo, const float4 *hi, const int *count_ptr,
                       int static_count, bool layered, SortScratch &s, cudaStream_t st);

}  // namespace edp

namespace edp {

// Pool capacities of an extraction (warp_peel/events.py:19-33, solver.py:10-31).
struct Caps {
  int64_t frontier, regions, hits, vertices, triangles, rounds, layers, edge_vertices;
};

constexpr int kRayCells = 16;  // most source-grid cells one source is listed in
constexpr int kSegCells = 4;   // most segment-grid cells one contour segment is listed in

// Device scalars kept between kernels of one extraction.
enum Scalar : int {
  kLivePolygons = 0,   // min(status[2], regions)
  kPatchEdges = 1,     // patch edges of all live polygons
  kLiveHits = 2,       // min(metrics[5], hits)
  kLiveVertices = 3,   // min(status[6], vertices)
  kSourceCount = 4,    // n (constant)
  kSegmentCount = 5,   // distinct contour segments (the hierarchy's items)
  kFrontierLive = 6,   // min(status[0], frontier)
  kUniqueVertices = 7, // distinct (layer, point) boundary vertices
  kSortHits = 8,       // hits for the global hit sort: all when a group is large, else 0
  kSegmentSlots = 9,   // 8 n (constant): candidate contour segment slots
  kMergedLive = 10,    // polygons left after optional convex merging
  kGridOn = 11,        // 1 when the point grid holds every layer of this extraction
  kGridCells = 12,     // grid cells in use: layers x G^2 when the grid is on, else 0
  kTreePoints = 13,    // points of the point hierarchy: 0 when the grid is on
  kHeavyJobs = 14,     // rays queued for the continuation
  kRayGridOn = 15,     // 1 when rays read their candidates from the source grid
  kRayBig = 16,        // sources too large for the grid's cells
  kRayGridCells = 17,  // G^2 (constant): cells of the source and segment grids
  kSegGridOn = 18,     // 1 when connection tests read segments from the segment grid
  kSegBig = 19,        // contour segments too large for the grid's cells
  kHeavyPolygons = 20, // polygons queued for warp-wide noding
  kFrontierNext = 8,   // next frontier patch a subdivision warp takes
  // Iterative clipping (DevicePeeler): live pieces of this round, pieces
  // appended for the next round, hidden pieces of this layer, the current
  // work pool, and the clipping-round loop's condition.
  kClipLive = 21,
  kClipNext = 22,
  kClipHidden = 23,
  kClipParity = 24,
  kClipCondition = 25,
  // Subdivision in the filter-only form: patches deferred to the exact pass
  // this round (kept at the top of the next frontier), and the next of them
  // an exact-pass warp takes.
  kDeferred = 26,
  kDeferredNext = 27,
  // Ranks in the filter-only form: containment tests, hit groups and polygon
  // searches left for the exact passes.
  kRayDeferred = 28,
  kSortDeferred = 29,
  kAssignDeferred = 30,
  kDeepGroups = 31,  // hit groups sorted a warp each (k_group_sort_deep)
  kScalarCount = 32  // k_reset clears them with one warp
};

// Predicate tallies: six classes by three deciding stages (edp_filtered.cuh).
constexpr int kPredCounters = 18;

// Every device pointer of a workspace, passed by value to the kernels.
struct Dev {
  const double *vertices;
  const int *faces;
  const double *camera;
  const double *settings;
  int nv, n;
  int limit, all_layers, share_regions, propagate_ranks, merge_regions;
  // Sign predicates: 0 plain binary64, 1 filtered exact, 2 filtered exact
  // and counted into pred_counts ([class][stage], edp_filtered.cuh).
  int predicates;
  unsigned long long *pred_counts;
  // Tuning knobs (edp_tuning): subdivision walk steps per patch and round,
  // subdivision blocks per SM, candidate x edge tests above which a polygon
  // is noded by a warp, clipping candidate tests per piece and round.  None
  // changes a result, only how the work is spread.
  int step_budget, subdivide_blocks, heavy_noding_work, clip_budget;
  Caps cap;

  int *status;
  long long *metrics;
  int *sc;
  int *parity;
  int *condition;
  double *inverse;  // 4x4 row-major camera inverse

  // welding
  int *canonical, *weld_table, *weld_min, *weld_slot;
  int weld_mask;
  // projected sources, at most kSourceVertices vertices each
  V2 *src_v;
  int *src_n;
  Plane *scores;
  int *facing, *clipped;
  float4 *src_lo, *src_hi;
  // undirected mesh edges
  unsigned long long *ekey_table;
  int *ekey_count, *ekey_member, *edge_slot, *masks;
  unsigned long long *edge_keys;  // welded edge key of each face edge (topology owner)
  int ekey_mask;
  // contour segments: kSourceVertices slots per source
  V2 *slot_a, *slot_b;      // per candidate slot (8 per source): canonical end points
  int *seg_flag, *seg_pos;  // per slot: representative of its group, its compact index
  double *seg_za, *seg_zb;  // per table slot: minimum endpoint depths
  int *seg_srca, *seg_srcb; // per table slot: smallest source attaining each minimum
  // Distinct segments, compacted in slot order: end points, (near depth a, near
  // depth b) and boxes; the contour hierarchy is built over these.
  V2 *seg_a, *seg_b, *seg_near;
  int2 *seg_near_src;  // the sources whose depth planes give seg_near (exact depth tests)
  V2 *seg_near_mag;    // per end, |a x| + |b y| + |c| of that plane: the depth's error scale
  int2 *seg_vid;       // per end, its welded mesh vertex (-1 when not a mesh vertex)
  float4 *seg_lo, *seg_hi;
  int *seg_table, *seg_min, *seg_slot;
  int seg_mask;
  Tree source_tree, seg_tree, point_tree;
  // frontier ping-pong
  V2 *fv[2];
  int *fn[2], *fsrc[2], *fcur[2];
  // output polygons
  V2 *out_v;
  int *out_n, *out_src, *out_layer;
  // patch connectivity
  int *counts, *offsets;
  int2 *tasks;
  unsigned long long *owners;
  V2 *starts, *ends;
  int *partners, *edge_hash, *parents, *reps;
  int edge_hash_mask;
  // samples and query groups
  V2 *samples;
  int *groups, *sample_table, *sample_min, *sample_slot;
  int sample_mask;
  double *cell_bounds;  // [1024][4]
  int *cell_min, *cell_valid;
  int2 *heavy_beams, *heavy_queries;
  // shared ray hits
  double *hit_depth;
  int *hit_src, *hit_group, *hit_ids, *hit_ids_tmp;
  unsigned long long *hkeys, *hkeys_tmp;
  int *group_counts, *group_offsets;
  int *group_fill;  // hits placed in each group so far
  // Filtered binary64 ranks: the (ray, source) containment tests, and then
  // the hit groups and the polygons, whose binary64 filters left a sign
  // undecided, for the exact passes.
  int2 *ray_defer;
  int64_t ray_defer_cap;
  int *rank_defer;  // [regions]
  int *deep_groups; // [regions]: hit groups too deep for one thread's sort
  // Optional convex merging: each polygon's chosen patch edge, and the
  // compaction copy of the outputs (allocated with merge_regions only).
  int *merge_choice;
  V2 *merged_v;
  int *merged_n, *merged_src, *merged_layer;
  // boundary noding and triangles
  V2 *bverts;      // per polygon vertex slot
  int *blayers;
  V2 *uverts;      // distinct (layer, point) vertices, indexed by the point hierarchy
  int *point_table;
  int point_mask;
  // Layered point grid: point_grid x point_grid cells per layer over the
  // unit window for up to grid_layers layers; cell_start is the exclusive scan
  // of the per-cell point counts (with the total at the end) and grid_pts the
  // points by cell.
  int point_grid, grid_layers;
  int grid_size;  // cells per axis of the source and segment grids
  // Source grid for rays (EventPeeler): grid_size x grid_size cells over the
  // window, listing each source whose box (grown by 1e-6) meets at most kRayCells of
  // them; larger sources in ray_big.  leaf_of: each source's leaf in the
  // source hierarchy.
  int *ray_count, *ray_start, *ray_entries, *ray_big, *leaf_of;
  // Contour segment grid for the connection test: distinct segments listed in
  // the cells their box (grown by 1e-6) meets, at most kSegCells each.
  int *seg_count, *seg_start, *seg_entries, *seg_big;
  int *cell_count, *cell_start;
  V2 *grid_pts;
  int *heavy_polygons;  // polygons with many grid candidates, noded a warp each
  float4 *pt_lo, *pt_hi;
  // A processing order of the live output polygons by the Morton code of
  // their box centre (optionally below the layer), rebuilt by each stage that
  // uses it, so that neighbouring threads walk neighbouring parts of a
  // hierarchy.  No result depends on it.
  uint64_t *order_keys, *order_keys_tmp;
  int *order, *order_tmp;
  V2 *tri_uv;        // [triangles][3]
  double *tri_world; // [triangles][3][3]
  int *tri_src, *tri_layer;
  unsigned long long cond_handle;  // cudaGraphConditionalHandle of the subdivision loop
  int use_handle;

  // DevicePeeler (iterative clipping) only.
  float4 *contour_lo, *contour_hi;  // per source: box of its contour edges
  Tree contour_tree;
  int *ranks;                       // whole-source rank, -1 = needs clipping
  V2 *res_v[2];                     // residual patches, ping-pong [residual][32]
  int *res_n[2], *res_src[2];
  float4 *res_lo, *res_hi;
  Tree residual_tree;
  // Clipping work: ping-pong pools of live pieces [work_cap][32], each with
  // its target (a residual patch index) and the position of its candidate
  // walk; the layer's hidden pieces [hidden_cap][32] with their targets; per
  // target its visible and hidden piece counts.
  V2 *work_v[2];
  int *work_n[2], *work_target[2], *work_cursor[2];
  int work_cap;
  V2 *hid_v;
  int *hid_n, *hid_target;
  int hidden_cap;
  int *target_visible, *target_hidden;
  long long *stats;                 // [layers][3]: targets, candidate tests, restored whole
  int workers, pieces;              // clipping threads; pieces one target may hold
  unsigned long long inner_handle;  // cudaGraphConditionalHandle of the clipping rounds
  int use_inner;
  // Host-side: a second stream of the workspace, on which conditional node
  // bodies are recorded while the workspace stream captures.
  cudaStream_t aux_stream;
};

// Polygon edge `edge` of source `source` is a contour: every edge of a
// camera-clipped source, else the mesh edge's mark; a back-facing source's
// polygon was reversed (kernels.py:523-536).
__device__ inline bool contour_edge(const Dev &d, int64_t source, int edge) {
  if (d.clipped[source] != 0) return true;
  int j = edge;
  if (d.facing[source] < 0) j = (4 - edge) % 3;
  return d.masks[3 * source + j] != 0;
}

// Reset, validation, welding, projection, mesh contours and the source
// hierarchy: the part of preparation both peelers share.
cudaError_t stage_prepare_common(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                                 cudaStream_t st);
cudaError_t stage_device_prepare(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                                 TreeBuffers &contour_tree, cudaStream_t st);
cudaError_t stage_device_finish(const Dev &d, cudaStream_t st);
// One layer pass on `st`; its clipping rounds are recorded on `rounds` when
// `st` is capturing (a nested conditional WHILE node), else host-driven.
cudaError_t stage_device_layer(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                               TreeBuffers &residual_tree, cudaStream_t st, cudaStream_t rounds);
// Bring the source hierarchy's leaves up to date with its item boxes without
// re-sorting (solver.py:72-89).
cudaError_t tree_refit(TreeBuffers &t, const float4 *lo, const float4 *hi, cudaStream_t st);

// Rebuild Dev::order over the live output polygons: by Morton code of the box
// centre, below the layer when `layered`.
cudaError_t order_polygons(const Dev &d, bool layered, SortScratch &s, cudaStream_t st);

// Stage launchers (edp_prepare.cu, edp_frontier.cu, edp_rank.cu, edp_mesh.cu).  Each
// enqueues kernels on `st`.
cudaError_t stage_prepare(const Dev &d, SortScratch &s, TreeBuffers &source_tree,
                          TreeBuffers &seg_tree, cudaStream_t st);
cudaError_t stage_step(const Dev &d, cudaStream_t st);
cudaError_t stage_rank(const Dev &d, SortScratch &s, cudaStream_t st);
cudaError_t stage_mesh(const Dev &d, SortScratch &s, TreeBuffers &point_tree, cudaStream_t st);
// The two halves of stage_mesh: boundary vertices and point hierarchy, then
// the noding / emission / lifting kernel.
cudaError_t stage_mesh_index(const Dev &d, SortScratch &s, TreeBuffers &point_tree,
                             cudaStream_t st);
cudaError_t stage_mesh_emit(const Dev &d, cudaStream_t st);

}  // namespace edp

namespace edp {
// Host-side count of kernel launches issued by this thread (every launch site
// calls note_launch), used to report how many kernels a captured graph runs.
void note_launch();
int64_t launch_count();
// Takes back n noted launches (kernels recorded in a conditional IF body that
// an ordinary replay skips).
void forget_launches(int64_t n);

// Stage marks.  While a workspace captures its own graph, `events` holds
// EDP_STAGE_COUNT + 1 timing events; stage_mark(-1, st) records the start
// (event 0) and stage_mark(k, st) the end of every stage up to k not yet
// marked (a skipped stage gets a zero-length interval), as external event
// nodes of the graph.  With no events set (eager runs, other captures) it
// does nothing.
void set_stage_marks(cudaEvent_t *events);
cudaError_t stage_mark(int stage, cudaStream_t st);
}  // namespace edp

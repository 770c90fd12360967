/*
 * edp.h - C ABI of libedp_b200, the B200 analytic depth peeler.
 *
 * Plain pointers and sizes only.  All geometry pointers are CUDA device
 * pointers owned by the caller; the workspace owns every pool and output
 * buffer and must outlive any CUDA graph that replays it.  Each entry point
 * returns an edp_status code (0 on success); device-side failures are not
 * return codes but sticky bits in status[9], read with edp_read_status.
 *
 * The reference binds this path through Python (Warp arrays, not an FFI); the
 * entry points below replace its call surface one to one:
 *
 *   edp_event_create   warp_peel/events.py:43-138   EventPeeler.__init__
 *   edp_device_create  warp_peel/solver.py:103-212  DevicePeeler.__init__
 *   edp_warmup         warp_peel/events.py:782-796  EventPeeler.warmup
 *   edp_enqueue        warp_peel/events.py:798-806  EventPeeler.enqueue
 *   edp_capture        warp_peel/solver.py:471-480  DevicePeeler.capture
 *   edp_run            warp_peel/solver.py:482-486  DevicePeeler.run
 *   edp_read_status    warp_peel/events.py:808-845  EventPeeler.read_status
 *                      (status[16] and metrics[20] arrays; solver.py:154-156,
 *                      events.py:103)
 *   edp_get_outputs    the device attributes read by warp_peel/io.py:51-72
 *                      and tests/gpu/test_peeler.py:24-34
 *   edp_destroy        workspace release (Warp frees arrays on collection)
 */
#ifndef EDP_H
#define EDP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct edp_peeler edp_peeler;

enum edp_status {
  EDP_OK = 0,
  EDP_ERR_ARGUMENT = 1, /* invalid argument (the reference raises ValueError) */
  EDP_ERR_STATE = 2,    /* capture misuse (the reference raises RuntimeError) */
  EDP_ERR_CUDA = 3,     /* a CUDA runtime call failed; see edp_last_cuda_error */
  EDP_ERR_MEMORY = 4    /* pool allocation failed */
};

/* Status slots and error bits (warp_peel/kernels.py:17-21, README.md:175-184). */
enum {
  EDP_STATUS_SLOTS = 16,
  EDP_METRICS = 24,
  EDP_ABI_VERSION = 5,
  EDP_ERR_BIT_POLYGON = 1,
  EDP_ERR_BIT_WORKER = 2,
  EDP_ERR_BIT_RESIDUAL = 4,
  EDP_ERR_BIT_OUTPUT = 8,
  EDP_ERR_BIT_VERTICES = 16,
  EDP_ERR_BIT_TRIANGLES = 32,
  EDP_ERR_BIT_LAYERS = 64,
  EDP_ERR_BIT_EDGE_NODING = 128,
  EDP_ERR_BIT_INPUT = 256,
  EDP_ERR_BIT_HITS = 1024,
  EDP_ERR_BIT_ROUNDS = 2048
};

/* warp_peel/events.py:19-33 (EventCapacities). */
typedef struct edp_event_capacities {
  int64_t frontier, regions, hits, vertices, triangles, rounds, layers, edge_vertices;
} edp_event_capacities;

/* warp_peel/events.py:43-55 (layers, share_regions, propagate_ranks, merge_regions). */
typedef struct edp_event_options {
  int32_t layers; /* 0 = all layers */
  int32_t share_regions, propagate_ranks, merge_regions;
} edp_event_options;

/* warp_peel/solver.py:10-31 (Capacities).  The same fields, with the
 * clipping redesigned: the work queue holds polygons + residual pieces and
 * the hidden pool residual pieces, shared by all targets; pieces_per_worker
 * bounds the visible and the hidden pieces of one target (error bit 2 above
 * it, as the reference's per-worker pool); workers is kept for the interface
 * (the clipping grid is sized for the GPU). */
typedef struct edp_device_capacities {
  int64_t residual, polygons, vertices, triangles, workers, pieces_per_worker, layers,
      edge_vertices;
} edp_device_capacities;

/* Device pointers of the workspace's buffers.  Counts live in status:
 * status[2] polygons, status[3] triangles, status[6] boundary vertices. */
typedef struct edp_outputs {
  int32_t *status;          /* [16] */
  int64_t *metrics;         /* [20] */
  double *output_vertices;  /* [regions][32][2] polygon vertices */
  int32_t *output_sizes;    /* [regions] vertex counts (0 = suppressed) */
  int32_t *output_sources;  /* [regions] dense source (face) index */
  int32_t *output_layers;   /* [regions] zero-based depth rank */
  double *triangles_uv;     /* [triangles][3][2] normalised window coordinates */
  double *triangles_world;  /* [triangles][3][3] world coordinates */
  int32_t *triangle_sources;
  int32_t *triangle_layers;
  int32_t *canonical;       /* [nv] welded vertex ids */
  int64_t regions, triangles, vertices;
} edp_outputs;

/* Create an EventPeeler workspace (contour subdivision + shared ray ranks).
 * vertices: double[nv][3]; faces: int32[nf][3]; camera: double[4][4] row-major
 * affine world-to-camera; settings: double[6] = xmin, ymin, xmax, ymax,
 * perspective (0/1), near.  stream: the workspace's cudaStream_t.  cap and opt
 * may be NULL for the reference defaults (EventCapacities.for_mesh). */
int edp_event_create(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                     const double *camera, const double *settings,
                     const edp_event_capacities *cap, const edp_event_options *opt, void *stream,
                     edp_peeler **out);

/* Default capacities for a mesh of nf faces (events.py:30-33 / solver.py:21-31). */
void edp_event_default_capacities(int64_t nf, edp_event_capacities *cap);
void edp_device_default_capacities(int64_t nf, edp_device_capacities *cap);

/* Create a DevicePeeler workspace (iterative per-layer clipping). */
int edp_device_create(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                      const double *camera, const double *settings,
                      const edp_device_capacities *cap, int32_t layers, void *stream,
                      edp_peeler **out);

/* One eager extraction with host-driven loop control, then synchronise. */
int edp_warmup(edp_peeler *p);
/* Record the whole extraction into the capture in progress on `stream`, which
 * must be the workspace stream.  No host reads or allocations are recorded. */
int edp_enqueue(edp_peeler *p, void *stream);
/* Capture and instantiate the workspace's own graph (idempotent). */
int edp_capture(edp_peeler *p);
/* Asynchronous replay of the captured graph on the workspace stream. */
int edp_run(edp_peeler *p);
/* Synchronise the workspace stream and copy status[16] / metrics[24] out
 * (either may be NULL). */
int edp_read_status(edp_peeler *p, int32_t *status, int64_t *metrics);
int edp_get_outputs(edp_peeler *p, edp_outputs *out);
void edp_destroy(edp_peeler *p);

/* Replay one stage alone, from its own captured graph, on the workspace
 * stream, after at least one full run: 0 preparation, 1 boundary vertices +
 * point hierarchy, 2 the noding / emission / lifting kernel.  Used to time
 * stages with CUDA events, as the reference's profiler times separately
 * captured stage graphs (scripts/profile_events.py:35-98).  Replaying stage 0
 * resets the counters, so run the full graph again before reading outputs. */
int edp_run_stage(edp_peeler *p, int32_t stage);
/* Sign predicates of the kernels (orientation, containment, depth order):
 * the reference's plain binary64 expressions, or exact signs through
 * escalating filters (binary32 with a static error bound, then binary64, then
 * exact expansion arithmetic), optionally tallied per class and deciding
 * stage.  Workspaces start FILTERED64 (the faster exact form on a B200).
 * Constructions stay binary64.  FILTERED64 runs each kernel with exact signs
 * as two passes: binary64 filters alone, which leave what they cannot decide
 * (a subdivision patch from the undecided test on, a containment test, a
 * hit group, a polygon's rank search) to a second pass with the exact stage;
 * metrics[20..23] count that work per extraction. */
enum edp_predicates {
  EDP_PREDICATES_BINARY64 = 0,
  EDP_PREDICATES_FILTERED = 1,   /* binary32 filter, binary64 filter, exact */
  EDP_PREDICATES_COUNTED = 2,    /* FILTERED, tallied per class and stage */
  EDP_PREDICATES_FILTERED64 = 3  /* binary64 filter, exact (same signs) */
};
/* Predicate classes of edp_predicate_counts (three stages each: binary32,
 * binary64, exact). */
enum edp_predicate_class {
  EDP_PRED_SIDE = 0,    /* patch vertex against a contour segment's line */
  EDP_PRED_SEGMENT,     /* contour segment end against a patch edge */
  EDP_PRED_DEPTH,       /* patch plane against a segment end's near plane */
  EDP_PRED_CONTAIN,     /* ray sample against a source edge */
  EDP_PRED_ORDER,       /* depth order of two sources at a ray sample */
  EDP_PRED_CLIP,        /* clipping piece against an occluder (DevicePeeler) */
  EDP_PRED_CLASSES
};
/* Selects the predicate form (enum edp_predicates) for the next capture or
 * warm-up; EDP_ERR_STATE once the workspace's own graph exists.  No
 * counterpart in the reference, whose kernels are plain binary64. */
int edp_set_predicates(edp_peeler *p, int32_t mode);
/* counts[3 * class + stage] of the last extraction run with
 * EDP_PREDICATES_COUNTED (zero otherwise); synchronises the workspace
 * stream. */
int edp_predicate_counts(edp_peeler *p, int64_t *counts);

/* Work-distribution knobs, read at the next capture or warm-up (0 keeps the
 * current value); setting them drops the workspace's own graph, which the
 * next edp_run records again.  None changes a result; the autotuner (peel_b200.autotune)
 * times replays under each and keeps the fastest.  No counterpart in the
 * reference, whose kernels fix them (frontier.py:149 and kernels.py:815-908
 * use 32 candidates per round and 4096 persistent workers).
 *   step_budget        subdivision: hierarchy walk steps a patch spends in a
 *                      round before it carries over (default 48)
 *   subdivide_blocks   subdivision: blocks of 4 warps per SM (default 8)
 *   heavy_noding_work  noding: candidate x edge tests above which a polygon
 *                      is noded by a warp instead of a thread (default 1024)
 *   clip_budget        DevicePeeler: candidate tests per piece and clipping
 *                      round (default 32) */
typedef struct edp_tuning {
  int32_t step_budget, subdivide_blocks, heavy_noding_work, clip_budget;
} edp_tuning;
int edp_set_tuning(edp_peeler *p, const edp_tuning *t);
int edp_get_tuning(edp_peeler *p, edp_tuning *t);

/* Stages timed by edp_stage_times, in extraction order: the reference
 * profiler's phases (scripts/profile_events.py:35-56) with its rank and mesh
 * phases split where this build's kernels split.  The DevicePeeler fills
 * PREPARE, SUBDIVIDE (its layer loop), RANK_ASSIGN (its finish), and the
 * three MESH stages; its other stages read 0. */
enum edp_stage {
  EDP_STAGE_PREPARE = 0,       /* validation, weld, projection, contours, hierarchies */
  EDP_STAGE_SUBDIVIDE,         /* the subdivision (or layer) loop, all rounds */
  EDP_STAGE_RANK_ORDER,        /* Morton order of the output polygons */
  EDP_STAGE_RANK_CONNECTIVITY, /* patch edges, edge match, connection test */
  EDP_STAGE_RANK_SAMPLES,      /* union-find roots and representative samples */
  EDP_STAGE_RANK_QUERY_GROUPS, /* exact-coordinate sample groups */
  EDP_STAGE_RANK_CERTIFY,      /* certified rectangles */
  EDP_STAGE_RANK_RAY_GRID,     /* the source grid the rays read */
  EDP_STAGE_RANK_RAY_PRIMARY,  /* primary ray hits */
  EDP_STAGE_RANK_RAY_HEAVY,    /* heavy-ray continuation */
  EDP_STAGE_RANK_HIT_SORT,     /* hit counts, scan and per-group hit order */
  EDP_STAGE_RANK_ASSIGN,       /* layer assignment */
  EDP_STAGE_RANK_MERGE,        /* optional convex merge */
  EDP_STAGE_MESH_VERTICES,     /* boundary vertex scan and distinct points */
  EDP_STAGE_MESH_INDEX,        /* point grid and point hierarchy */
  EDP_STAGE_MESH_EMIT,         /* noding, fans, world lift */
  EDP_STAGE_COUNT
};
/* Per-stage device milliseconds of the most recent replay of the workspace's
 * own graph (edp_capture / edp_run), from timing events the graph records at
 * each stage's end; waits for that replay.  ms receives EDP_STAGE_COUNT
 * values, which sum to the replay's time.  No counterpart call in the
 * reference, whose profiler captures each stage as a separate graph. */
int edp_stage_times(edp_peeler *p, float *ms);

/* Kernel nodes of the captured graph (the workspace's own, or the caller's
 * graph that edp_enqueue recorded it into): outside the subdivision loop, and
 * per loop iteration (a replay launches outside + per_round * rounds
 * kernels). */
int edp_graph_kernels(edp_peeler *p, int64_t *outside_loop, int64_t *per_round);

/* Exact-position welding without any device allocation.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc where they need
 * welded ids - a plugin whose host framework owns all device memory through its
 * own arena or caching allocator, or a real-time loop that must not allocate
 * after start-up because an allocation can block on the driver.
 * canonical[i] receives the smallest index j with vertices[j] equal to
 * vertices[i] (signed zeros equal) - the same ids as edp_get_outputs'
 * `canonical`.  Vertices must be finite: a vertex with a NaN coordinate equals
 * no vertex, itself included, and keeps its own index (the workspace path
 * flags such input with EDP_ERR_BIT_INPUT instead).  Both buffers are the
 * caller's device memory; kernels run on `stream`.  The hash-table scratch is
 * a fixed 5 MiB device array that every GPU loading this library holds until
 * the process exits, so nv is limited to EDP_WELD_NOALLOC_MAX_VERTICES (larger
 * nv returns EDP_ERR_ARGUMENT).  The first call on a device, made with that
 * device current, resolves that array's device address; make it before any
 * stream capture (a failed lookup returns EDP_ERR_CUDA and is retried by the
 * next call).  All calls on a device share the array, which keeps the last
 * call's contents; each call clears the part it uses first.  Calls that
 * overlap on the GPU (different streams, or different host threads) race and
 * give undefined ids. */
#define EDP_WELD_NOALLOC_MAX_VERTICES 262144
int edp_weld_noalloc(const double *vertices, int64_t nv, int32_t *canonical, void *stream);

/* Device bytes the workspace holds (pools, hierarchies, scratch).  No
 * counterpart in the reference. */
int edp_workspace_bytes(edp_peeler *p, int64_t *bytes);

/* Learned pool sizing.  No counterpart in the reference, which sizes every
 * pool at worst case from the face count (warp_peel/events.py:19-33).
 *
 * edp_tile_features projects the mesh into EDP_TILE_AXIS^2 screen tiles and
 * writes EDP_MLP_INPUTS features per tile (row-major [tiles][inputs]) to
 * `features`; `scratch` holds EDP_TILE_SCRATCH floats of the caller's device
 * memory.  edp_mlp_infer evaluates the 16 -> 64 -> 64 -> 3 perceptron on
 * `rows` feature rows (BF16 weights on the tensor cores, FP32 accumulation);
 * `params` holds EDP_MLP_PARAMS floats: W1[64][16], b1[64], W2[64][64],
 * b2[64], W3[3][64], b3[3].  edp_mlp_grad adds the gradient of
 * sum(mask * (y - target)^2) * scale to `grad` and the unscaled sum to
 * loss[0]; edp_adam_step applies one Adam step to `params` (moments m, v)
 * and clears `grad`.  All pointers are device memory; kernels run on
 * `stream`. */
#define EDP_TILE_AXIS 16
#define EDP_MLP_INPUTS 16
#define EDP_MLP_HIDDEN 64
#define EDP_MLP_OUTPUTS 3
#define EDP_MLP_PARAMS 5443
#define EDP_TILE_SCRATCH (EDP_TILE_AXIS * EDP_TILE_AXIS * 12 + 4)
int edp_tile_features(const double *vertices, int64_t nv, const int32_t *faces, int64_t nf,
                      const double *camera, const double *settings, float *scratch,
                      float *features, void *stream);
int edp_mlp_infer(const float *params, const float *x, int64_t rows, float *y, void *stream);
int edp_mlp_grad(const float *params, const float *x, const float *target, const float *mask,
                 int64_t rows, float scale, float *grad, float *loss, void *stream);
int edp_adam_step(float *params, float *grad, float *m, float *v, int64_t count, float lr,
                  float beta1, float beta2, float eps, int32_t step, void *stream);

/* Human-readable edp_status; the last CUDA error code of this thread. */
const char *edp_status_string(int code);
int edp_last_cuda_error(void);
/* Source location ("file:line") of the CUDA call behind the last EDP_ERR_CUDA. */
const char *edp_last_error_site(void);
/* EDP_ABI_VERSION of the library: 5 since metrics[] has 24 counters (the
 * filtered binary64 form's deferred work); 4 since the predicate forms, 3
 * since edp_stage_times; 2 had metrics[] of 20 counters (heavy_noded_polygons
 * added); 1 had 19. */
int edp_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* EDP_H */

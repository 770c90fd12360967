/* Exact intersection splitting of a binary64 triangle scene on the host cores
 * (libedp_resolve.so).
 *
 * Replaces the reference's `resolve_intersections INPUT.json OUTPUT.json`
 * (src/resolve_intersections.cpp:19-105: CGAL autorefine with provenance,
 * run before either peeler, since the peelers take resolved meshes).  The
 * construction is this library's own: every triangle is split, in exact
 * arithmetic, by the supporting lines of the contact segments that cross its
 * interior; every point made by a contact or a cut is inserted into every
 * piece edge it lies inside; pieces that are not triangles are fanned around
 * the centroid of their first three corners.  Each output triangle keeps the
 * index of the input triangle it came from (its provenance).
 *
 * Plain C ABI: pointers and sizes only, no exceptions across the boundary.
 */
#ifndef EDP_RESOLVE_H
#define EDP_RESOLVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDP_RESOLVE_ABI_VERSION 1

/* Status codes. */
enum edp_resolve_status {
  EDP_RESOLVE_OK = 0,
  EDP_RESOLVE_COPLANAR_OVERLAP = 1, /* two coplanar triangles overlap with positive area */
  EDP_RESOLVE_TOO_LARGE = 2,        /* an exact number exceeded the native size limit */
  EDP_RESOLVE_BAD_INPUT = 3,        /* a non-finite or subnormal coordinate, or count < 0 */
  EDP_RESOLVE_NO_MEMORY = 4
};

typedef struct edp_resolution edp_resolution;

int edp_resolve_abi_version(void);

/* Resolve `count` triangles given as count x 3 vertices x 3 binary64
 * coordinates (row-major).  `threads` <= 0 uses every hardware thread.  With
 * `exact_text` nonzero the exact output coordinates are kept as text (see
 * edp_resolution_exact).  *out receives the result object (also on error,
 * for edp_resolution_overlap); free it with edp_resolution_free. */
int edp_resolve(const double *triangles, int64_t count, int threads, int exact_text,
                edp_resolution **out);

/* Output triangle count. */
int64_t edp_resolution_triangles(const edp_resolution *r);

/* summary[0..5]: contact segments that cut a triangle, cut triangles,
 * candidate pairs, pairs tested exactly, distinct created points, the scale
 * exponent E (coordinates are integers x 2^-E). */
void edp_resolution_summary(const edp_resolution *r, int64_t summary[6]);

/* Correctly rounded binary64 output: vertices [T][3][3] and the input
 * triangle index of each output triangle, parents [T]. */
int edp_resolution_binary64(const edp_resolution *r, double *vertices, int64_t *parents);

/* Exact output as text: for each output triangle and corner, one line
 * "X Y Z W\n" of hexadecimal integers ('-' for negatives), the corner being
 * (X / W, Y / W, Z / W) x 2^-E.  Returns the bytes needed (including the
 * terminating NUL); writes them when `size` is large enough.  Zero when the
 * resolution was made without exact_text. */
int64_t edp_resolution_exact(const edp_resolution *r, char *text, int64_t size);

/* The two input triangles of a coplanar overlap (status 1). */
void edp_resolution_overlap(const edp_resolution *r, int64_t *a, int64_t *b);

void edp_resolution_free(edp_resolution *r);

#ifdef __cplusplus
}
#endif

#endif /* EDP_RESOLVE_H */

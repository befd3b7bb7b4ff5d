/*
 * dgt.h -- C ABI of the B200 periodic Delaunay one-ring library (libdgt.so).
 *
 * Drop-in boundary for the hot path of the reference class DelaunayGPU
 * (src/model/DelaunayGPU.h:18-130): per-point construction of the Delaunay one-ring in a
 * periodic box, and test-and-repair of an existing triangulation.  Plain pointers and sizes
 * only; every call returns a status code, no exception crosses this boundary.
 *
 * Output layout (same as the reference, DelaunayGPU.cpp:47 Index2D(MaxSize, N)):
 *   tri[i*stride + k], k < neighnum[i]: indices of the Delaunay neighbours of point i in
 *   counter-clockwise order; rows start at the smallest neighbour index.
 * Points: double2[n] as 2n doubles (x0,y0,x1,y1,...), every coordinate in [0, L) of its box
 * (any finite coordinates in a general box, dgt_set_box_general).
 * All pointers named d_* are device pointers on the context's device; `stream` is a
 * cudaStream_t (NULL = legacy default stream).
 * Contexts are not thread-safe (like the reference class); use one per host thread.
 */
#ifndef DGT_H
#define DGT_H

#ifdef __cplusplus
extern "C" {
#endif

#define DGT_OK 0
#define DGT_ERR_INVALID_ARGUMENT 1
#define DGT_ERR_CUDA 2
#define DGT_ERR_NEED_RESIZE 3   /* a ring is longer than the row stride; see dgt_get_max_size */
#define DGT_ERR_DEGENERATE 4    /* a ring could not be closed (duplicate/collinear input) */
#define DGT_ERR_OUT_OF_MEMORY 5
#define DGT_ERR_BAD_POINTS 6    /* a coordinate outside [0, L) or not finite */
#define DGT_ERR_NOT_CONVERGED 7

#define DGT_PRECISION_FP32_FILTER 0 /* float32 filter, float64 recheck, exact residue (default) */
#define DGT_PRECISION_FP64 1        /* float64 predicates, exact residue */

typedef struct dgt_context dgt_context;

/* counters of the last triangulation / test-and-repair call */
typedef struct dgt_stats {
    long long points;          /* ring constructions (build: n; repair: rebuilt points) */
    long long candidates;      /* candidate points examined */
    long long tests;           /* circle tests evaluated by the filter stage */
    long long fp32_undecided;  /* tests the float32 filter left open (re-run in float64) */
    long long fp64_undecided;  /* tests float64 left open (resolved by exact arithmetic) */
    long long exact_points;    /* deferred points rebuilt by a warp each (float64 + exact, 64-entry ring) */
    long long mismatches;      /* check mode: filter decisions contradicted by float64 */
    long long insertions;      /* ring insertions */
    long long flagged;         /* test-and-repair: points flagged by the local test */
    long long repaired;        /* test-and-repair: points rebuilt (all rounds) */
    long long cells;           /* grid cells scanned */
    int repair_rounds;         /* test-and-repair: rounds until no ring changed */
    int max_ring;              /* largest ring of the call */
    int error_flags;           /* DGT_FLAG_* bits of the last call */
    int launches;              /* kernels this library launched in the last call */
    int sticky_flags;          /* DGT_FLAG_* bits of every call since dgt_clear_flags */
    int reserved;
    long long repair_calls;    /* test-and-repair calls completed on the device */
    long long md_step;         /* device step counter used by DGT_STEP_AUTO */
    long long heavy_points;    /* points rebuilt by the warp-per-point kernel (over the work budget) */
    long long flips;           /* test-and-repair: edge flips applied */
    long long flip_spilled;    /* test-and-repair: flip candidates handed to the rebuild rounds */
    int flip_rounds;           /* test-and-repair: flip rounds run */
    int rebinned;              /* test-and-repair: 1 when the call rebuilt the cell lists (a point
                                  moved more than half a cell since the last binning), 0 when it
                                  reused them with widened certification */
} dgt_stats;

/* phases timed with CUDA events when timing is on (dgt_set_timing) */
#define DGT_PHASE_BIN 0        /* cell grid: count, scan, scatter, in-cell order */
#define DGT_PHASE_BUILD 1      /* one-ring kernel over all points (global triangulation) */
#define DGT_PHASE_SLOW 2       /* deferred points: warp-per-point kernel, exact / large-ring path */
#define DGT_PHASE_TEST 3       /* local Delaunay test (test-and-repair) */
#define DGT_PHASE_REPAIR 4     /* all repair rounds (test-and-repair) */
#define DGT_NUM_PHASES 5

/* dgt_stats.error_flags */
#define DGT_FLAG_UNBOUNDED 1    /* a ring kept a virtual corner after scanning the whole box */
#define DGT_FLAG_NONCONTIG 2    /* degenerate conflict set (duplicate / cocircular input) */
#define DGT_FLAG_RING_OVERFLOW 4 /* a ring outgrew the deferred path's 64 entries */
#define DGT_FLAG_UNRESOLVED 8
#define DGT_FLAG_BAD_POINTS 16
/* warning only: some Delaunay circle reached past half the box, where minimum-image
   offsets are no longer unique (the reference has the same limit); results for such
   points follow the minimum-image convention */
#define DGT_FLAG_MINIMUM_IMAGE 32
#define DGT_FLAG_NOT_CONVERGED 64 /* an unsynchronised repair ran out of rounds with points queued */

/* DelaunayGPU(int N, int maximumNeighborsGuess, double cellSize, PeriodicBoxPtr bx)
 * (src/model/DelaunayGPU.h:25, DelaunayGPU.cpp:11-37).  Rectangular periodic box Lx x Ly.
 * cell_size <= 0 picks the cell edge automatically (the mean point spacing). */
int dgt_create(int n, int max_neighs, double cell_size, double Lx, double Ly, dgt_context **out);

/* Many independent periodic sets in one context: set s has sizes[s] points (concatenated
 * in set order) and box boxes[2s] x boxes[2s+1].  Rings hold global point indices.
 * cell_size is relative to each set's mean spacing (<= 0: automatic).  No reference
 * counterpart: the reference triangulates one set per DelaunayGPU object. */
int dgt_create_batch(int num_sets, const int *sizes, const double *boxes, double cell_size, int max_neighs,
                     dgt_context **out);
/* dgt_create_batch with general periodic boxes: boxes4 holds (xx, xy, yx, yy) per set, as
 * dgt_set_box_general (a rectangle is (Lx, 0, 0, Ly)); each basis is reduced.  No reference
 * counterpart (see dgt_create_batch and dgt_set_box_general). */
int dgt_create_batch_general(int num_sets, const int *sizes, const double *boxes4, double cell_size, int max_neighs,
                             dgt_context **out);

void dgt_destroy(dgt_context *ctx);

/* globalDelaunayTriangulation(points, GPUTriangulation, cellNeighborNum)
 * (DelaunayGPU.h:30, DelaunayGPU.cpp:118-157).  d_tri holds n*stride ints.
 * Returns DGT_ERR_NEED_RESIZE when some ring is longer than stride; dgt_get_max_size then
 * reports the stride needed (the reference grows its own array, DelaunayGPU.cpp:137-156). */
int dgt_global_triangulation(dgt_context *ctx, const double *d_points, int *d_tri, int *d_neighnum, int stride,
                             void *stream);

/* testAndRepairDelaunayTriangulation(points, GPUTriangulation, cellNeighborNum)
 * (DelaunayGPU.h:33, DelaunayGPU.cpp:567-602): (d_tri, d_neighnum) must hold a valid
 * triangulation of earlier positions; afterwards they hold the Delaunay triangulation of
 * d_points.  Only rings that changed are rewritten. */
int dgt_test_and_repair(dgt_context *ctx, const double *d_points, int *d_tri, int *d_neighnum, int stride,
                        void *stream);

/* updateList(points) (DelaunayGPU.h:42): rebuild only the cell grid of d_points. */
int dgt_update_list(dgt_context *ctx, const double *d_points, void *stream);

/* setCellListSize(csize) (DelaunayGPU.h:40) */
int dgt_set_cell_size(dgt_context *ctx, double cell_size);
/* setBox(bx) (DelaunayGPU.h:44); single-set contexts only */
int dgt_set_box(dgt_context *ctx, double Lx, double Ly);
/* setBox with a general (non-rectangular) periodicBoundaries box, setGeneral(a, b, c, d)
 * (periodicBoundaries.h:86-101): a point is (x11 u + x12 v, x21 u + x22 v) for fractional
 * coordinates (u, v), i.e. the lattice vectors are the columns (x11, x21) and (x12, x22).  The
 * reference's cell list and kernels are rectangular-only (cellListGPU.h:14-16); here the
 * kernels run in the box's fractional frame.  The basis is first reduced (Lagrange-Gauss: the
 * same lattice, most nearly orthogonal basis; the triangulation depends on the lattice only).
 * Points may lie anywhere (fractional coordinates are wrapped); non-finite coordinates raise
 * DGT_EF_BAD_INPUT.  A diagonal matrix with positive entries is dgt_set_box.  Single-set
 * contexts only; DGT_ERR_INVALID_ARGUMENT for a degenerate or non-finite matrix. */
int dgt_set_box_general(dgt_context *ctx, double x11, double x12, double x21, double x22);
/* getBoxDims(xx, xy, yx, yy) (periodicBoundaries.h:36-37) of the box the kernels use: the
 * reduced basis after dgt_set_box_general, (Lx, 0, 0, Ly) for a rectangular box. */
int dgt_get_box(const dgt_context *ctx, double *out4);
/* setSafetyMode(sm) (DelaunayGPU.h:46).  On: each call synchronises and reports
 * DGT_ERR_NEED_RESIZE.  Off: calls return without synchronising; overflowing rings are
 * written with neighnum 0 and show in dgt_get_stats (never silently truncated). */
int dgt_set_safety_mode(dgt_context *ctx, int on);
/* DGT_PRECISION_* */
int dgt_set_precision(dgt_context *ctx, int precision);
/* 1: additionally evaluate every float32 decision in float64 and count contradictions */
int dgt_set_check_mode(dgt_context *ctx, int on);
/* resize(nmax) (DelaunayGPU.h:38): the ring capacity MaxSize callers should allocate */
int dgt_resize(dgt_context *ctx, int max_neighs);
/* MaxSize (DelaunayGPU.h:56): after DGT_ERR_NEED_RESIZE, the stride required */
int dgt_get_max_size(const dgt_context *ctx, int *out);
int dgt_get_num_points(const dgt_context *ctx, int *out);

/* Copy rows into an array of another stride (rows keep their neighbours; unused slots 0).
 * Needed when growing MaxSize of an existing triangulation before a repair. */
int dgt_restride(const int *d_src, int src_stride, int *d_dst, int dst_stride, const int *d_neighnum, int n,
                 void *stream);

/* Counters of the last call (synchronises the context's last stream). */
int dgt_get_stats(dgt_context *ctx, dgt_stats *out);

/* Device-side validation of a triangulation in the caller's arrays (no reference
 * counterpart: the reference compares its output with CGAL on the host).  One pass over the
 * points with exact predicates; every row read is bounds-checked, so corrupt rows are
 * counted, never followed.  Needs no earlier call on the context besides creation (the
 * context supplies the box / batched sets); synchronises the stream. */
typedef struct dgt_validation {
    long long points;         /* points checked */
    long long sum_neighbors;  /* sum of all ring lengths (6 * points for a triangulation of the
                                 torus: 3n edges) */
    long long bad_rows;       /* length outside [3, stride], index out of range, self or repeated */
    long long asymmetric;     /* spokes (i, j) where ring(j) lacks i or disagrees on i's two
                                 adjacent neighbours (the two triangles seen from j) */
    long long not_ccw;        /* fan triangles (i, P_k, P_k+1) not strictly counter-clockwise */
    long long winding;        /* fans that do not wind exactly once around their point (or have
                                 a triangle counted in not_ccw) */
    long long not_delaunay;   /* spokes whose opposite vertex lies strictly inside the circle
                                 through the point and its two other neighbours (exact) */
    int valid;                /* 1: all counts above are 0 and sum_neighbors == 6 * points */
    int reserved;
} dgt_validation;
int dgt_validate(dgt_context *ctx, const double *d_points, const int *d_tri, const int *d_neighnum, int stride,
                 dgt_validation *out, void *stream);

/* Spatial order of the points (the reference offers a Hilbert-curve pre-pass for the same
 * purpose, src/utilities/hilbert_curve.cpp; this is the cell order of the last binning):
 * d_order[k] = index of the k-th point in cell order (cells row-major, points of a cell by
 * index; for batched contexts set by set).  Renumbering the points in this order puts
 * Delaunay neighbours at nearby indices.  Needs a global triangulation or test-and-repair on
 * the context first (DGT_ERR_INVALID_ARGUMENT otherwise); d_order is int[n] on the device. */
int dgt_get_cell_order(dgt_context *ctx, int *d_order, void *stream);

/* Hilbert-curve order of d_points (replaces the reference's hilbertSortArray pre-pass,
 * triangulation.cpp:63-88 over xy2d, src/utilities/hilbert_curve.cpp:229, which sorts on the
 * host along a curve of unit squares): d_order[k] = index of the k-th point along a Hilbert
 * curve laid over each set's box (a general box: over its fractional frame) with a 2^k x 2^k
 * grid, the smallest with at least one square per point (k <= 15); points of one square by
 * index; batched contexts set by set.  Needs no earlier call; d_points double2[n] and d_order
 * int[n] on the device.  Allocates its scratch on first use (16 to 40 bytes per point, with
 * the grid) and synchronises `stream` before it returns. */
int dgt_get_hilbert_order(dgt_context *ctx, const double *d_points, int *d_order, void *stream);
/* The reference's hilbertSortArray (triangulation.cpp:63-88) on the device: reorders
 * d_points in place along the order of dgt_get_hilbert_order (point k becomes the old point
 * d_order[k]); d_order (int[n] on the device) receives that order, or may be null.  Existing
 * triangulations refer to the old numbering: triangulate again after sorting. */
int dgt_hilbert_sort_points(dgt_context *ctx, double *d_points, int *d_order, void *stream);

/* 1: record CUDA events around each phase of every call (on the call's stream). */
int dgt_set_timing(dgt_context *ctx, int on);
/* Milliseconds per phase of the last call (DGT_NUM_PHASES values, -1 for phases the call did
 * not run); synchronises the last stream. */
int dgt_get_phase_times(dgt_context *ctx, double *out_ms);

/* MD-like helper: every point += sigma * N(0,1) per axis (counter-based normals of
 * (seed, step, index)), wrapped into its box (periodicBoundaries::move,
 * periodicBoundaries.h:181-189).  step == DGT_STEP_AUTO takes the step from a counter in
 * device memory and advances it (so a captured graph draws new noise on every replay). */
#define DGT_STEP_AUTO 0xFFFFFFFFFFFFFFFFULL
int dgt_displace(dgt_context *ctx, double *d_points, double sigma, unsigned long long seed, unsigned long long step,
                 void *stream);

/* One MD-like step without any host synchronisation, suitable for stream capture:
 * dgt_displace(DGT_STEP_AUTO) then test-and-repair with exactly `rounds` repair rounds.
 * Overflow / unfinished repair show up in dgt_stats.sticky_flags.  No reference
 * counterpart: the reference's driver moves points on the host (triangulation.cpp:349-364). */
int dgt_md_step(dgt_context *ctx, double *d_points, int *d_tri, int *d_neighnum, int stride, double sigma,
                unsigned long long seed, int rounds, void *stream);

/* `steps` MD steps captured into one CUDA graph on `stream` (must not be the legacy default
 * stream); every dgt_md_graph_launch replays them with fresh noise and fresh repair epochs. */
typedef struct dgt_graph dgt_graph;
int dgt_md_graph_create(dgt_context *ctx, double *d_points, int *d_tri, int *d_neighnum, int stride, double sigma,
                        unsigned long long seed, int steps, int rounds, void *stream, dgt_graph **out);
int dgt_md_graph_launch(dgt_graph *graph, void *stream);
void dgt_md_graph_destroy(dgt_graph *graph);
/* reset dgt_stats.sticky_flags */
int dgt_clear_flags(dgt_context *ctx, void *stream);

/* Kernel shape of the one-ring kernel: (ring entries kept on chip, threads per block) =
 * 0: (14, 64) default, 1: (12, 64), 2: (16, 64), 3: (14, 32), 4: (12, 32), one thread per
 * point; 5: (14, 64) with a group of 4 lanes per point, 6: (14, 64) with 8 lanes per point.
 * Rings longer than the on-chip capacity continue on the deferred (warp-per-point) path, so
 * every shape gives the same output.  The shape applies to global triangulations; the
 * rebuild rounds of test-and-repair always take shape 0. */
int dgt_set_kernel_shape(dgt_context *ctx, int shape);
/* Work budget (no reference counterpart): cells plus candidates one point may scan in the
 * thread-per-point kernel before it is handed to the warp-per-point kernel (points on the rim
 * of dense clusters, whose circles reach over large regions).  Default 1024; 0 sends every
 * point to the warp-per-point kernel.  Both kernels give the same rings. */
int dgt_set_work_budget(dgt_context *ctx, int budget);
/* Global triangulations in `chunks` (1-8) pieces of the cell order, the points each piece
 * defers to the warp-per-point kernel rebuilt on a stream of their own while the next pieces
 * build, so the slowest deferred points start early (clustered input; default 1: the whole
 * build, then the deferred points).  The output is the same; while the call's stream is
 * capturing a CUDA graph the build is not split.  dgt_autotune chooses it for clustered
 * input. */
int dgt_set_deferred_overlap(dgt_context *ctx, int chunks);
/* Repair strategy (no reference counterpart): on (default), test-and-repair first flips the
 * illegal edges of valid fans (Lawson) and rebuilds only what flips cannot settle (inverted
 * or non-winding fans, inconsistent quadrilaterals); off, it rebuilds every flagged point
 * and the four points of every failing spoke, as the reference does.  Same result. */
int dgt_set_flip_repair(dgt_context *ctx, int on);
/* Flip rounds of the unsynchronised repair calls (dgt_md_step, and dgt_md_graph_create at
 * capture time; no reference counterpart): 0..24, default 3.  What the flips leave goes to
 * the rebuild rounds.  Measured on 256 sets / 3.98M points per MD step at sigma 0.01 / 0.02
 * / 0.05: 3 rounds 1.02 / 1.46 / 3.62 ms, 6 rounds 1.06 / 1.47 / 2.86 ms -- raise it for
 * larger displacements.  Synchronised calls decide on the host instead. */
int dgt_set_graph_flip_rounds(dgt_context *ctx, int rounds);
int dgt_get_tuning(const dgt_context *ctx, double *cell_size, int *shape, int *ring_capacity, int *block);

/* Autotuner (no reference counterpart): times global triangulations of d_points for cell
 * edges of 0.7-1.45 mean spacings and every kernel shape, keeps the fastest on the context
 * and caches it per (point count, set count, density contrast, precision) class for the
 * process.  d_tri / d_neighnum receive the triangulation made with the chosen settings. */
typedef struct dgt_tune_result {
    double cell_size;   /* chosen cell edge (relative to the mean spacing for batched contexts) */
    int shape;          /* chosen kernel shape */
    int trials;
    float best_ms;      /* build time with the chosen settings */
    float default_ms;   /* build time with cell edge = mean spacing, shape 0 */
    int from_cache;
    int work_budget;    /* chosen work budget of the per-thread kernel (dgt_set_work_budget) */
    int deferred_chunks; /* chosen overlap of the deferred points (dgt_set_deferred_overlap) */
    int reserved;
} dgt_tune_result;
int dgt_autotune(dgt_context *ctx, const double *d_points, int *d_tri, int *d_neighnum, int stride, void *stream,
                 dgt_tune_result *out);

/* Global triangulation that allocates nothing.  No counterpart in the reference: it is
 * for callers that must not call cudaMalloc (a host application owns the GPU allocator,
 * or the memory budget is fixed before this library is loaded).  All scratch lives in one
 * fixed device array inside the library (4,720,384 bytes, about 4.72 MB, present on every
 * GPU that loads the library until the process exits), so inputs are limited to
 * DGT_NOALLOC_MAX_POINTS points and a cell grid of DGT_NOALLOC_MAX_CELLS cells
 * (DGT_ERR_INVALID_ARGUMENT beyond that, with nothing written).  Output and precision are
 * those of dgt_global_triangulation (float32 filter) with safety mode on; on
 * DGT_ERR_NEED_RESIZE *out_required_stride (may be NULL) receives the row stride needed.
 * Every call looks up the array's device address in the current context, copies its status
 * to pageable host memory and synchronises `stream`: it must not be called while a stream
 * is capturing a CUDA graph.  All calls share the array: calls whose work overlaps on a GPU
 * race and must be ordered by the caller. */
#define DGT_NOALLOC_MAX_POINTS 65536
#define DGT_NOALLOC_MAX_CELLS (4 * DGT_NOALLOC_MAX_POINTS + 16)
int dgt_global_triangulation_noalloc(const double *d_points, int n, double Lx, double Ly, double cell_size,
                                     int *d_tri, int *d_neighnum, int stride, int *out_required_stride,
                                     void *stream);

const char *dgt_error_string(int code);
int dgt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DGT_H */

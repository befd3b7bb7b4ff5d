// Internal types shared by the binning, ring and API translation units.
//
// Data layout in HBM (all arrays device-resident, owned by the context unless noted):
//   points   double2[n]            caller-owned, original order, primary cell [0,Lx)x[0,Ly)
//   tri      int[n*stride]         caller-owned; row i holds the CCW ring of point i
//   nn       int[n]                caller-owned; ring lengths (reference "neighborNum")
//   cstart   int[cells+1]          CSR cell starts (cells of all sets, set-major)
//   spos     double2[n]            positions in cell order (coalesced candidate reads)
//   sidx     int[n]                cell-order slot -> point index
//   slot_of  int[n]                point index -> cell-order slot
//   set_of   int[n]                point/slot -> set (batched contexts only, else null)
// Point indices are global over the concatenated sets; the slots of set s are the range
// [point_base, point_base + n) because cells are numbered set-major.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dgt {

struct SetDesc {
    double Lx, Ly;      // periodic box edges
    double hLx, hLy;    // half edges (0.5 * L, exact)
    double icw, ich;    // 1 / cell edge per axis
    double cw, ch;      // cell edges
    int xsize, ysize;   // cells per axis (>= 1)
    int cell_base;      // first cell of the set in cstart
    int point_base;     // first point / slot of the set
    int n;              // points in the set
    float V;            // virtual corner coordinate: power of two >= max(Lx, Ly)
    int bxsize;         // occupancy blocks per row (BLOCK_CELLS x BLOCK_CELLS cells each)
    int bysize;
    int block_base;     // first block of the set in the block-count array
    int sbxsize;        // occupancy super-blocks per row (SBLOCK_CELLS x SBLOCK_CELLS cells each)
    int sbysize;
    int sblock_base;    // first super-block of the set in the block-count array
    // General periodic box (periodicBoundaries::setGeneral, periodicBoundaries.h:86-101): a
    // point is M u with u its fractional coordinates, and the cell grid is a grid over u, so
    // a cell is a parallelogram.  Used by the kernels' general-box instantiations only; the
    // rectangular ones read the fields above (Lx, Ly, icw, ... then describe the box's
    // bounding rectangle and are not used for geometry).
    int general;
    double m11, m12, m21, m22;   // box matrix; its columns are the two lattice vectors
    double i11, i12, i21, i22;   // its inverse
    double g11, g12, g21, g22;   // cells per unit of real offset: diag(xsize, ysize) * inverse
    double gnx, gny;             // cells spanned per axis by a disc of unit radius (row norms of g)
    double hxs, hys;             // half the grid, in cells: the reach of minimum-image offsets
};

constexpr int BLOCK_SHIFT = 3;   // occupancy blocks of 8 x 8 cells
constexpr int BLOCK_CELLS = 1 << BLOCK_SHIFT;
constexpr int SBLOCK_SHIFT = 6;  // occupancy super-blocks of 64 x 64 cells (8 x 8 blocks)
constexpr int SBLOCK_CELLS = 1 << SBLOCK_SHIFT;

// block and super-block grids of a set whose cell grid is already set, at block_base of the
// block-count array (the set's blocks, then its super-blocks); returns the number of entries
inline int set_block_grid(SetDesc &S, int block_base)
{
    S.bxsize = (S.xsize + BLOCK_CELLS - 1) / BLOCK_CELLS;
    S.bysize = (S.ysize + BLOCK_CELLS - 1) / BLOCK_CELLS;
    S.block_base = block_base;
    S.sbxsize = (S.xsize + SBLOCK_CELLS - 1) / SBLOCK_CELLS;
    S.sbysize = (S.ysize + SBLOCK_CELLS - 1) / SBLOCK_CELLS;
    S.sblock_base = block_base + S.bxsize * S.bysize;
    return S.bxsize * S.bysize + S.sbxsize * S.sbysize;
}

// Distance on a periodic axis of `size` cells from u (cell units) to cell [c, c + 1].
__device__ __forceinline__ double arc_gap(double u, int c, int size)
{
    const double lo = (double)c, hi = lo + 1.0;
    if (u >= lo && u <= hi) return 0.0;
    return u < lo ? fmin(lo - u, u + size - hi) : fmin(u - hi, lo + size - u);
}

// Position of p in cell units of its set's grid: [0, xsize) x [0, ysize) for a point inside
// the box.  General box: the fractional coordinates are wrapped into [0, 1) first, so any
// finite position is accepted (the result may equal xsize / ysize after rounding; cell
// indices are clamped).
template <bool GEN>
__device__ __forceinline__ double2 cell_pos(const SetDesc &S, double2 p)
{
    if (!GEN) return make_double2(p.x * S.icw, p.y * S.ich);
    double u = __fma_rn(S.i11, p.x, __dmul_rn(S.i12, p.y));
    double v = __fma_rn(S.i21, p.x, __dmul_rn(S.i22, p.y));
    u -= floor(u);
    v -= floor(v);
    return make_double2(u * (double)S.xsize, v * (double)S.ysize);
}

// General box: offset c - p to the image of c whose fractional offset lies in [-1/2, 1/2]
// per component (the general branch of periodicBoundaries::minDist, periodicBoundaries.h:
// 165-178).  The lattice shift l is chosen in fractional coordinates and taken off c when it
// is positive, added to p otherwise, per axis: with a diagonal box matrix this is the
// rectangular offset (wrap_off) bit for bit, except where a difference lies within rounding
// of exactly half the box.  Explicit roundings throughout; the oracle performs the same
// operations.
__device__ __forceinline__ double gen_off1(double c, double p, double l)
{
    return l >= 0.0 ? __dsub_rn(__dsub_rn(c, l), p) : __dsub_rn(c, __dadd_rn(p, l));
}
__device__ __forceinline__ double2 gen_off(double2 c, double2 p, const SetDesc &S)
{
    const double dx = __dsub_rn(c.x, p.x), dy = __dsub_rn(c.y, p.y);
    const double su = rint(__fma_rn(S.i11, dx, __dmul_rn(S.i12, dy)));
    const double sv = rint(__fma_rn(S.i21, dx, __dmul_rn(S.i22, dy)));
    const double lx = __fma_rn(S.m11, su, __dmul_rn(S.m12, sv));
    const double ly = __fma_rn(S.m21, su, __dmul_rn(S.m22, sv));
    return make_double2(gen_off1(c.x, p.x, lx), gen_off1(c.y, p.y, ly));
}

// How far, in cells per axis, point p now lies outside the cell c that lists it (0 while
// inside), rounded up: the margin by which certification must widen while the cell lists
// are kept (a point strictly inside a circle is listed by a cell within that margin of it).
template <bool GEN = false>
__device__ __forceinline__ float outside_cell(const SetDesc &S, int c, double2 p)
{
    const int lc = c - S.cell_base, cy = lc / S.xsize, cx = lc - cy * S.xsize;
    const double2 f = cell_pos<GEN>(S, p);
    const double g = fmax(arc_gap(f.x, cx, S.xsize), arc_gap(f.y, cy, S.ysize));
    return g > 0.0 ? (float)g * 1.0001f + 1e-6f : 0.0f;
}

// device-side status / counters of one call (zeroed at the start of each call)
struct DevStatus {
    int need_stride;            // largest ring that did not fit the caller's stride
    int max_ring;               // largest ring produced
    int err_flags;              // DGT_EF_* bits
    int rounds;                 // repair rounds executed (device-side count)
    int list_count[2];          // repair work lists (ping-pong)
    int defer_count;            // items queued for the warp-per-point kernel
    int flip_count[2];          // flip candidate lists (ping-pong)
    int pad;
    unsigned long long points;          // ring constructions
    unsigned long long candidates;      // candidates examined
    unsigned long long tests;           // circle tests evaluated
    unsigned long long f32_undecided;   // undecided by the float32 filter
    unsigned long long f64_undecided;   // undecided by the float64 recheck
    unsigned long long exact_points;    // deferred points (warp-per-point kernel: float64 + exact)
    unsigned long long capacity_points; // points whose ring outgrew on-chip capacity
    unsigned long long mismatches;      // check mode: filter decisions contradicted by float64
    unsigned long long insertions;      // ring insertions
    unsigned long long flagged;         // points queued by the test kernel
    unsigned long long repaired;        // points rebuilt by repair rounds
    unsigned long long cells;           // grid cells scanned
    unsigned long long heavy_points;    // deferred because they outgrew the per-thread work budget
    unsigned long long flips;           // test-and-repair: edge flips applied
    unsigned long long flip_spilled;    // flip candidates left after the last flip round
    int flip_rounds;                    // flip rounds run
    int rebin;                          // repair: 1 when this call rebuilt the cell lists
    float skin_measured;                // repair: largest move since binning, in cells (per axis)
    float skin;                         // certification margin of this call's rebuilds, in cells
};

enum : int {
    EF_UNBOUNDED = 1,      // a ring still held a virtual corner after the whole box was scanned
    EF_NONCONTIG = 2,      // a conflict set was not one contiguous arc (degenerate input)
    EF_SLOW_OVERFLOW = 4,  // a ring outgrew even the 64 entries of the deferred path
    EF_EXACT_UNRESOLVED = 8,
    EF_BAD_INPUT = 16,     // coordinates not finite
    // warning, not an error: a certified circle reached past half the box, where minimum-
    // image offsets stop being unique (the box is too small for that point's Delaunay star)
    EF_MINIMAGE = 32,
    EF_NOT_CONVERGED = 64, // repair rounds ran out with points still queued
};

// device-resident control block of a context: everything that changes from call to call
// lives here so a captured CUDA graph replays correctly
struct DevCtl {
    int epoch;                  // last repair epoch used (marks >= epoch+1 belong to the next call)
    int sticky;                 // error flags of every call since the last reset
    unsigned long long step;    // displacement step counter (dgt_displace with DGT_STEP_AUTO)
    unsigned long long calls;   // test-and-repair calls completed
    unsigned flip_stamp;        // last flip-round stamp used (claims of later rounds are larger)
    int pad;
};

enum : int { MODE_F32 = 0, MODE_F64 = 1 };

struct BinArgs {
    const double2 *pos;
    int n;
    const SetDesc *sets;
    const int *set_of;
    int total_cells;
    int *ccount;     // total_cells + 1
    int *cstart;     // total_cells + 1
    int *bcount;     // points per occupancy block, then non-empty blocks per super-block (zeroed by the caller)
    int *cell_of;    // n
    int *rank;       // n
    int *sidx, *slot_of;
    double2 *spos;
    int *block_sums;
    int deterministic;
    const int *cond;    // null: bin; else bin only when *cond != 0 (device-side decision)
    int num_sets;       // entries of sets
    int total_blocks;   // entries of bcount (blocks and super-blocks of every set)
};

struct RingArgs {
    const SetDesc *sets;
    const int *set_of;
    const double2 *pos;
    const double2 *spos;
    const int *sidx;
    const int *slot_of;
    const int *cstart;
    const int *bcount;  // points per occupancy block, then non-empty blocks per super-block:
                        // empty ones are skipped by the scan
    int *tri;
    int *nn;
    int stride;
    int npoints;       // total points (bound for indices read back from caller rows)
    // work selection: worklist == null -> item t is slot t (t < n_items)
    const int *worklist;
    const int *worklist_count;  // device count (used when worklist != null)
    int n_items;
    // repair bookkeeping: this call's base epoch is *epoch_ptr + 1, round r's items carry
    // mark base + r and queue the next round with base + r + 1
    int repair;        // 1: rebuild listed points and propagate consistency checks
    int *mark;
    const int *epoch_ptr;
    int round;
    int *next_list;
    int *next_count;
    // points deferred to the warp-per-point kernel (float64 + exact, 64-entry ring): rings
    // longer than the per-thread capacity, predicates float32 and float64 cannot decide, and
    // scans longer than work_budget (cells + candidates)
    int *defer_list;
    int *defer_count;
    int item_base;     // without a work list: item t is slot item_base + t
    int work_budget;
    int warp_items;    // work lists of at most this many items are rebuilt by the warp kernel alone
    // Cell lists older than the positions (repair without rebinning): every point is at most
    // *skin cells (per axis) from the cell that lists it, so certification widens each
    // circle's cell rectangle by that much.  Null or 0: the lists are current.
    const float *skin;
    int cand_by_index;   // 1: candidate and own positions from pos[] through the index (repair)
    int check;         // 1: count float32 decisions contradicted by float64
    int general = 0;   // 1: general-box instantiations (SetDesc::general)
    DevStatus *st;
};

struct TestArgs {
    const SetDesc *sets;
    const int *set_of;
    const double2 *pos;
    const int *sidx;        // cell-order slot -> point (null: index order)
    const double2 *spos;    // positions in cell order (used with sidx)
    const int *tri;
    const int *nn;
    int stride;
    int n;
    int *mark;
    const int *epoch_ptr;   // this call's base epoch is *epoch_ptr + 1
    int *list;
    int *list_count;
    // flip mode (flip_list != null): illegal edges (i < j) of valid fans go to the flip list,
    // invalid fans to the rebuild list
    int2 *flip_list;
    int *flip_count;
    int flip_cap;
    // cells of the last binning (index order; null: not measured): how far the points now
    // lie outside the cells that list them, largest -> st->skin_measured (outside_cell)
    const int *rcell_of;
    int general = 0;        // 1: general-box instantiation (SetDesc::general)
    DevStatus *st;
};

struct FlipArgs {
    const SetDesc *sets;
    const int *set_of;
    const double2 *pos;
    int *tri;
    int *nn;
    int stride;
    int n;
    int *mark;                  // rebuild marks (this call's base epoch is *epoch_ptr + 1)
    const int *epoch_ptr;
    int *rebuild_list;          // points for the rebuild rounds
    int *rebuild_count;
    unsigned long long *claim;  // per point: (stamp << 32) | slot of the candidate holding it
    const unsigned *stamp_ptr;  // round r of this call uses stamp *stamp_ptr + 1 + r
    int2 *cur;                  // candidates (i < j) of this round
    const int *cur_count;
    int2 *quad;                 // per candidate: (a, b) when it claimed, (-1, -1) otherwise
    int2 *next;                 // candidates of the next round
    int *next_count;
    int cap;                    // capacity of cur / next / quad
    int general = 0;            // 1: general-box instantiations (SetDesc::general)
    DevStatus *st;
};

// launchers (defined in the .cu files)
cudaError_t launch_bin_st(const BinArgs &a, DevStatus *st, cudaStream_t s);
// Repair without a full rebin.  The cell lists of the last binning stay usable as candidate
// lists while no point lies more than MAX_SKIN_CELLS cells outside the cell that lists it:
// launch_refresh copies the current positions into cell order and measures that distance
// (st->skin_measured, in cells), launch_rebin_decide sets st->rebin (too far) and st->skin
// (the margin the ring kernels must add; 0 after a rebin); binning launched with
// a.cond = &st->rebin then runs only when needed, all decided on the device.
cudaError_t launch_refresh(const BinArgs &a, DevStatus *st, float max_skin, cudaStream_t s);
cudaError_t launch_rebin_decide(DevStatus *st, float max_skin, cudaStream_t s);
cudaError_t launch_clear_counts(int *ccount, int ncell, int *bcount, int nblock, const int *cond, cudaStream_t s);
constexpr float MAX_SKIN_CELLS = 0.5f;
cudaError_t launch_scan(const int *in, int n, int *bsum, int *out, cudaStream_t s);
int scan_block_count(int n);

// Hilbert order of the points (dgt_hilbert.cu): per set, the curve's 2^k x 2^k grid, the
// scale from a position (rectangular box) or a fractional coordinate (general box) to grid
// squares, and the set's first key
struct HilbertSet {
    double sx, sy;
    int k, base;
};
struct HilbertArgs {
    const double2 *pos;
    int n;
    const SetDesc *sets;
    const int *set_of;
    const HilbertSet *hsets;
    int buckets;       // keys of all sets
    int *hcount;       // buckets + 1 (zeroed by the launcher)
    int *hstart;       // buckets + 1
    int *bsum;         // scan_block_count(buckets + 1)
    int *hbucket, *hrank;   // n each
    int *order;        // n: the result
};
cudaError_t launch_hilbert_order(const HilbertArgs &a, cudaStream_t s);
// dst[k] = src[order[k]]
cudaError_t launch_gather_points(const double2 *src, const int *order, int n, double2 *dst, cudaStream_t s);
constexpr int KERNEL_SHAPES = 7;
int kernel_shape_cap(int shape);
int kernel_shape_block(int shape);
cudaError_t launch_build(const RingArgs &a, int mode, int sms, int shape, cudaStream_t s);
// the one-ring kernel with `lanes` (4 or 8) lanes per point (dgt_group.cu)
cudaError_t launch_build_group(const RingArgs &a, int mode, int sms, int lanes, cudaStream_t s);
cudaError_t launch_deferred(const RingArgs &a, int sms, cudaStream_t s);
// cells + candidates one point may scan in the per-thread kernel before the warp-per-point
// kernel takes it over (clustered 1M-point mixture: 13.4 ms build at 1024 against 19.2 ms at
// 4096; uniform points stay far below it)
constexpr int DEFAULT_WORK_BUDGET = 1024;
cudaError_t launch_test(const TestArgs &a, cudaStream_t s);
// device validation counts (sum, bad_rows, asymmetric, not_ccw, winding, not_delaunay, points)
cudaError_t launch_validate(const SetDesc *sets, const int *set_of, const double2 *pos, const int *tri,
                            const int *nn, int stride, int n, unsigned long long *out, int sms, int general,
                            cudaStream_t s);
cudaError_t launch_flip_round(const FlipArgs &a, int round, int sms, cudaStream_t s);
// leftover candidates to the rebuild list; advances the context's flip stamp by rounds + 1
cudaError_t launch_flip_spill(const FlipArgs &a, int rounds, DevCtl *ctl, int sms, cudaStream_t s);
cudaError_t launch_restride(const int *src, int old_stride, int *dst, int new_stride, const int *nn, int n,
                            cudaStream_t s);
// step_ptr != null: the step comes from (and is advanced in) device memory
cudaError_t launch_displace(double2 *pos, int n, const SetDesc *sets, const int *set_of, double sigma,
                            unsigned long long seed, unsigned long long step, unsigned long long *step_ptr,
                            cudaStream_t s);
// MD step: displacement + wrap, and (cell_of != null) the distance each moved point lies
// outside the cell that lists it, into st->skin_measured (st cleared beforehand); the step is
// read from *step_ptr and advanced by the end of the call (launch_call_end, advance_step)
cudaError_t launch_displace_md(double2 *pos, int n, const SetDesc *sets, const int *set_of, double sigma,
                               unsigned long long seed, unsigned long long *step_ptr, const int *cell_of,
                               DevStatus *st, cudaStream_t s);
// end of a test-and-repair call: fold flags into the sticky word, check convergence,
// advance the epoch by rounds + 1 (and the displacement step counter when advance_step)
cudaError_t launch_call_end(DevCtl *ctl, DevStatus *st, int rounds, cudaStream_t s, bool advance_step = false);
// first rebuild round of a flip-mode repair: the current ring neighbours of its points join it
cudaError_t launch_expand(int *list, int *count, int cap, const int *tri, const int *nn, int stride, int n,
                          int *mark, const int *epoch_ptr, int sms, cudaStream_t s);

}  // namespace dgt

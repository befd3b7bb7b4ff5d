// C ABI of the library (include/dgt.h): context, scratch memory and the call sequences.
//
// global triangulation   bin -> build (all points, cell order) -> slow path (device list)
// test and repair        bin -> local test (queue) -> rounds of rebuild over the queue
//
// Repair rounds.  The test queues every point whose fan is not certainly Delaunay, with
// the vertices of each failing spoke's quadrilateral.  A round rebuilds its queued points
// from scratch (exact rings) and queues, for the next round, every point not yet rebuilt in
// this call whose ring the rebuilt ring contradicts: an old neighbour that was dropped, or a
// new neighbour whose ring does not list the point with the same two adjacent neighbours.
// At the fixed point every point is either rebuilt (exact) or untouched, untouched fans
// passed the local test and agree with every neighbour, so all edges are locally Delaunay
// in a consistent triangulation of the torus, which makes it the Delaunay triangulation
// (Lawson).  Marks are epochs (mark[i] >= base: already queued in this call), so nothing is
// cleared between calls and each point is rebuilt at most once per call.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "dgt.h"
#include "dgt_internal.cuh"

using namespace dgt;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t want)
    {
        if (p && bytes >= want) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, want ? want : 16);
        if (e == cudaSuccess) bytes = want ? want : 16;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

constexpr int FIRST_ROUNDS = 3;     // repair rounds launched before the first host check
constexpr int NEXT_ROUNDS = 2;      // rounds per later batch (each kernel exits at once on an empty list)
constexpr int ASYNC_ROUNDS = 6;     // rounds of an unsynchronised call (convergence flagged on the device)
constexpr int FLIP_BATCH = 4;       // flip rounds launched before each host check (empty rounds exit at once)
// A checked call stops flipping once at most this many candidates per SM are left and hands
// them to the rebuild rounds: a rebuild round costs about the same for a few points as for
// a wave of them, while each further flip round costs its own launches (measured on 4M
// points, sigma 0.02: repair 1.64 -> 1.49 ms against flipping to the end)
constexpr int SPILL_EDGES_PER_SM = 64;
constexpr int MAX_DEFER_CHUNKS = 8;   // slot chunks of an overlapped global build (dgt_set_deferred_overlap)
constexpr int MAX_FLIP_ROUNDS = 24; // flip rounds of a checked call before the rest is rebuilt
constexpr int ASYNC_FLIP_ROUNDS = 3; // default flip rounds of an unsynchronised call (best of 1-10 for MD steps at sigma 0.01)

}  // namespace

struct dgt_context {
    int device = 0;
    int num_sets = 1;
    int n = 0;
    bool batch = false;
    std::vector<int> sizes;
    std::vector<double> boxes;
    // general periodic boxes: per set the reduced basis the kernels use (4 values, columns
    // (g[0], g[2]) and (g[1], g[3])); boxes then holds each set's bounding rectangle.  A
    // rectangular set of a general batch is the diagonal matrix.
    int general = 0;
    std::vector<double> gboxes;
    double cell_size = 1.0;
    int max_size = 16;
    int safety = 1;
    int precision = DGT_PRECISION_FP32_FILTER;
    int check = 0;
    int deterministic = 1;
    std::vector<SetDesc> sets;
    int total_cells = 0;
    int total_blocks = 0;
    DevBuf d_sets, d_set_of, ccount, cstart, cell_of, rank, sidx, slot_of, spos, bsum, mark, list0, list1,
        defer_list, st, ctl, bcount, claim, flip0, flip1, quad, vcount, hsets, hcount, hstart, hsum, hbucket, hrank, horder, hperm;
    DevStatus *h_st = nullptr;
    cudaStream_t last_stream = nullptr;
    bool stats_valid = false;
    int launches = 0;                          // kernels launched by the last call
    bool timing = false;
    cudaEvent_t ev[DGT_NUM_PHASES][2] = {};
    bool ev_used[DGT_NUM_PHASES] = {};
    int sms = 0;
    int shape = 0;   // kernel shape (ring capacity, block size), see dgt_set_kernel_shape
    int work_budget = DEFAULT_WORK_BUDGET;   // per-point cells + candidates of the per-thread kernel
    int flip = 1;    // test-and-repair starts with edge flips (0: rebuild every flagged point)
    int graph_flip_rounds = ASYNC_FLIP_ROUNDS;   // flip rounds of unsynchronised calls
    bool binned = false;   // the cell lists hold a binning of the current grid
    int flip_cap = 0;
    // global builds in this many pieces of the cell order, each on a stream of its own with
    // the points it defers (1: the whole build, then the deferred points)
    int defer_chunks = 1;
    cudaStream_t aux[MAX_DEFER_CHUNKS] = {};
    cudaEvent_t fork_ev = nullptr, aux_ev[MAX_DEFER_CHUNKS] = {};
    DevBuf dcount;   // deferred count of each piece
};

namespace {

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return DGT_OK;
    if (e == cudaErrorMemoryAllocation) return DGT_ERR_OUT_OF_MEMORY;
    return DGT_ERR_CUDA;
}

#define DGT_TRY(expr)                                   \
    do {                                                \
        cudaError_t e_ = (expr);                        \
        if (e_ != cudaSuccess) return cuda_status(e_);  \
    } while (0)

struct PhaseTimer {
    dgt_context *c;
    int ph;
    cudaStream_t s;
    PhaseTimer(dgt_context *cc, int p, cudaStream_t ss) : c(cc), ph(p), s(ss)
    {
        if (c->timing) {
            cudaEventRecord(c->ev[ph][0], s);
            c->ev_used[ph] = true;
        }
    }
    ~PhaseTimer()
    {
        if (c->timing) cudaEventRecord(c->ev[ph][1], s);
    }
};

void phase_begin(dgt_context *c, int ph, cudaStream_t s)
{
    if (c->timing) {
        cudaEventRecord(c->ev[ph][0], s);
        c->ev_used[ph] = true;
    }
}
void phase_end(dgt_context *c, int ph, cudaStream_t s)
{
    if (c->timing) cudaEventRecord(c->ev[ph][1], s);
}

void begin_call(dgt_context *c, cudaStream_t s)
{
    c->last_stream = s;
    c->stats_valid = false;
    c->launches = 0;
    for (int p = 0; p < DGT_NUM_PHASES; ++p) c->ev_used[p] = false;
}

double pow2_at_least(double x)
{
    double v = 1.0;
    while (v < x) v *= 2.0;
    return v;
}

// Lagrange-Gauss reduction of a 2D lattice basis (columns (m[0], m[2]) and (m[1], m[3])):
// afterwards |a| <= |b| and |a.b| <= |a|^2 / 2, the most nearly orthogonal basis of the same
// lattice.  The periodic Delaunay triangulation depends on the lattice only; a reduced basis
// makes the fractional minimum image the nearest image for every offset that matters and
// keeps the cells compact.
void reduce_basis(double m[4])
{
    double ax = m[0], ay = m[2], bx = m[1], by = m[3];
    for (int it = 0; it < 64; ++it) {
        if (ax * ax + ay * ay > bx * bx + by * by) {
            std::swap(ax, bx);
            std::swap(ay, by);
        }
        const double mu = std::nearbyint((ax * bx + ay * by) / (ax * ax + ay * ay));
        if (mu == 0.0) break;
        bx -= mu * ax;
        by -= mu * ay;
    }
    m[0] = ax;
    m[2] = ay;
    m[1] = bx;
    m[3] = by;
}

// general-box fields of a set whose grid is chosen from the cell edge a (see plan_grid)
void plan_general_set(SetDesc &S, const double m[4], double a, int ns)
{
    const double det = m[0] * m[3] - m[1] * m[2];
    const double area = std::fabs(det);
    const double la = std::hypot(m[0], m[2]), lb = std::hypot(m[1], m[3]);
    // the strip between cell lines u = k / xsize is (area / |b|) / xsize wide
    double amin = std::sqrt(area / (64.0 * std::max(ns, 1) + 64.0));
    if (a < amin) a = amin;
    const int xs = std::max(1, (int)std::floor(area / lb / a));
    const int ys = std::max(1, (int)std::floor(area / la / a));
    S.general = 1;
    S.m11 = m[0];
    S.m12 = m[1];
    S.m21 = m[2];
    S.m22 = m[3];
    S.i11 = m[3] / det;
    S.i12 = -m[1] / det;
    S.i21 = -m[2] / det;
    S.i22 = m[0] / det;
    S.xsize = xs;
    S.ysize = ys;
    S.g11 = xs * S.i11;
    S.g12 = xs * S.i12;
    S.g21 = ys * S.i21;
    S.g22 = ys * S.i22;
    S.gnx = std::hypot(S.g11, S.g12) * (1.0 + 1e-12);
    S.gny = std::hypot(S.g21, S.g22) * (1.0 + 1e-12);
    S.hxs = 0.5 * xs;
    S.hys = 0.5 * ys;
    // bounding rectangle (not used for geometry by the general-box kernels)
    S.Lx = std::fabs(m[0]) + std::fabs(m[1]);
    S.Ly = std::fabs(m[2]) + std::fabs(m[3]);
    S.hLx = 0.5 * S.Lx;
    S.hLy = 0.5 * S.Ly;
    S.cw = S.Lx / xs;
    S.ch = S.Ly / ys;
    S.icw = xs / S.Lx;
    S.ich = ys / S.Ly;
    S.V = (float)pow2_at_least(std::max(S.Lx, S.Ly));
}

// cell grid of every set from the requested cell edge
int plan_grid(dgt_context *c)
{
    c->sets.assign(c->num_sets, SetDesc());
    long long cells = 0, blocks = 0;
    int pbase = 0;
    for (int s = 0; s < c->num_sets; ++s) {
        double Lx = c->boxes[2 * s], Ly = c->boxes[2 * s + 1];
        int ns = c->sizes[s];
        if (c->general) {
            const double *g = &c->gboxes[4 * s];
            const double spacing = std::sqrt(std::fabs(g[0] * g[3] - g[1] * g[2]) / std::max(ns, 1));
            double a;
            if (c->batch) a = (c->cell_size > 0 ? c->cell_size : 1.0) * spacing;
            else a = c->cell_size > 0 ? c->cell_size : spacing;
            SetDesc &S = c->sets[s];
            plan_general_set(S, g, a, ns);
            S.cell_base = (int)cells;
            S.point_base = pbase;
            S.n = ns;
            blocks += set_block_grid(S, (int)blocks);
            cells += (long long)S.xsize * S.ysize;
            pbase += ns;
            if (cells > (1LL << 30)) return DGT_ERR_INVALID_ARGUMENT;
            continue;
        }
        double spacing = std::sqrt(Lx * Ly / std::max(ns, 1));
        double a;
        if (c->batch) a = (c->cell_size > 0 ? c->cell_size : 1.0) * spacing;
        else a = c->cell_size > 0 ? c->cell_size : spacing;
        // at most 64 cells per point (finer cells pay off only inside dense clusters: the 1M
        // mixture builds in 5.8 ms at a fifth of the mean spacing, 7.6 at a quarter, 6.4 at an
        // eighth, where the binning grows to 0.6 ms)
        double amin = std::sqrt(Lx * Ly / (64.0 * std::max(ns, 1) + 64.0));
        if (a < amin) a = amin;
        int xs = std::max(1, (int)std::floor(Lx / a));
        int ys = std::max(1, (int)std::floor(Ly / a));
        SetDesc &S = c->sets[s];
        S.Lx = Lx;
        S.Ly = Ly;
        S.hLx = 0.5 * Lx;
        S.hLy = 0.5 * Ly;
        S.xsize = xs;
        S.ysize = ys;
        S.cw = Lx / xs;
        S.ch = Ly / ys;
        S.icw = (double)xs / Lx;
        S.ich = (double)ys / Ly;
        S.cell_base = (int)cells;
        S.point_base = pbase;
        S.n = ns;
        S.V = (float)pow2_at_least(std::max(Lx, Ly));
        blocks += set_block_grid(S, (int)blocks);
        cells += (long long)xs * ys;
        pbase += ns;
        if (cells > (1LL << 30)) return DGT_ERR_INVALID_ARGUMENT;
    }
    c->total_cells = (int)cells;
    c->total_blocks = (int)blocks;
    return DGT_OK;
}

int alloc_all(dgt_context *c)
{
    int n = std::max(c->n, 1);
    size_t C = (size_t)c->total_cells + 1;
    DGT_TRY(c->d_sets.ensure(sizeof(SetDesc) * c->sets.size()));
    DGT_TRY(cudaMemcpy(c->d_sets.p, c->sets.data(), sizeof(SetDesc) * c->sets.size(), cudaMemcpyHostToDevice));
    if (c->batch) {
        std::vector<int> so(c->n);
        for (int s = 0; s < c->num_sets; ++s)
            for (int k = 0; k < c->sizes[s]; ++k) so[c->sets[s].point_base + k] = s;
        DGT_TRY(c->d_set_of.ensure(sizeof(int) * n));
        DGT_TRY(cudaMemcpy(c->d_set_of.p, so.data(), sizeof(int) * c->n, cudaMemcpyHostToDevice));
    }
    DGT_TRY(c->ccount.ensure(sizeof(int) * C));
    DGT_TRY(c->bcount.ensure(sizeof(int) * ((size_t)c->total_blocks + 1)));
    DGT_TRY(c->cstart.ensure(sizeof(int) * C));
    DGT_TRY(c->bsum.ensure(sizeof(int) * (scan_block_count((int)C) + 1)));
    DGT_TRY(c->cell_of.ensure(sizeof(int) * n));
    DGT_TRY(c->rank.ensure(sizeof(int) * n));
    DGT_TRY(c->sidx.ensure(sizeof(int) * n));
    DGT_TRY(c->slot_of.ensure(sizeof(int) * n));
    DGT_TRY(c->spos.ensure(sizeof(double2) * n));
    DGT_TRY(c->list0.ensure(sizeof(int) * n));
    DGT_TRY(c->list1.ensure(sizeof(int) * n));
    DGT_TRY(c->defer_list.ensure(sizeof(int) * n));
    c->flip_cap = 2 * n + 1024;
    const bool fresh_claim = c->claim.bytes < sizeof(unsigned long long) * (size_t)n;
    DGT_TRY(c->claim.ensure(sizeof(unsigned long long) * n));
    if (fresh_claim) DGT_TRY(cudaMemset(c->claim.p, 0, sizeof(unsigned long long) * n));   // below every key
    DGT_TRY(c->flip0.ensure(sizeof(int2) * (size_t)c->flip_cap));
    DGT_TRY(c->flip1.ensure(sizeof(int2) * (size_t)c->flip_cap));
    DGT_TRY(c->quad.ensure(sizeof(int2) * (size_t)c->flip_cap));
    bool fresh_mark = c->mark.bytes < sizeof(int) * (size_t)n || !c->ctl.p;
    DGT_TRY(c->mark.ensure(sizeof(int) * n));
    DGT_TRY(c->ctl.ensure(sizeof(DevCtl)));
    if (fresh_mark) {
        // marks and the epoch counter start together at zero
        DGT_TRY(cudaMemset(c->mark.p, 0, sizeof(int) * n));
        DGT_TRY(cudaMemset(c->ctl.p, 0, sizeof(DevCtl)));
    }
    DGT_TRY(c->st.ensure(sizeof(DevStatus)));
    if (!c->h_st) DGT_TRY(cudaMallocHost(&c->h_st, sizeof(DevStatus)));
    return DGT_OK;
}

int init_context(dgt_context *c)
{
    if (!c->sms) {
        cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
        if (c->sms <= 0) c->sms = 148;
    }
    c->binned = false;
    int r = plan_grid(c);
    if (r != DGT_OK) return r;
    return alloc_all(c);
}

BinArgs bin_args(dgt_context *c, const double *pts)
{
    BinArgs a;
    a.pos = reinterpret_cast<const double2 *>(pts);
    a.n = c->n;
    a.sets = c->d_sets.as<SetDesc>();
    a.set_of = c->batch ? c->d_set_of.as<int>() : nullptr;
    a.total_cells = c->total_cells;
    a.ccount = c->ccount.as<int>();
    a.cstart = c->cstart.as<int>();
    a.bcount = c->bcount.as<int>();
    a.cell_of = c->cell_of.as<int>();
    a.rank = c->rank.as<int>();
    a.sidx = c->sidx.as<int>();
    a.slot_of = c->slot_of.as<int>();
    a.spos = c->spos.as<double2>();
    a.block_sums = c->bsum.as<int>();
    a.deterministic = c->deterministic;
    a.cond = nullptr;
    a.num_sets = c->num_sets;
    a.total_blocks = c->total_blocks;
    return a;
}

cudaError_t run_bin(dgt_context *c, const double *pts, cudaStream_t s)
{
    PhaseTimer t(c, DGT_PHASE_BIN, s);
    cudaError_t e = cudaMemsetAsync(c->ccount.p, 0, sizeof(int) * ((size_t)c->total_cells + 1), s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(c->bcount.p, 0, sizeof(int) * ((size_t)c->total_blocks + 1), s);
    if (e != cudaSuccess) return e;
    // count, super-block occupancy and scatter; three scan kernels; the in-cell order
    c->launches += (c->n > 0 ? 3 : 0) + 3 + (c->deterministic && c->total_cells > 0 ? 1 : 0);
    e = launch_bin_st(bin_args(c, pts), c->st.as<DevStatus>(), s);
    if (e == cudaSuccess) c->binned = true;
    return e;
}

// Binning for a repair when the context holds a binning of this grid: refresh the
// cell-order positions and rebin only if some point lies more than MAX_SKIN_CELLS cells
// outside the cell that lists it (decided on the device).
cudaError_t run_bin_refresh(dgt_context *c, const double *pts, cudaStream_t s)
{
    PhaseTimer t(c, DGT_PHASE_BIN, s);
    DevStatus *st = c->st.as<DevStatus>();
    BinArgs a = bin_args(c, pts);
    cudaError_t e = launch_refresh(a, st, MAX_SKIN_CELLS, s);
    if (e != cudaSuccess) return e;
    a.cond = &st->rebin;
    e = launch_clear_counts(c->ccount.as<int>(), c->total_cells + 1, c->bcount.as<int>(), c->total_blocks + 1,
                            a.cond, s);
    if (e != cudaSuccess) return e;
    c->launches += (c->n > 0 ? 6 : 3) + 3 + (c->deterministic && c->total_cells > 0 ? 1 : 0);
    return launch_bin_st(a, st, s);
}

RingArgs ring_args(dgt_context *c, const double *pts, int *tri, int *nn, int stride)
{
    RingArgs a;
    std::memset(&a, 0, sizeof(a));
    a.sets = c->d_sets.as<SetDesc>();
    a.set_of = c->batch ? c->d_set_of.as<int>() : nullptr;
    a.pos = reinterpret_cast<const double2 *>(pts);
    a.spos = c->spos.as<double2>();
    a.sidx = c->sidx.as<int>();
    a.slot_of = c->slot_of.as<int>();
    a.cstart = c->cstart.as<int>();
    a.bcount = c->bcount.as<int>();
    a.tri = tri;
    a.nn = nn;
    a.stride = stride;
    a.npoints = c->n;
    a.n_items = c->n;
    a.mark = c->mark.as<int>();
    a.defer_list = c->defer_list.as<int>();
    a.defer_count = &c->st.as<DevStatus>()->defer_count;
    a.skin = &c->st.as<DevStatus>()->skin;
    a.work_budget = c->work_budget;
    a.check = c->check;
    a.general = c->general;
    a.st = c->st.as<DevStatus>();
    return a;
}

// the deferred points (a warp each: long rings, undecided predicates, long scans)
cudaError_t run_deferred(dgt_context *c, const RingArgs &a, cudaStream_t s)
{
    c->launches += 1;
    return launch_deferred(a, c->sms, s);
}

// The kernel shape (and the autotuner's choice of it) applies to global triangulations; the
// rebuild rounds of a repair take the default shape, which is the fastest for their short,
// latency-bound work lists (measured: 256-set ensemble MD step 0.99 ms against 1.05 ms with
// the shape tuned for its build; 4M-point repair 1.07 ms against 1.14 ms with shape 1)
cudaError_t run_build(dgt_context *c, const RingArgs &a, cudaStream_t s)
{
    c->launches += a.n_items > 0 ? 1 : 0;
    return launch_build(a, c->precision == DGT_PRECISION_FP64 ? MODE_F64 : MODE_F32, c->sms,
                        a.repair ? 0 : c->shape, s);
}

// A global build in c->defer_chunks pieces of the cell order, each on a stream of its own
// and followed there by the warp kernel for the points it deferred.  Each piece appends to
// its own segment of the deferred list (its own slots' range, so it cannot overflow) with its
// own counter, so its warp kernel reads an exact count in stream order while the other pieces
// still build.  The pieces overlap one another (no drain between them), and the slowest
// deferred points start as soon as their piece is done.  Nothing spins: events fork the
// pieces from the call's stream and join them back into it.
cudaError_t run_build_chunked(dgt_context *c, const RingArgs &a, cudaStream_t s)
{
    const int K = c->defer_chunks;
    cudaError_t e = c->dcount.ensure(sizeof(int) * MAX_DEFER_CHUNKS);
    if (e != cudaSuccess) return e;
    if (!c->fork_ev && (e = cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    for (int k = 0; k < K; ++k) {
        if (!c->aux[k] && (e = cudaStreamCreateWithFlags(&c->aux[k], cudaStreamNonBlocking)) != cudaSuccess) return e;
        if (!c->aux_ev[k] && (e = cudaEventCreateWithFlags(&c->aux_ev[k], cudaEventDisableTiming)) != cudaSuccess)
            return e;
    }
    int *cnt = c->dcount.as<int>();
    if ((e = cudaMemsetAsync(cnt, 0, sizeof(int) * MAX_DEFER_CHUNKS, s)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(c->fork_ev, s)) != cudaSuccess) return e;
    const int per = (c->n + K - 1) / K;
    int used = 0;
    for (int k = 0; k < K; ++k) {
        const int lo = k * per, items = std::min(per, c->n - lo);
        if (items <= 0) break;
        if ((e = cudaStreamWaitEvent(c->aux[k], c->fork_ev, 0)) != cudaSuccess) return e;
        RingArgs ak = a;
        ak.item_base = lo;
        ak.n_items = items;
        ak.defer_list = a.defer_list + lo;
        ak.defer_count = cnt + k;
        if ((e = run_build(c, ak, c->aux[k])) != cudaSuccess) return e;
        if ((e = run_deferred(c, ak, c->aux[k])) != cudaSuccess) return e;
        if ((e = cudaEventRecord(c->aux_ev[k], c->aux[k])) != cudaSuccess) return e;
        used = k + 1;
    }
    for (int k = 0; k < used; ++k)
        if ((e = cudaStreamWaitEvent(s, c->aux_ev[k], 0)) != cudaSuccess) return e;
    return cudaSuccess;
}

void to_stats(const DevStatus &d, dgt_stats *o)
{
    std::memset(o, 0, sizeof(*o));
    o->points = (long long)d.points;
    o->candidates = (long long)d.candidates;
    o->tests = (long long)d.tests;
    o->fp32_undecided = (long long)d.f32_undecided;
    o->fp64_undecided = (long long)d.f64_undecided;
    o->exact_points = (long long)d.exact_points;
    o->mismatches = (long long)d.mismatches;
    o->insertions = (long long)d.insertions;
    o->flagged = (long long)d.flagged;
    o->repaired = (long long)d.repaired;
    o->cells = (long long)d.cells;
    o->heavy_points = (long long)d.heavy_points;
    o->flips = (long long)d.flips;
    o->flip_spilled = (long long)d.flip_spilled;
    o->flip_rounds = d.flip_rounds;
    o->rebinned = d.rebin;
    o->repair_rounds = d.rounds;
    o->max_ring = d.max_ring;
    o->error_flags = d.err_flags;
}

// read the device status (synchronising) and turn it into a status code
int conclude(dgt_context *c, cudaStream_t s, bool repair_pending)
{
    DGT_TRY(cudaMemcpyAsync(c->h_st, c->st.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, s));
    DGT_TRY(cudaStreamSynchronize(s));
    c->stats_valid = true;
    const DevStatus &d = *c->h_st;
    if (d.err_flags & EF_BAD_INPUT) return DGT_ERR_BAD_POINTS;
    if (d.need_stride > 0) {
        c->max_size = std::max(c->max_size, d.need_stride);
        return DGT_ERR_NEED_RESIZE;
    }
    if (d.err_flags & EF_NOT_CONVERGED) return DGT_ERR_NOT_CONVERGED;
    if (d.err_flags & ~EF_MINIMAGE) return DGT_ERR_DEGENERATE;
    if (repair_pending) return DGT_ERR_NOT_CONVERGED;
    return DGT_OK;
}

bool valid_stride(int stride) { return stride >= 3 && stride <= (1 << 16); }

}  // namespace

extern "C" {

int dgt_version(void) { return 1; }

const char *dgt_error_string(int code)
{
    switch (code) {
    case DGT_OK: return "ok";
    case DGT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case DGT_ERR_CUDA: return "CUDA error";
    case DGT_ERR_NEED_RESIZE: return "a ring is longer than the row stride (see dgt_get_max_size)";
    case DGT_ERR_DEGENERATE: return "degenerate input: a ring could not be closed";
    case DGT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case DGT_ERR_BAD_POINTS: return "a coordinate lies outside [0, L) or is not finite";
    case DGT_ERR_NOT_CONVERGED: return "repair did not reach a fixed point";
    default: return "unknown error";
    }
}

int dgt_create(int n, int max_neighs, double cell_size, double Lx, double Ly, dgt_context **out)
{
    if (!out) return DGT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (n < 0 || !(Lx > 0) || !(Ly > 0) || !std::isfinite(Lx) || !std::isfinite(Ly) || !std::isfinite(cell_size))
        return DGT_ERR_INVALID_ARGUMENT;
    dgt_context *c = new (std::nothrow) dgt_context();
    if (!c) return DGT_ERR_OUT_OF_MEMORY;
    cudaGetDevice(&c->device);
    c->n = n;
    c->num_sets = 1;
    c->sizes.assign(1, n);
    c->boxes = { Lx, Ly };
    c->cell_size = cell_size;
    c->max_size = std::max(4, max_neighs);   // DelaunayGPU.cpp:21
    int r = init_context(c);
    if (r != DGT_OK) {
        dgt_destroy(c);
        return r;
    }
    *out = c;
    return DGT_OK;
}

int dgt_create_batch_general(int num_sets, const int *sizes, const double *boxes4, double cell_size, int max_neighs,
                             dgt_context **out)
{
    if (!out) return DGT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (num_sets <= 0 || !sizes || !boxes4 || !std::isfinite(cell_size)) return DGT_ERR_INVALID_ARGUMENT;
    long long total = 0;
    std::vector<double> g(boxes4, boxes4 + 4 * (size_t)num_sets), rect(2 * (size_t)num_sets);
    for (int s = 0; s < num_sets; ++s) {
        double *b = &g[4 * (size_t)s];
        bool finite = true;
        for (int k = 0; k < 4; ++k) finite &= std::isfinite(b[k]);
        const double det = b[0] * b[3] - b[1] * b[2];
        const double scale = (std::fabs(b[0]) + std::fabs(b[2])) * (std::fabs(b[1]) + std::fabs(b[3]));
        if (sizes[s] < 0 || !finite || !(std::fabs(det) > 1e-12 * scale)) return DGT_ERR_INVALID_ARGUMENT;
        reduce_basis(b);
        rect[2 * s] = std::fabs(b[0]) + std::fabs(b[1]);
        rect[2 * s + 1] = std::fabs(b[2]) + std::fabs(b[3]);
        total += sizes[s];
    }
    if (total > (1LL << 30)) return DGT_ERR_INVALID_ARGUMENT;
    dgt_context *c = new (std::nothrow) dgt_context();
    if (!c) return DGT_ERR_OUT_OF_MEMORY;
    cudaGetDevice(&c->device);
    c->batch = true;
    c->num_sets = num_sets;
    c->n = (int)total;
    c->sizes.assign(sizes, sizes + num_sets);
    c->boxes = rect;
    c->general = 1;
    c->gboxes = g;
    c->cell_size = cell_size;
    c->max_size = std::max(4, max_neighs);
    int r = init_context(c);
    if (r != DGT_OK) {
        dgt_destroy(c);
        return r;
    }
    *out = c;
    return DGT_OK;
}

int dgt_create_batch(int num_sets, const int *sizes, const double *boxes, double cell_size, int max_neighs,
                     dgt_context **out)
{
    if (!out) return DGT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (num_sets <= 0 || !sizes || !boxes || !std::isfinite(cell_size)) return DGT_ERR_INVALID_ARGUMENT;
    long long total = 0;
    for (int s = 0; s < num_sets; ++s) {
        if (sizes[s] < 0 || !(boxes[2 * s] > 0) || !(boxes[2 * s + 1] > 0) || !std::isfinite(boxes[2 * s]) ||
            !std::isfinite(boxes[2 * s + 1]))
            return DGT_ERR_INVALID_ARGUMENT;
        total += sizes[s];
    }
    if (total > (1LL << 30)) return DGT_ERR_INVALID_ARGUMENT;
    dgt_context *c = new (std::nothrow) dgt_context();
    if (!c) return DGT_ERR_OUT_OF_MEMORY;
    cudaGetDevice(&c->device);
    c->batch = true;
    c->num_sets = num_sets;
    c->n = (int)total;
    c->sizes.assign(sizes, sizes + num_sets);
    c->boxes.assign(boxes, boxes + 2 * num_sets);
    c->cell_size = cell_size;
    c->max_size = std::max(4, max_neighs);
    int r = init_context(c);
    if (r != DGT_OK) {
        dgt_destroy(c);
        return r;
    }
    *out = c;
    return DGT_OK;
}

void dgt_destroy(dgt_context *c)
{
    if (!c) return;
    DevBuf *bufs[] = { &c->d_sets, &c->d_set_of, &c->ccount, &c->cstart, &c->cell_of, &c->rank, &c->sidx,
                       &c->slot_of, &c->spos, &c->bsum, &c->mark, &c->list0, &c->list1, &c->defer_list,
                       &c->st, &c->ctl, &c->bcount, &c->claim, &c->flip0, &c->flip1, &c->quad, &c->vcount,
                       &c->hsets, &c->hcount, &c->hstart, &c->hsum, &c->hbucket, &c->hrank, &c->dcount, &c->horder, &c->hperm };
    for (DevBuf *b : bufs) b->release();
    for (int k = 0; k < MAX_DEFER_CHUNKS; ++k) {
        if (c->aux[k]) cudaStreamDestroy(c->aux[k]);
        if (c->aux_ev[k]) cudaEventDestroy(c->aux_ev[k]);
    }
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->h_st) cudaFreeHost(c->h_st);
    for (int p = 0; p < DGT_NUM_PHASES; ++p)
        for (int k = 0; k < 2; ++k)
            if (c->ev[p][k]) cudaEventDestroy(c->ev[p][k]);
    delete c;
}

int dgt_update_list(dgt_context *c, const double *d_points, void *stream)
{
    if (!c || (c->n > 0 && !d_points)) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    DGT_TRY(cudaMemsetAsync(c->st.p, 0, sizeof(DevStatus), s));
    DGT_TRY(run_bin(c, d_points, s));
    c->last_stream = s;
    return DGT_OK;
}

int dgt_global_triangulation(dgt_context *c, const double *d_points, int *d_tri, int *d_nn, int stride,
                             void *stream)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (c->n == 0) return DGT_OK;   // DelaunayGPU.cpp:121-125: nothing to do
    if (!d_points || !d_tri || !d_nn || !valid_stride(stride)) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    begin_call(c, s);
    DGT_TRY(cudaMemsetAsync(c->st.p, 0, sizeof(DevStatus), s));
    DGT_TRY(run_bin(c, d_points, s));
    RingArgs a = ring_args(c, d_points, d_tri, d_nn, stride);
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    DGT_TRY(cudaStreamIsCapturing(s, &capturing));
    if (c->defer_chunks > 1 && capturing == cudaStreamCaptureStatusNone) {
        // the deferred points overlap the build: one phase time for both
        PhaseTimer t(c, DGT_PHASE_BUILD, s);
        DGT_TRY(run_build_chunked(c, a, s));
    } else {
        {
            PhaseTimer t(c, DGT_PHASE_BUILD, s);
            DGT_TRY(run_build(c, a, s));
        }
        {
            PhaseTimer t(c, DGT_PHASE_SLOW, s);
            DGT_TRY(run_deferred(c, a, s));
        }
    }
    c->launches += 1;
    DGT_TRY(launch_call_end(c->ctl.as<DevCtl>(), c->st.as<DevStatus>(), 0, s));
    if (!c->safety) return DGT_OK;
    return conclude(c, s, false);
}

}  // extern "C"

namespace {

// Test-and-repair on the context's stream.  fixed_rounds == 0: rounds are launched in
// batches and the host stops once a list is empty (needs a synchronisation per batch);
// fixed_rounds > 0: exactly that many rounds, no host synchronisation (graph capture),
// an unfinished queue sets DGT_FLAG_NOT_CONVERGED in the device flags.
// An MD step's displacement, fused into the repair: one kernel moves and wraps every point
// and measures how far it now lies outside the cell that lists it (the local test then skips
// that measurement); the step counter advances at the end of the call.
struct MdMove {
    double sigma;
    unsigned long long seed;
};

int repair_impl(dgt_context *c, const double *d_points, int *d_tri, int *d_nn, int stride, cudaStream_t s,
                int fixed_rounds, bool conclude_now, const MdMove *md = nullptr)
{
    DevStatus *dst = c->st.as<DevStatus>();
    DevCtl *ctl = c->ctl.as<DevCtl>();
    DGT_TRY(cudaMemsetAsync(c->st.p, 0, sizeof(DevStatus), s));
    const bool measured = md && c->flip && c->binned;
    if (md) {
        c->launches += 1;
        DGT_TRY(launch_displace_md(reinterpret_cast<double2 *>(const_cast<double *>(d_points)), c->n,
                                   c->d_sets.as<SetDesc>(), c->batch ? c->d_set_of.as<int>() : nullptr, md->sigma,
                                   md->seed, &ctl->step, measured ? c->cell_of.as<int>() : nullptr, dst, s));
    }
    // With the cell lists of an earlier binning of this grid, flip mode measures how far the
    // points left their cells in the local test and decides on rebinning only once the rebuild rounds
    // need the lists (they read candidate positions through the index, so the cell-order copy
    // needs no refresh); rebuild-only mode refreshes it first (its test runs in cell order).
    const bool fold = c->flip && c->binned;
    if (!c->binned) DGT_TRY(run_bin(c, d_points, s));
    else if (!fold) DGT_TRY(run_bin_refresh(c, d_points, s));
    int *lists[2] = { c->list0.as<int>(), c->list1.as<int>() };
    TestArgs t;
    t.sets = c->d_sets.as<SetDesc>();
    t.set_of = c->batch ? c->d_set_of.as<int>() : nullptr;
    t.pos = reinterpret_cast<const double2 *>(d_points);
    t.sidx = c->sidx.as<int>();
    t.spos = c->spos.as<double2>();
    t.tri = d_tri;
    t.nn = d_nn;
    t.stride = stride;
    t.n = c->n;
    t.mark = c->mark.as<int>();
    t.epoch_ptr = &ctl->epoch;
    t.list = lists[0];
    t.list_count = &dst->list_count[0];
    int2 *flips[2] = { c->flip0.as<int2>(), c->flip1.as<int2>() };
    t.flip_list = c->flip ? flips[0] : nullptr;
    t.flip_count = &dst->flip_count[0];
    t.flip_cap = c->flip_cap;
    t.rcell_of = (fold && !measured) ? c->cell_of.as<int>() : nullptr;
    t.general = c->general;
    t.st = dst;
    {
        PhaseTimer pt(c, DGT_PHASE_TEST, s);
        c->launches += 1;
        DGT_TRY(launch_test(t, s));
    }
    phase_begin(c, DGT_PHASE_REPAIR, s);
    if (c->flip) {
        // Lawson flips first; what they cannot settle joins the rebuild list (list 0)
        FlipArgs f;
        std::memset(&f, 0, sizeof(f));
        f.sets = t.sets;
        f.set_of = t.set_of;
        f.general = c->general;
        f.pos = t.pos;
        f.tri = d_tri;
        f.nn = d_nn;
        f.stride = stride;
        f.n = c->n;
        f.mark = t.mark;
        f.epoch_ptr = &ctl->epoch;
        f.rebuild_list = lists[0];
        f.rebuild_count = &dst->list_count[0];
        f.claim = c->claim.as<unsigned long long>();
        f.stamp_ptr = &ctl->flip_stamp;
        f.quad = c->quad.as<int2>();
        f.cap = c->flip_cap;
        f.st = dst;
        int fr = 0;
        for (;;) {
            const int batch = fixed_rounds > 0 ? c->graph_flip_rounds : FLIP_BATCH;
            for (int b = 0; b < batch; ++b, ++fr) {
                f.cur = flips[fr & 1];
                f.cur_count = &dst->flip_count[fr & 1];
                f.next = flips[(fr + 1) & 1];
                f.next_count = &dst->flip_count[(fr + 1) & 1];
                c->launches += 2;
                DGT_TRY(launch_flip_round(f, fr, c->sms, s));
            }
            if (fixed_rounds > 0 || fr >= MAX_FLIP_ROUNDS) break;
            int left = 0;
            DGT_TRY(cudaMemcpyAsync(&left, &dst->flip_count[fr & 1], sizeof(int), cudaMemcpyDeviceToHost, s));
            DGT_TRY(cudaStreamSynchronize(s));
            if (left <= c->sms * SPILL_EDGES_PER_SM) break;
        }
        f.cur = flips[fr & 1];
        f.cur_count = &dst->flip_count[fr & 1];
        c->launches += 2;
        DGT_TRY(launch_flip_spill(f, fr, ctl, c->sms, s));
    }
    if (fold) {
        // timed as the bin phase (inside the repair phase's span)
        PhaseTimer bt(c, DGT_PHASE_BIN, s);
        DGT_TRY(launch_rebin_decide(dst, MAX_SKIN_CELLS, s));
        BinArgs a = bin_args(c, d_points);
        a.cond = &dst->rebin;
        DGT_TRY(launch_clear_counts(c->ccount.as<int>(), c->total_cells + 1, c->bcount.as<int>(), c->total_blocks + 1,
                                    a.cond, s));
        DGT_TRY(launch_bin_st(a, dst, s));
        c->launches += 2 + (c->n > 0 ? 3 : 0) + 3 + (c->deterministic && c->total_cells > 0 ? 1 : 0);
    }
    if (c->flip) {
        c->launches += 1;
        DGT_TRY(launch_expand(lists[0], &dst->list_count[0], c->n, d_tri, d_nn, stride, c->n, c->mark.as<int>(),
                              &ctl->epoch, c->sms, s));
    }
    int round = 0;
    bool pending = false;
    for (;;) {
        // a batch of rounds; each kernel reads its item count on the device
        int batch = fixed_rounds > 0 ? fixed_rounds : (round == 0 ? FIRST_ROUNDS : NEXT_ROUNDS);
        for (int b = 0; b < batch; ++b, ++round) {
            int cur = round & 1, nxt = cur ^ 1;
            DGT_TRY(cudaMemsetAsync(&dst->list_count[nxt], 0, sizeof(int), s));
            DGT_TRY(cudaMemsetAsync(&dst->defer_count, 0, sizeof(int), s));
            RingArgs a = ring_args(c, d_points, d_tri, d_nn, stride);
            a.worklist = lists[cur];
            a.worklist_count = &dst->list_count[cur];
            a.n_items = c->n;
            a.repair = 1;
            a.cand_by_index = 1;
            // a round of at most 16 points per SM goes to the warp-per-point kernel whole (two
            // points per resident warp)
            a.warp_items = c->sms * 16;
            a.epoch_ptr = &ctl->epoch;
            a.round = round;
            a.next_list = lists[nxt];
            a.next_count = &dst->list_count[nxt];
            DGT_TRY(run_build(c, a, s));
            DGT_TRY(run_deferred(c, a, s));
        }
        if (fixed_rounds > 0) break;
        int left = 0;
        DGT_TRY(cudaMemcpyAsync(&left, &dst->list_count[round & 1], sizeof(int), cudaMemcpyDeviceToHost, s));
        DGT_TRY(cudaStreamSynchronize(s));
        if (left == 0) break;
        if (round > 256) {
            pending = true;
            break;
        }
    }
    phase_end(c, DGT_PHASE_REPAIR, s);
    c->launches += 1;
    DGT_TRY(launch_call_end(ctl, dst, round, s, md != nullptr));
    if (!conclude_now) return DGT_OK;
    return conclude(c, s, pending);
}

}  // namespace

extern "C" {

int dgt_test_and_repair(dgt_context *c, const double *d_points, int *d_tri, int *d_nn, int stride, void *stream)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (c->n == 0) return DGT_OK;
    if (!d_points || !d_tri || !d_nn || !valid_stride(stride)) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    begin_call(c, s);
    if (c->safety) return repair_impl(c, d_points, d_tri, d_nn, stride, s, 0, true);
    return repair_impl(c, d_points, d_tri, d_nn, stride, s, ASYNC_ROUNDS, false);
}

int dgt_set_cell_size(dgt_context *c, double cell_size)
{
    if (!c || !std::isfinite(cell_size)) return DGT_ERR_INVALID_ARGUMENT;
    c->cell_size = cell_size;
    return init_context(c);
}

int dgt_set_box(dgt_context *c, double Lx, double Ly)
{
    if (!c || c->batch || !(Lx > 0) || !(Ly > 0) || !std::isfinite(Lx) || !std::isfinite(Ly))
        return DGT_ERR_INVALID_ARGUMENT;
    c->boxes = { Lx, Ly };
    c->general = 0;
    return init_context(c);
}

int dgt_set_box_general(dgt_context *c, double x11, double x12, double x21, double x22)
{
    if (!c || c->batch) return DGT_ERR_INVALID_ARGUMENT;
    const double m[4] = { x11, x12, x21, x22 };
    for (double v : m)
        if (!std::isfinite(v)) return DGT_ERR_INVALID_ARGUMENT;
    const double det = x11 * x22 - x12 * x21;
    const double scale = (std::fabs(x11) + std::fabs(x21)) * (std::fabs(x12) + std::fabs(x22));
    if (!(std::fabs(det) > 1e-12 * scale)) return DGT_ERR_INVALID_ARGUMENT;   // degenerate lattice
    if (x12 == 0.0 && x21 == 0.0 && x11 > 0.0 && x22 > 0.0) return dgt_set_box(c, x11, x22);
    double g[4] = { x11, x12, x21, x22 };
    reduce_basis(g);
    c->gboxes.assign(g, g + 4);
    c->general = 1;
    c->boxes = { std::fabs(g[0]) + std::fabs(g[1]), std::fabs(g[2]) + std::fabs(g[3]) };
    return init_context(c);
}

int dgt_get_box(const dgt_context *c, double *out4)
{
    if (!c || !out4 || c->batch) return DGT_ERR_INVALID_ARGUMENT;
    if (c->general) {
        std::memcpy(out4, c->gboxes.data(), sizeof(double) * 4);
    } else {
        out4[0] = c->boxes[0];
        out4[1] = 0.0;
        out4[2] = 0.0;
        out4[3] = c->boxes[1];
    }
    return DGT_OK;
}

int dgt_set_safety_mode(dgt_context *c, int on)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    c->safety = on ? 1 : 0;
    return DGT_OK;
}

int dgt_set_precision(dgt_context *c, int precision)
{
    if (!c || (precision != DGT_PRECISION_FP32_FILTER && precision != DGT_PRECISION_FP64))
        return DGT_ERR_INVALID_ARGUMENT;
    c->precision = precision;
    return DGT_OK;
}

int dgt_set_check_mode(dgt_context *c, int on)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    c->check = on ? 1 : 0;
    return DGT_OK;
}

int dgt_resize(dgt_context *c, int max_neighs)
{
    if (!c || max_neighs < 3) return DGT_ERR_INVALID_ARGUMENT;
    c->max_size = max_neighs;
    return DGT_OK;
}

int dgt_get_max_size(const dgt_context *c, int *out)
{
    if (!c || !out) return DGT_ERR_INVALID_ARGUMENT;
    *out = c->max_size;
    return DGT_OK;
}

int dgt_get_num_points(const dgt_context *c, int *out)
{
    if (!c || !out) return DGT_ERR_INVALID_ARGUMENT;
    *out = c->n;
    return DGT_OK;
}

int dgt_restride(const int *d_src, int src_stride, int *d_dst, int dst_stride, const int *d_nn, int n, void *stream)
{
    if (n < 0 || (n > 0 && (!d_src || !d_dst)) || src_stride < 1 || dst_stride < 1 || d_src == d_dst)
        return DGT_ERR_INVALID_ARGUMENT;
    DGT_TRY(launch_restride(d_src, src_stride, d_dst, dst_stride, d_nn, n, (cudaStream_t)stream));
    return DGT_OK;
}

int dgt_get_stats(dgt_context *c, dgt_stats *out)
{
    if (!c || !out) return DGT_ERR_INVALID_ARGUMENT;
    if (!c->stats_valid) {
        DGT_TRY(cudaMemcpyAsync(c->h_st, c->st.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->last_stream));
        DGT_TRY(cudaStreamSynchronize(c->last_stream));
        c->stats_valid = true;
    }
    to_stats(*c->h_st, out);
    out->launches = c->launches;
    DevCtl ctl;
    DGT_TRY(cudaMemcpy(&ctl, c->ctl.p, sizeof(DevCtl), cudaMemcpyDeviceToHost));
    out->sticky_flags = ctl.sticky;
    out->repair_calls = (long long)ctl.calls;
    out->md_step = (long long)ctl.step;
    return DGT_OK;
}

int dgt_set_timing(dgt_context *c, int on)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (on && !c->ev[0][0]) {
        for (int p = 0; p < DGT_NUM_PHASES; ++p)
            for (int k = 0; k < 2; ++k) DGT_TRY(cudaEventCreate(&c->ev[p][k]));
    }
    c->timing = on != 0;
    return DGT_OK;
}

int dgt_get_phase_times(dgt_context *c, double *out_ms)
{
    if (!c || !out_ms) return DGT_ERR_INVALID_ARGUMENT;
    DGT_TRY(cudaStreamSynchronize(c->last_stream));
    for (int p = 0; p < DGT_NUM_PHASES; ++p) {
        out_ms[p] = -1.0;
        if (c->timing && c->ev_used[p]) {
            float ms = 0.f;
            DGT_TRY(cudaEventElapsedTime(&ms, c->ev[p][0], c->ev[p][1]));
            out_ms[p] = ms;
        }
    }
    return DGT_OK;
}

int dgt_displace(dgt_context *c, double *d_points, double sigma, unsigned long long seed, unsigned long long step,
                 void *stream)
{
    if (!c || (c->n > 0 && !d_points) || !(sigma >= 0) || !std::isfinite(sigma)) return DGT_ERR_INVALID_ARGUMENT;
    unsigned long long *step_ptr = step == DGT_STEP_AUTO ? &c->ctl.as<DevCtl>()->step : nullptr;
    DGT_TRY(launch_displace(reinterpret_cast<double2 *>(d_points), c->n, c->d_sets.as<SetDesc>(),
                            c->batch ? c->d_set_of.as<int>() : nullptr, sigma, seed, step, step_ptr,
                            (cudaStream_t)stream));
    return DGT_OK;
}

int dgt_md_step(dgt_context *c, double *d_points, int *d_tri, int *d_nn, int stride, double sigma,
                unsigned long long seed, int rounds, void *stream)
{
    if (!c || rounds < 1 || rounds > 64) return DGT_ERR_INVALID_ARGUMENT;
    if (c->n == 0) return DGT_OK;
    if (!d_points || !d_tri || !d_nn || !valid_stride(stride)) return DGT_ERR_INVALID_ARGUMENT;
    if (!(sigma >= 0) || !std::isfinite(sigma)) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    begin_call(c, s);
    const MdMove md{ sigma, seed };
    return repair_impl(c, d_points, d_tri, d_nn, stride, s, rounds, false, &md);
}

struct dgt_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int steps = 0;
};

int dgt_md_graph_create(dgt_context *c, double *d_points, int *d_tri, int *d_nn, int stride, double sigma,
                        unsigned long long seed, int steps, int rounds, void *stream, dgt_graph **out)
{
    if (!out) return DGT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!c || !stream || steps < 1 || steps > 100000) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    const bool timing = c->timing;
    c->timing = false;   // no event records inside the graph
    DGT_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int r = DGT_OK;
    for (int k = 0; k < steps && r == DGT_OK; ++k) r = dgt_md_step(c, d_points, d_tri, d_nn, stride, sigma, seed, rounds, stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    c->timing = timing;
    if (r != DGT_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return cuda_status(e);
    dgt_graph *G = new (std::nothrow) dgt_graph();
    if (!G) {
        cudaGraphDestroy(g);
        return DGT_ERR_OUT_OF_MEMORY;
    }
    G->graph = g;
    G->steps = steps;
    e = cudaGraphInstantiate(&G->exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        delete G;
        return cuda_status(e);
    }
    *out = G;
    return DGT_OK;
}

int dgt_md_graph_launch(dgt_graph *g, void *stream)
{
    if (!g || !g->exec) return DGT_ERR_INVALID_ARGUMENT;
    DGT_TRY(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return DGT_OK;
}

void dgt_md_graph_destroy(dgt_graph *g)
{
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

int dgt_set_kernel_shape(dgt_context *c, int shape)
{
    if (!c || shape < 0 || shape >= KERNEL_SHAPES) return DGT_ERR_INVALID_ARGUMENT;
    c->shape = shape;
    return DGT_OK;
}

int dgt_validate(dgt_context *c, const double *d_points, const int *d_tri, const int *d_nn, int stride,
                 dgt_validation *out, void *stream)
{
    if (!c || !out) return DGT_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (c->n == 0) {
        out->valid = 1;
        return DGT_OK;
    }
    if (!d_points || !d_tri || !d_nn || !valid_stride(stride)) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    DGT_TRY(c->vcount.ensure(sizeof(unsigned long long) * 8));
    unsigned long long *d = c->vcount.as<unsigned long long>();
    DGT_TRY(launch_validate(c->d_sets.as<SetDesc>(), c->batch ? c->d_set_of.as<int>() : nullptr,
                            reinterpret_cast<const double2 *>(d_points), d_tri, d_nn, stride, c->n, d, c->sms,
                            c->general, s));
    unsigned long long h[7];
    DGT_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
    DGT_TRY(cudaStreamSynchronize(s));
    out->sum_neighbors = (long long)h[0];
    out->bad_rows = (long long)h[1];
    out->asymmetric = (long long)h[2];
    out->not_ccw = (long long)h[3];
    out->winding = (long long)h[4];
    out->not_delaunay = (long long)h[5];
    out->points = (long long)h[6];
    out->valid = out->bad_rows == 0 && out->asymmetric == 0 && out->not_ccw == 0 && out->winding == 0 &&
                 out->not_delaunay == 0 && out->sum_neighbors == 6 * out->points;
    return DGT_OK;
}

int dgt_get_cell_order(dgt_context *c, int *d_order, void *stream)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (c->n == 0) return DGT_OK;
    if (!d_order || !c->binned) return DGT_ERR_INVALID_ARGUMENT;
    DGT_TRY(cudaMemcpyAsync(d_order, c->sidx.p, sizeof(int) * (size_t)c->n, cudaMemcpyDeviceToDevice,
                            (cudaStream_t)stream));
    return DGT_OK;
}

int dgt_get_hilbert_order(dgt_context *c, const double *d_points, int *d_order, void *stream)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (c->n == 0) return DGT_OK;
    if (!d_points || !d_order) return DGT_ERR_INVALID_ARGUMENT;
    // per set: the smallest 2^k x 2^k grid with at least one square per point (k <= 15),
    // its scale over the box (a general box: over the fractional frame) and its first key
    std::vector<HilbertSet> hs((size_t)c->num_sets);
    long long buckets = 0;
    for (int s = 0; s < c->num_sets; ++s) {
        int k = 1;
        while (k < 15 && (1LL << (2 * k)) < (long long)c->sizes[s]) ++k;
        const double g = (double)(1 << k);
        hs[s].k = k;
        hs[s].base = (int)buckets;
        hs[s].sx = c->general ? g : g / c->boxes[2 * s];
        hs[s].sy = c->general ? g : g / c->boxes[2 * s + 1];
        buckets += 1LL << (2 * k);
        if (buckets >= (1LL << 31) - 1) return DGT_ERR_INVALID_ARGUMENT;
    }
    const int nb = (int)buckets;
    cudaStream_t st = (cudaStream_t)stream;
    DGT_TRY(c->hsets.ensure(sizeof(HilbertSet) * hs.size()));
    DGT_TRY(c->hcount.ensure(sizeof(int) * ((size_t)nb + 1)));
    DGT_TRY(c->hstart.ensure(sizeof(int) * ((size_t)nb + 1)));
    DGT_TRY(c->hsum.ensure(sizeof(int) * ((size_t)scan_block_count(nb + 1) + 1)));
    DGT_TRY(c->hbucket.ensure(sizeof(int) * (size_t)c->n));
    DGT_TRY(c->hrank.ensure(sizeof(int) * (size_t)c->n));
    DGT_TRY(cudaMemcpyAsync(c->hsets.p, hs.data(), sizeof(HilbertSet) * hs.size(), cudaMemcpyHostToDevice, st));
    HilbertArgs a;
    a.pos = reinterpret_cast<const double2 *>(d_points);
    a.n = c->n;
    a.sets = c->d_sets.as<SetDesc>();
    a.set_of = c->batch ? c->d_set_of.as<int>() : nullptr;
    a.hsets = c->hsets.as<HilbertSet>();
    a.buckets = nb;
    a.hcount = c->hcount.as<int>();
    a.hstart = c->hstart.as<int>();
    a.bsum = c->hsum.as<int>();
    a.hbucket = c->hbucket.as<int>();
    a.hrank = c->hrank.as<int>();
    a.order = d_order;
    DGT_TRY(launch_hilbert_order(a, st));
    // the host copy of the descriptors must outlive the transfer
    DGT_TRY(cudaStreamSynchronize(st));
    return DGT_OK;
}

int dgt_hilbert_sort_points(dgt_context *c, double *d_points, int *d_order, void *stream)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (c->n == 0) return DGT_OK;
    if (!d_points) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    int *order = d_order;
    if (!order) {
        DGT_TRY(c->horder.ensure(sizeof(int) * (size_t)c->n));
        order = c->horder.as<int>();
    }
    int r = dgt_get_hilbert_order(c, d_points, order, stream);
    if (r != DGT_OK) return r;
    DGT_TRY(c->hperm.ensure(sizeof(double2) * (size_t)c->n));
    DGT_TRY(launch_gather_points(reinterpret_cast<const double2 *>(d_points), order, c->n, c->hperm.as<double2>(), s));
    DGT_TRY(cudaMemcpyAsync(d_points, c->hperm.p, sizeof(double2) * (size_t)c->n, cudaMemcpyDeviceToDevice, s));
    return DGT_OK;
}

int dgt_set_graph_flip_rounds(dgt_context *c, int rounds)
{
    if (!c || rounds < 0 || rounds > MAX_FLIP_ROUNDS) return DGT_ERR_INVALID_ARGUMENT;
    c->graph_flip_rounds = rounds;
    return DGT_OK;
}

int dgt_set_flip_repair(dgt_context *c, int on)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    c->flip = on ? 1 : 0;
    return DGT_OK;
}

int dgt_set_deferred_overlap(dgt_context *c, int chunks)
{
    if (!c || chunks < 1 || chunks > MAX_DEFER_CHUNKS) return DGT_ERR_INVALID_ARGUMENT;
    c->defer_chunks = chunks;
    return DGT_OK;
}

int dgt_set_work_budget(dgt_context *c, int budget)
{
    if (!c || budget < 0) return DGT_ERR_INVALID_ARGUMENT;
    c->work_budget = budget;
    return DGT_OK;
}

int dgt_get_tuning(const dgt_context *c, double *cell_size, int *shape, int *ring_capacity, int *block)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    if (cell_size) *cell_size = c->cell_size;
    if (shape) *shape = c->shape;
    if (ring_capacity) *ring_capacity = kernel_shape_cap(c->shape);
    if (block) *block = kernel_shape_block(c->shape);
    return DGT_OK;
}

}  // extern "C"

namespace {

// tuned (cell size relative to the mean spacing, kernel shape, work budget) per class of input
typedef std::tuple<int, int, int, int> TuneKey;   // log2 points, log2 sets, contrast class, precision
struct TuneVal {
    double rel;
    int shape;
    int budget;
    int chunks;
};
std::map<TuneKey, TuneVal> g_tune_cache;
std::mutex g_tune_mutex;

__global__ void k_max_count(const int *ccount, int cells, int *out)
{
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cells; i += gridDim.x * blockDim.x) m = max(m, ccount[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

int ilog2(long long v)
{
    int r = 0;
    while (v > 1) {
        v >>= 1;
        ++r;
    }
    return r;
}

// mean spacing of a single-set context (cell sizes are absolute there)
double spacing_of(const dgt_context *c)
{
    const double area = c->general ? std::fabs(c->gboxes[0] * c->gboxes[3] - c->gboxes[1] * c->gboxes[2])
                                   : c->boxes[0] * c->boxes[1];
    return std::sqrt(area / std::max(c->n, 1));
}

void set_relative_cell(dgt_context *c, double rel)
{
    c->cell_size = c->batch ? rel : rel * spacing_of(c);
}

}  // namespace

extern "C" {

int dgt_autotune(dgt_context *c, const double *d_points, int *d_tri, int *d_nn, int stride, void *stream,
                 dgt_tune_result *out)
{
    if (!c || !out) return DGT_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (c->n == 0) return DGT_OK;
    if (!d_points || !d_tri || !d_nn || !valid_stride(stride)) return DGT_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    const int safety = c->safety, timing = c->timing;
    const double cell0 = c->cell_size;
    const int shape0 = c->shape, budget0 = c->work_budget, chunks0 = c->defer_chunks;
    c->safety = 1;
    c->timing = false;
    // density contrast of the input on the mean-spacing grid: largest cell count
    set_relative_cell(c, 1.0);
    int r = init_context(c);
    if (r != DGT_OK) return r;
    DGT_TRY(cudaMemsetAsync(c->st.p, 0, sizeof(DevStatus), s));
    DGT_TRY(run_bin(c, d_points, s));
    int *dmax = &c->st.as<DevStatus>()->need_stride;   // scratch word: every call clears the status
    DGT_TRY(cudaMemsetAsync(dmax, 0, sizeof(int), s));
    k_max_count<<<std::min(1024, (c->total_cells + 255) / 256 + 1), 256, 0, s>>>(c->ccount.as<int>(), c->total_cells,
                                                                                dmax);
    int maxc = 0;
    DGT_TRY(cudaMemcpyAsync(&maxc, dmax, sizeof(int), cudaMemcpyDeviceToHost, s));
    DGT_TRY(cudaStreamSynchronize(s));
    const int contrast = maxc <= 8 ? 0 : (maxc <= 32 ? 1 : 2);
    const TuneKey key(ilog2(c->n), ilog2(c->num_sets), contrast, c->precision);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            set_relative_cell(c, it->second.rel);
            c->shape = it->second.shape;
            c->work_budget = it->second.budget;
            c->defer_chunks = it->second.chunks;
            c->safety = safety;
            c->timing = timing;
            out->cell_size = c->cell_size;
            out->shape = c->shape;
            out->work_budget = c->work_budget;
            out->deferred_chunks = c->defer_chunks;
            out->from_cache = 1;
            return init_context(c);
        }
    }
    cudaEvent_t e0, e1;
    DGT_TRY(cudaEventCreate(&e0));
    DGT_TRY(cudaEventCreate(&e1));
    auto trial = [&](double rel, int shape, float *ms) -> int {
        set_relative_cell(c, rel);
        c->shape = shape;
        int rr = init_context(c);
        if (rr != DGT_OK) return rr;
        rr = dgt_global_triangulation(c, d_points, d_tri, d_nn, stride, stream);   // warm-up
        if (rr != DGT_OK) return rr;
        cudaEventRecord(e0, s);
        rr = dgt_global_triangulation(c, d_points, d_tri, d_nn, stride, stream);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms, e0, e1);
        out->trials++;
        return rr;
    };
    // uniform-ish inputs: around the mean spacing; dense clusters: much finer cells too
    const double rels_uniform[] = { 1.0, 0.7, 0.85, 1.2, 1.45 };
    const double rels_clustered[] = { 1.0, 0.5, 0.35, 0.25, 0.18, 0.125 };
    const std::vector<double> rels = contrast < 2 ? std::vector<double>(rels_uniform, rels_uniform + 5)
                                                  : std::vector<double>(rels_clustered, rels_clustered + 6);
    double best_rel = 1.0;
    int best_shape = 0;
    float best = 1e30f;
    int rr = DGT_OK;
    c->defer_chunks = 1;
    // any failure (including a stride too small for some ring: the caller grows the
    // array and tunes again) ends the sweep with the original settings restored
    for (double rel : rels) {
        float ms = 0;
        rr = trial(rel, 0, &ms);
        if (rr != DGT_OK) break;
        if (rel == 1.0) out->default_ms = ms;
        if (ms < best) {
            best = ms;
            best_rel = rel;
        }
    }
    for (int shape = 1; shape < KERNEL_SHAPES && rr == DGT_OK; ++shape) {
        float ms = 0;
        rr = trial(best_rel, shape, &ms);
        if (rr != DGT_OK) break;
        if (ms < best) {
            best = ms;
            best_shape = shape;
        }
    }
    // clustered inputs: how long a point may scan in the per-thread kernel before the warp
    // kernel takes it over (uniform inputs stay far below any of these)
    int best_budget = budget0;
    if (contrast == 2) {
        const int budgets[] = { 512, 2048 };
        for (int b : budgets) {
            if (rr != DGT_OK) break;
            float ms = 0;
            c->work_budget = b;
            rr = trial(best_rel, best_shape, &ms);
            if (rr != DGT_OK) break;
            if (ms < best) {
                best = ms;
                best_budget = b;
            }
        }
        c->work_budget = best_budget;
    }
    // clustered inputs: the build in 2-4 pieces, the deferred points of each overlapping the
    // rest (the deferred phase is set by its slowest points, which then start before the
    // per-thread kernel has finished; 1M-point mixture: 8.2-8.4 ms in one piece, 7.2-8.1 ms
    // in 2-8, varying with where the slowest points fall)
    int best_chunks = 1;
    for (int k = 2; k <= 4 && contrast == 2 && rr == DGT_OK; ++k) {
        float ms = 0;
        c->defer_chunks = k;
        rr = trial(best_rel, best_shape, &ms);
        if (rr == DGT_OK && ms < best) {
            best = ms;
            best_chunks = k;
        }
    }
    c->defer_chunks = best_chunks;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->safety = safety;
    c->timing = timing;
    if (rr != DGT_OK) {
        c->cell_size = cell0;
        c->shape = shape0;
        c->work_budget = budget0;
        c->defer_chunks = chunks0;
        init_context(c);
        return rr;
    }
    set_relative_cell(c, best_rel);
    c->shape = best_shape;
    c->work_budget = best_budget;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune_cache[key] = TuneVal{ best_rel, best_shape, best_budget, best_chunks };
    }
    out->cell_size = c->cell_size;
    out->shape = best_shape;
    out->work_budget = best_budget;
    out->deferred_chunks = best_chunks;
    out->best_ms = best;
    r = init_context(c);
    if (r != DGT_OK) return r;
    // leave a triangulation of d_points with the chosen configuration in the outputs
    return dgt_global_triangulation(c, d_points, d_tri, d_nn, stride, stream);
}

int dgt_clear_flags(dgt_context *c, void *stream)
{
    if (!c) return DGT_ERR_INVALID_ARGUMENT;
    DGT_TRY(cudaMemsetAsync(&c->ctl.as<DevCtl>()->sticky, 0, sizeof(int), (cudaStream_t)stream));
    return DGT_OK;
}

}  // extern "C"

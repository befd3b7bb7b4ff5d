// Bucket grid as a CSR counting sort by cell (replaces the reference's fixed-capacity
// buckets idxs[bin*Nmax+k] with an overflow-retry loop, cellListGPU.cpp:404-460 and
// cellListGPU.cu:20-58):
//   count    cell of every point (floor(x / cell edge), clamped), atomic rank in its cell
//   scan     exclusive prefix sum of the counts -> cstart (one pass of reduce / scan / apply)
//   scatter  slot = cstart[cell] + rank; cell-order copies of index and position
//   order    points of a cell sorted by index, so the cell order (and every candidate order
//            derived from it) is independent of atomic arrival order
// No host round trip: capacity is exact by construction.
//
// Repair without rebinning: the cell lists of the last binning stay valid as candidate
// lists while no point lies more than half a cell outside the cell that lists it; the ring
// kernels then read candidate positions through the index and widen certification by that
// distance.
// Every binning kernel takes a device-side condition, so deciding needs no host round trip
// (and a captured graph replays the decision).
#include "dgt_internal.cuh"

namespace dgt {

__device__ __forceinline__ int cell_index(const SetDesc &S, double2 p)
{
    const double2 f = S.general ? cell_pos<true>(S, p) : cell_pos<false>(S, p);
    int cx = (int)floor(f.x), cy = (int)floor(f.y);
    cx = min(max(cx, 0), S.xsize - 1);
    cy = min(max(cy, 0), S.ysize - 1);
    return S.cell_base + cy * S.xsize + cx;
}

// Inputs the kernels accept: inside the rectangular box; any finite position for a general
// box (its fractional coordinates are wrapped)
__device__ __forceinline__ bool bad_input(const SetDesc &S, double2 p)
{
    if (S.general) return !(isfinite(p.x) && isfinite(p.y));
    return !(p.x >= 0.0 && p.x < S.Lx && p.y >= 0.0 && p.y < S.Ly);
}

__device__ __forceinline__ bool skip(const int *cond) { return cond && *cond == 0; }

// the zeroed counters a binning starts from (replaces two memsets when the binning is
// conditional)
__global__ void __launch_bounds__(256) k_clear_counts(int *ccount, int ncell, int *bcount, int nblock, const int *cond)
{
    if (skip(cond)) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncell || k < nblock; k += gridDim.x * blockDim.x) {
        if (k < ncell) ccount[k] = 0;
        if (k < nblock) bcount[k] = 0;
    }
}

// The cell of every point and its rank among the points of that cell, plus the occupancy of
// the 8 x 8-cell blocks.  (Warp-aggregated atomics, one
// per group of lanes sharing a cell via __match_any_sync, were measured and left out: points
// arrive in index order, which is spatially random even for the clustered inputs, so a warp
// almost never holds two points of one cell, and the match made the 4M-point binning 0.26 ->
// 0.33 ms.)
__global__ void __launch_bounds__(256) k_count(BinArgs a, DevStatus *st)
{
    if (skip(a.cond)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const SetDesc &S = a.sets[a.set_of ? a.set_of[i] : 0];
        double2 p = a.pos[i];
        if (bad_input(S, p)) {
            atomicOr(&st->err_flags, EF_BAD_INPUT);
            p = make_double2(0.0, 0.0);
        }
        int c = cell_index(S, p);
        a.cell_of[i] = c;
        a.rank[i] = atomicAdd(&a.ccount[c], 1);
        int lc = c - S.cell_base, cy = lc / S.xsize, cx = lc - cy * S.xsize;
        atomicAdd(&a.bcount[S.block_base + (cy >> BLOCK_SHIFT) * S.bxsize + (cx >> BLOCK_SHIFT)], 1);
    }
}

// Super-block occupancy from the block counts: every non-empty block adds one to its
// super-block.  A second pass over the blocks rather than a returning atomic per point in
// k_count (the first point of a block marking it): 4M-point binning 0.256 ms without
// super-blocks, 0.275 ms with the returning atomic, 0.261 ms with this pass.
__global__ void __launch_bounds__(256) k_mark_sblocks(BinArgs a)
{
    if (skip(a.cond)) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.total_blocks; k += gridDim.x * blockDim.x) {
        // the set whose entries hold k (sets are laid out in order)
        int lo = 0, hi = a.num_sets - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.sets[mid].block_base <= k) lo = mid;
            else hi = mid - 1;
        }
        const SetDesc &S = a.sets[lo];
        const int lb = k - S.block_base;
        if (lb >= S.bxsize * S.bysize || a.bcount[k] == 0) continue;   // a super-block, or empty
        const int by = lb / S.bxsize, bx = lb - by * S.bxsize;
        constexpr int R = SBLOCK_SHIFT - BLOCK_SHIFT;
        atomicAdd(&a.bcount[S.sblock_base + (by >> R) * S.sbxsize + (bx >> R)], 1);
    }
}

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// block-wide exclusive scan of per-thread values; returns the block total in *total
__device__ __forceinline__ int block_exclusive(int v, int *wsum, int *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (blockDim.x >> 5) ? wsum[lane] : 0;
        int wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        wsum[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    int r = wsum[warp] + incl - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const int *in, int n, int *bsum, const int *cond)
{
    if (skip(cond)) return;
    __shared__ int wsum[32];
    __shared__ int total;
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) s += (base + k < n) ? in[base + k] : 0;
    block_exclusive(s, wsum, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// single block: exclusive scan of the block sums in place
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_top(int *bsum, int nb, const int *cond)
{
    if (skip(cond)) return;
    __shared__ int wsum[32];
    __shared__ int total;
    int carry = 0;
    for (int start = 0; start < nb; start += SCAN_TILE) {
        int base = start + threadIdx.x * SCAN_ITEMS;
        int v[SCAN_ITEMS];
        int s = 0;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            v[k] = (base + k < nb) ? bsum[base + k] : 0;
            s += v[k];
        }
        int ex = block_exclusive(s, wsum, &total) + carry;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            if (base + k < nb) bsum[base + k] = ex;
            ex += v[k];
        }
        carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const int *in, int n, const int *bsum, int *out,
                                                             const int *cond)
{
    if (skip(cond)) return;
    __shared__ int wsum[32];
    __shared__ int total;
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int ex = block_exclusive(s, wsum, &total) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
}

__global__ void __launch_bounds__(256) k_scatter(BinArgs a)
{
    if (skip(a.cond)) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        int slot = a.cstart[a.cell_of[i]] + a.rank[i];
        a.sidx[slot] = i;
        if (!a.deterministic) {
            a.spos[slot] = a.pos[i];
            a.slot_of[i] = slot;
        }
    }
}

// per cell: order its points by index (insertion sort of the indices; cells hold a handful
// of points), then the cell-order positions, written once and contiguously per cell
__global__ void __launch_bounds__(256) k_cell_order(BinArgs a)
{
    if (skip(a.cond)) return;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < a.total_cells; c += gridDim.x * blockDim.x) {
        int lo = a.cstart[c], hi = a.cstart[c + 1];
        for (int k = lo + 1; k < hi; ++k) {
            int id = a.sidx[k];
            int j = k - 1;
            while (j >= lo && a.sidx[j] > id) {
                a.sidx[j + 1] = a.sidx[j];
                --j;
            }
            a.sidx[j + 1] = id;
        }
        for (int k = lo; k < hi; ++k) {
            const int id = a.sidx[k];
            a.slot_of[id] = k;
            a.spos[k] = a.pos[id];
        }
    }
}

// current positions into cell order; largest distance outside the listing cell (index order:
// the reads are contiguous, only the cell-order write scatters)
__global__ void __launch_bounds__(256) k_refresh(BinArgs a, DevStatus *st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float mv = 0.0f;
    if (i < a.n) {
        const SetDesc &S = a.sets[a.set_of ? a.set_of[i] : 0];
        double2 p = a.pos[i];
        if (bad_input(S, p)) {
            atomicOr(&st->err_flags, EF_BAD_INPUT);
            p = make_double2(0.0, 0.0);
        }
        a.spos[a.slot_of[i]] = p;
        mv = S.general ? outside_cell<true>(S, a.cell_of[i], p) : outside_cell<false>(S, a.cell_of[i], p);
    }
    for (int o = 16; o > 0; o >>= 1) mv = fmaxf(mv, __shfl_down_sync(0xffffffffu, mv, o));
    if ((threadIdx.x & 31) == 0 && mv > 0.0f) atomicMax(reinterpret_cast<int *>(&st->skin_measured), __float_as_int(mv));
}

// non-negative floats order like their bit patterns, hence the integer atomicMax above
__global__ void k_rebin_decide(DevStatus *st, float max_skin)
{
    const float mv = st->skin_measured;
    const int rebin = !(mv <= max_skin);
    st->rebin = rebin;
    st->skin = rebin ? 0.0f : mv;
}

static cudaError_t launch_scan_c(const int *in, int n, int *bsum, int *out, const int *cond, cudaStream_t s)
{
    int nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_reduce<<<nb, SCAN_THREADS, 0, s>>>(in, n, bsum, cond);
    k_scan_top<<<1, SCAN_THREADS, 0, s>>>(bsum, nb, cond);
    k_scan_apply<<<nb, SCAN_THREADS, 0, s>>>(in, n, bsum, out, cond);
    return cudaGetLastError();
}

cudaError_t launch_scan(const int *in, int n, int *bsum, int *out, cudaStream_t s)
{
    return launch_scan_c(in, n, bsum, out, nullptr, s);
}

int scan_block_count(int n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

// One thread per item; a binning that may be skipped on the device (a.cond) runs a capped,
// grid-stride grid instead, so a skipped launch costs a few microseconds, not one block per
// 256 items
static int bin_grid(int items, const int *cond)
{
    const int full = (items + 255) / 256;
    return cond ? (full < 1024 ? full : 1024) : full;
}

// BinArgs.ccount must hold total_cells + 1 zeros when this is called (the API clears it)
cudaError_t launch_bin_st(const BinArgs &a, DevStatus *st, cudaStream_t s)
{
    if (a.n > 0) k_count<<<bin_grid(a.n, a.cond), 256, 0, s>>>(a, st);
    if (a.n > 0 && a.total_blocks > 0) k_mark_sblocks<<<bin_grid(a.total_blocks, a.cond), 256, 0, s>>>(a);
    cudaError_t e = launch_scan_c(a.ccount, a.total_cells + 1, a.block_sums, a.cstart, a.cond, s);
    if (e != cudaSuccess) return e;
    if (a.n > 0) k_scatter<<<bin_grid(a.n, a.cond), 256, 0, s>>>(a);
    if (a.deterministic && a.total_cells > 0) k_cell_order<<<bin_grid(a.total_cells, a.cond), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_refresh(const BinArgs &a, DevStatus *st, float max_skin, cudaStream_t s)
{
    if (a.n > 0) k_refresh<<<(a.n + 255) / 256, 256, 0, s>>>(a, st);
    k_rebin_decide<<<1, 1, 0, s>>>(st, max_skin);
    return cudaGetLastError();
}

cudaError_t launch_rebin_decide(DevStatus *st, float max_skin, cudaStream_t s)
{
    k_rebin_decide<<<1, 1, 0, s>>>(st, max_skin);
    return cudaGetLastError();
}

cudaError_t launch_clear_counts(int *ccount, int ncell, int *bcount, int nblock, const int *cond, cudaStream_t s)
{
    const int m = ncell > nblock ? ncell : nblock;
    int blocks = (m + 255) / 256;
    if (blocks > (cond ? 1024 : 4096)) blocks = cond ? 1024 : 4096;
    if (blocks < 1) blocks = 1;
    k_clear_counts<<<blocks, 256, 0, s>>>(ccount, ncell, bcount, nblock, cond);
    return cudaGetLastError();
}

// ----------------------------------------------------------------- MD displacement helper
// x += sigma * N(0,1) per axis, wrapped into the primary cell.  Normals by Box-Muller from a
// SplitMix64 hash of (seed, step, point); deterministic for given arguments.
__device__ __forceinline__ unsigned long long smix(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double wrap_coord(double x, double L)
{
    if (x >= L) x -= L;
    else if (x < 0.0) x += L;
    if (!(x < L)) x = 0.0;   // x + L rounded up to L
    if (x < 0.0) x = 0.0;
    return x;
}

// cell_of (MD steps of a context that holds a binning): the cell that lists each point; the
// kernel then also measures how far the moved point lies outside that cell (the margin the
// repair's certification needs while it keeps the cell lists, outside_cell) into
// st->skin_measured, so the repair's local test does not have to
__global__ void __launch_bounds__(256) k_displace(double2 *pos, int n, const SetDesc *sets, const int *set_of,
                                                  double sigma, unsigned long long seed, unsigned long long step,
                                                  const unsigned long long *step_ptr, const int *cell_of,
                                                  DevStatus *st)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float mv = 0.0f;
    if (i < n) {
        if (step_ptr) step = *step_ptr;
        const SetDesc &S = sets[set_of ? set_of[i] : 0];
        unsigned long long h = smix(seed ^ smix(step * 0x100000001B3ULL + (unsigned long long)i));
        unsigned long long h2 = smix(h);
        double u1 = ((h >> 11) + 1) * (1.0 / 9007199254740993.0);   // (0, 1]
        double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
        double r = sigma * sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        double2 p = pos[i];
        if (S.general) {
            // periodicBoundaries::move (periodicBoundaries.h:181-189): displace, then back into
            // the unit cell through fractional coordinates
            p.x += r * cs;
            p.y += r * sn;
            double u = S.i11 * p.x + S.i12 * p.y, v = S.i21 * p.x + S.i22 * p.y;
            u -= floor(u);
            v -= floor(v);
            if (!(u < 1.0)) u = 0.0;
            if (!(v < 1.0)) v = 0.0;
            p = make_double2(S.m11 * u + S.m12 * v, S.m21 * u + S.m22 * v);
        } else {
            p.x = wrap_coord(p.x + r * cs, S.Lx);
            p.y = wrap_coord(p.y + r * sn, S.Ly);
    }
    pos[i] = p;
    if (cell_of) mv = S.general ? outside_cell<true>(S, cell_of[i], p) : outside_cell<false>(S, cell_of[i], p);
    }
    if (cell_of) {
        for (int o = 16; o > 0; o >>= 1) mv = fmaxf(mv, __shfl_down_sync(0xffffffffu, mv, o));
        if ((threadIdx.x & 31) == 0 && mv > 0.0f)
            atomicMax(reinterpret_cast<int *>(&st->skin_measured), __float_as_int(mv));
    }
}

__global__ void k_advance_step(unsigned long long *step_ptr) { *step_ptr += 1; }

cudaError_t launch_displace(double2 *pos, int n, const SetDesc *sets, const int *set_of, double sigma,
                            unsigned long long seed, unsigned long long step, unsigned long long *step_ptr,
                            cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_displace<<<(n + 255) / 256, 256, 0, s>>>(pos, n, sets, set_of, sigma, seed, step, step_ptr, nullptr, nullptr);
    if (step_ptr) k_advance_step<<<1, 1, 0, s>>>(step_ptr);
    return cudaGetLastError();
}

cudaError_t launch_displace_md(double2 *pos, int n, const SetDesc *sets, const int *set_of, double sigma,
                               unsigned long long seed, unsigned long long *step_ptr, const int *cell_of,
                               DevStatus *st, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_displace<<<(n + 255) / 256, 256, 0, s>>>(pos, n, sets, set_of, sigma, seed, 0ull, step_ptr, cell_of, st);
    return cudaGetLastError();
}

}  // namespace dgt

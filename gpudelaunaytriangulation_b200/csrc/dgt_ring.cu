// One-ring construction, repair and the local Delaunay test.
//
// Per point p (one thread per point, points taken in cell order so a warp works on a compact
// patch of cells and shares candidate cells through L1):
//   1. start from a square of four virtual corners (+-V, +-V) (the reference's virtual
//      polygon, DelaunayGPU.cu:340-351, with V a power of two >= the box so the initial cell
//      covers every minimum-image offset);
//   2. insert candidates from p's own cell, then its 3x3 block: a candidate d conflicts with
//      ring edge (P_k, P_k+1) iff it lies strictly inside the circle through (0, P_k, P_k+1)
//      (the Voronoi vertex of that edge is on d's side of the bisector, the reference's test
//      at DelaunayGPU.cu:767-791); the conflicting edges form one arc, whose inner vertices
//      are replaced by d (DelaunayGPU.cu:795-926 does the same bookkeeping vertex by vertex);
//   3. certify: every edge circle must lie inside the scanned rectangle of cells; grow the
//      rectangle one cell per side towards the union of the circles' bounding boxes and
//      scan the new cells until it does (the reference scans a square spiral around each
//      Voronoi vertex instead, DelaunayGPU.cu:715-749);
//   4. write the ring rotated to start at its smallest index (a canonical start; the
//      reference's start depends on insertion order) into row p of the caller's array.
// The ring lives in shared memory (per-thread columns, conflict-free).  Points whose ring
// outgrows that capacity, that meet a predicate neither float32 nor float64 can decide, or
// whose scan outgrows a work budget are rebuilt by a warp each (float64 + exact arithmetic,
// 64-entry ring; k_build_warp).
#include "dgt_builder.cuh"

namespace dgt {
// hot kernel: shared-memory ring of CAP entries per thread; IDX: candidate and own positions
// through the index (repair rounds), else from the cell-order copy (global build); GEN:
// general periodic box
template <typename T, int CAP, int BLOCK, bool IDX, bool GEN = false>
__global__ void __launch_bounds__(BLOCK) k_build(RingArgs A)
{
    typedef typename Prec<T>::T4 E4;
    typedef typename Prec<T>::T2 V2;
    __shared__ E4 se[CAP][BLOCK];
    __shared__ V2 sv[CAP][BLOCK];
    __shared__ int si[CAP][BLOCK];
    __shared__ int swork[BLOCK];
    __shared__ unsigned srare[5][BLOCK];
    SmemRing<T, CAP, BLOCK> ring{ se, sv, si, swork, (int)threadIdx.x };
    for (int k = 0; k < 5; ++k) srare[k][threadIdx.x] = 0;
    SmemCtr<BLOCK> ctr{ 0, 0, srare };
    unsigned pts = 0;
    int maxr = 0;
    const int n = item_count(A);
    if (A.worklist && n <= A.warp_items) return;   // a short work list: k_build_warp takes it
    if (A.repair && blockIdx.x == 0 && threadIdx.x == 0 && n > 0) {
        atomicAdd(&A.st->repaired, (unsigned long long)n);
        atomicMax(&A.st->rounds, A.round + 1);
    }
    for (int base = blockIdx.x * BLOCK; base < n; base += gridDim.x * BLOCK) {
        // every lane runs the builder (it votes across the warp); lanes past the end idle
        int t = base + threadIdx.x;
        const bool act = t < n;
        int pid = -1, slot = -1;
        if (act) {
            if (A.worklist) {
                pid = A.worklist[t];
                slot = A.slot_of[pid];
            } else {
                slot = A.item_base + t;
                pid = __ldg(&A.sidx[slot]);
            }
        }
        const int si = (act && A.set_of) ? __ldg(&A.set_of[slot]) : 0;
        const SetDesc S = A.sets[si];
        double2 p = !act ? make_double2(0.0, 0.0) : (IDX ? __ldg(&A.pos[pid]) : __ldg(&A.spos[slot]));
        Builder<T, false, SmemRing<T, CAP, BLOCK>, SmemCtr<BLOCK>, IDX ? 1 : 0, GEN> b(A, S, ring, ctr, p, slot,
                                                                                    A.sets + si);
        int r = b.run(act);
        if (act) {
            pts++;
            if (r == R_OK) {
                finish(A, pid, ring, b.m, maxr);
            } else if (r == R_CAPACITY || r == R_EXACT || r == R_HEAVY) {
                // over-budget points go in complemented (counted by the warp kernel)
                A.defer_list[atomicAdd(A.defer_count, 1)] = r == R_HEAVY ? ~pid : pid;
            } else {
                atomicOr(&A.st->err_flags, r == R_UNBOUNDED ? EF_UNBOUNDED : EF_NONCONTIG);
                A.nn[pid] = 0;
            }
        }
    }
    flush_counters(A, ctr.total(), pts, maxr);
}

// ------------------------------------------------------------ deferred points: a warp per point
// Points the per-thread kernel hands on -- rings longer than its capacity, predicates neither
// float32 nor float64 decides, and scans longer than the work budget (typically on the rim of
// dense clusters, where the circles reach over large, partly empty and partly dense regions)
// -- are rebuilt by a whole warp.  The 32 lanes share one ring in shared memory (float32
// filter, float64 recheck, exact residue, 64 entries), take 32 new cells at a time (dropping
// cells that no current circle reaches; wide strips are first judged as tiles of 8 x 8 and
// 64 x 64 cells against the two occupancy levels) and 32 candidates at a time.  One lane
// inserts; lanes whose candidates conflicted test them again against the new ring (a
// candidate outside every circle stays outside, see cell_reached).  The scanned rectangle
// grows one cell per side while the ring keeps changing, by half its extent while virtual
// corners are left, and straight to the circles' cells once a layer changed nothing.
constexpr int WARP_KERNEL_CAP = 64;
constexpr int WARP_KERNEL_WARPS = 4;   // warps (points) per block

// New extent [g0,g1] of one axis: towards the needed [lo,hi] by at most `step` per side,
// never wider than the grid (a full-width extent covers every cell of the axis once)
__device__ __forceinline__ void grow_axis(int a0, int a1, int lo, int hi, int step, int size, int &g0, int &g1)
{
    g0 = a0;
    g1 = a1;
    int room = size - (a1 - a0 + 1);
    if (room <= 0) return;
    int want_lo = lo < a0 ? min(a0 - lo, step) : 0;
    int want_hi = hi > a1 ? min(hi - a1, step) : 0;
    if (want_lo + want_hi > room) {
        int l = min(want_lo, room - min(want_hi, room / 2));
        want_hi = min(want_hi, room - l);
        want_lo = l;
    }
    g0 = a0 - want_lo;
    g1 = a1 + want_hi;
}

// j-th index of [0, len) in the order c, c + 1, c - 1, c + 2, c - 2, ... (the longer side
// continues alone once the shorter one is used up)
__device__ __forceinline__ int around(int j, int c, int len)
{
    const int lo = c, hi = len - 1 - c, m = min(lo, hi);
    if (j <= 2 * m) return (j & 1) ? c + (j + 1) / 2 : c - j / 2;
    const int off = j - m;
    return hi > lo ? c + off : c - off;
}

// Tile ti of the strip [xa, xb] x [ya, yb] (cells relative to the own cell) cut into tiles of
// 2^sh x 2^sh cells, nearest first: the strip's tile columns (left / right strip, q = 0 / 1)
// or rows (bottom / top strip, q = 2 / 3) from the old rectangle outwards, and along each of
// them from the tile level with the own cell outwards in both directions
__device__ __forceinline__ void strip_tile(int ti, int q, int xa, int xb, int ya, int yb, int sh, int &ta, int &tb,
                                           int &tc, int &td)
{
    const int tw = ((xb - xa) >> sh) + 1, th = ((yb - ya) >> sh) + 1;
    int ix, iy;
    if (q < 2) {
        const int o = ti / th, c = min(max((0 - ya) >> sh, 0), th - 1);
        ix = q == 0 ? tw - 1 - o : o;
        iy = around(ti - o * th, c, th);
    } else {
        const int o = ti / tw, c = min(max((0 - xa) >> sh, 0), tw - 1);
        iy = q == 2 ? th - 1 - o : o;
        ix = around(ti - o * tw, c, tw);
    }
    ta = xa + (ix << sh);
    tb = min(ta + (1 << sh) - 1, xb);
    tc = ya + (iy << sh);
    td = min(tc + (1 << sh) - 1, yb);
}

// Whether any occupancy entry of 2^sh x 2^sh cells (row-major from `base`, `row` per row)
// that the cells [xa, xb] x [ya, yb] relative to (ocx, ocy), wrapped, touch holds points.  A
// span of at most 2^sh cells touches at most three entries per axis (two, plus the grid's
// partial last entry where it wraps); the loads are independent of each other.
__device__ __forceinline__ bool occupied(const int *cnt, int base, int row, int sh, const SetDesc &S, int ocx, int ocy,
                                         int xa, int xb, int ya, int yb)
{
    int ex[3], ey[3], nx = 0, ny = 0, xs = xa, ys = ya;
    for (; xs <= xb && nx < 3; ++nx) {
        const int ax = wrapi(ocx + xs, S.xsize);
        ex[nx] = ax >> sh;
        xs += min((ex[nx] + 1) << sh, S.xsize) - ax;
    }
    for (; ys <= yb && ny < 3; ++ny) {
        const int ay = wrapi(ocy + ys, S.ysize);
        ey[ny] = ay >> sh;
        ys += min((ey[ny] + 1) << sh, S.ysize) - ay;
    }
    if (xs <= xb || ys <= yb) return true;   // wider than 2^sh cells: judged occupied
    int acc = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < nx && j < ny) acc |= __ldg(&cnt[base + ey[j] * row + ex[i]]);
    return acc != 0;
}

template <class B>
__device__ int coop_run(B &b, const int lane)
{
    typedef typename B::Mask Mask;
    typedef typename B::V2 V2;
    const RingArgs &A = b.A;
    const SetDesc &S = b.S;
    if (lane == 0) b.init_ring();
    __syncwarp();
    b.init_local();
    const double2 fp = cell_pos<B::general>(S, b.p);
    const double fx = fp.x - (double)b.ocx, fy = fp.y - (double)b.ocy;
    int x0 = 0, x1 = 0, y0 = 0, y1 = 0;
    bool changed = true;
    int status = R_OK, nins = 0;
    const int max_phase = S.xsize + S.ysize + 8;

    // one candidate per lane (have): classify all, then insert the conflicting ones one at a
    // time, nearest first (a near candidate is the likelier Delaunay neighbour, and inserting
    // it shrinks the circles the farther ones conflict with); after each insertion the others
    // keep their decisions for the surviving edges and test only the two new ones
    auto settle = [&](int sl, bool have) {
        V2 d = B::PR::mk2(0, 0);
        double2 d64 = make_double2(0.0, 0.0);
        Mask mask = 0;
        if (have) b.classify(sl, d, mask, d64);
        unsigned want = __ballot_sync(0xffffffffu, have && mask != 0);
        while (want) {
            const float nd = (float)(d.x * d.x + d.y * d.y);
            unsigned key = ((want >> lane) & 1u) ? ((__float_as_uint(nd) & ~31u) | (unsigned)lane) : 0xffffffffu;
            for (int o = 16; o > 0; o >>= 1) key = min(key, __shfl_xor_sync(0xffffffffu, key, o));
            const int leader = (int)(key & 31u);
            const int m_old = b.m;
            const Mask lmask = __shfl_sync(0xffffffffu, mask, leader);
            int ir = R_OK;
            if (lane == leader) ir = b.insert(d, __ldg(&A.sidx[sl]), mask);
            ir = __shfl_sync(0xffffffffu, ir, leader);
            b.m = __shfl_sync(0xffffffffu, b.m, leader);
            b.r2max = __shfl_sync(0xffffffffu, b.r2max, leader);
            __syncwarp();
            if (ir != R_OK) {
                status = ir;
                break;
            }
            changed = true;
            ++nins;
            const bool again = ((want >> lane) & 1u) && lane != leader;
            if (again) {
                int s, e, c, ns;
                B::conflict_arc(lmask, m_old, s, e, c);
                mask = B::remap_mask(mask, s, e, ns);
                const int i0 = b.test_edge(ns, d, d64), i1 = b.test_edge(ns + 1, d, d64);
                mask |= (Mask)(i0 > 0) << ns;
                mask |= (Mask)(i1 > 0) << (ns + 1);
            } else {
                mask = 0;
            }
            want = __ballot_sync(0xffffffffu, again && mask != 0);
        }
    };
    // every candidate of the cells [xa, xb] x [ya, yb] (relative to the own cell): 32 cells
    // at a time, one per lane (with `prune`, the cells no current circle reaches are dropped),
    // then their candidates 32 at a time
    auto scan_cells = [&](int xa, int xb, int ya, int yb, bool prune) {
        const int w = xb - xa + 1, ncell = w * (yb - ya + 1);
        for (int cb = 0; cb < ncell && status == R_OK; cb += 32) {
            const int ci = cb + lane;
            int start = 0, cnt = 0, rx = 0, ry = 0;
            if (ci < ncell) {
                rx = xa + ci % w;
                ry = ya + ci / w;
                const int cx = wrapi(b.ocx + rx, S.xsize), cy = wrapi(b.ocy + ry, S.ysize);
                const int c = S.cell_base + cy * S.xsize + cx;
                start = __ldg(&A.cstart[c]);
                cnt = __ldg(&A.cstart[c + 1]) - start;
                if (cnt > 0 && prune && !b.cell_reached(rx, ry, fx, fy)) cnt = 0;
                if (cnt > 0) b.ctr.add_cells();
            }
            // the cells' candidates 32 at a time; after a chunk that changed the ring, the
            // cells with candidates left are tested against the shrunken circles again
            while (status == R_OK) {
                int incl = cnt;
                for (int o = 1; o < 32; o <<= 1) {
                    int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31), excl = incl - cnt;
                if (total == 0) break;
                int o = 0;   // the last lane whose cell range starts at or before this lane's slot
                for (int step = 16; step > 0; step >>= 1) {
                    int e = __shfl_sync(0xffffffffu, excl, o + step);
                    if (e <= lane) o += step;
                }
                const int sl = __shfl_sync(0xffffffffu, start, o) + lane - __shfl_sync(0xffffffffu, excl, o);
                const int m_before = nins;
                settle(sl, lane < total);
                const int used = min(cnt, max(0, 32 - excl));
                start += used;
                cnt -= used;
                if (prune && nins != m_before && cnt > 0 && !b.cell_reached(rx, ry, fx, fy)) cnt = 0;
            }
        }
    };

    for (int phase = 0; status == R_OK && phase < max_phase; ++phase) {
        int nx0 = x0, nx1 = x1, ny0 = y0, ny1 = y1;
        if (phase >= 1) {
            bool real = true;
            for (int k = 0; k < b.m; ++k) real &= b.R.idx(k) >= 0;
            int lx, hx, ly, hy;
            if (!b.need_rect(fx, fy, lx, hx, ly, hy)) {
                lx = ly = -(1 << 28);
                hx = hy = 1 << 28;
            }
            // one cell per side while the last phase changed the ring; else the extent doubles
            // (all-real ring) or grows by half (virtual corners left), so each phase
            // re-derives the rectangle from circles that nearer cells have already shrunk
            const int sx = changed ? 1 : (real ? max(1, x1 - x0 + 1) : max(1, (x1 - x0 + 1) >> 1));
            const int sy = changed ? 1 : (real ? max(1, y1 - y0 + 1) : max(1, (y1 - y0 + 1) >> 1));
            grow_axis(x0, x1, lx, hx, sx, S.xsize, nx0, nx1);
            grow_axis(y0, y1, ly, hy, sy, S.ysize, ny0, ny1);
            if (nx0 == x0 && nx1 == x1 && ny0 == y0 && ny1 == y1) break;
        }
        changed = false;
        // new cells: up to four strips (columns left and right of the old rectangle over its
        // rows, then rows below and above over the new columns); phase 0 is the own cell
        int sxa[4], sxb[4], sya[4], syb[4];
        if (phase == 0) {
            sxa[0] = sxb[0] = sya[0] = syb[0] = 0;
            for (int q = 1; q < 4; ++q) sxa[q] = 1, sxb[q] = 0, sya[q] = 1, syb[q] = 0;
        } else {
            sxa[0] = nx0; sxb[0] = x0 - 1; sya[0] = y0; syb[0] = y1;
            sxa[1] = x1 + 1; sxb[1] = nx1; sya[1] = y0; syb[1] = y1;
            sxa[2] = nx0; sxb[2] = nx1; sya[2] = ny0; syb[2] = y0 - 1;
            sxa[3] = nx0; sxb[3] = nx1; sya[3] = y1 + 1; syb[3] = ny1;
        }
        for (int q = 0; q < 4 && status == R_OK; ++q) {
            const int sw = sxb[q] - sxa[q] + 1, sh = syb[q] - sya[q] + 1;
            if (sw <= 0 || sh <= 0) continue;
            // a small strip (and the first two phases): its cells directly.  A large strip:
            // tiles first, one per lane, nearest first; a tile is opened only when an occupancy
            // block it touches holds points and its rectangle meets a current circle (empty
            // space costs one test per tile, not per cell).  A strip of more than 64 tiles of
            // 8 x 8 cells is cut into 64 x 64-cell tiles first, judged by the super-block
            // occupancy, and only those are opened into 8 x 8-cell tiles.  One loop with one
            // call of scan_cells: the candidate code is large and shared by few warps, and a
            // single copy of it stays in the instruction cache.
            const bool direct = phase < 2 || sw * sh <= 512;
            const bool super = !direct && (((sw - 1) >> BLOCK_SHIFT) + 1) * (((sh - 1) >> BLOCK_SHIFT) + 1) > 64;
            bool cells = direct;   // the rectangle [ca, cb] x [cc, cd] is to be scanned
            int ca = sxa[q], cb = sxb[q], cc = sya[q], cd = syb[q];
            bool prune = phase >= 2;
            // 8 x 8-cell tiles over [ra, rb] x [rc, rd]: batch t1 of n1, live ones in todo1
            int ra = sxa[q], rb = sxb[q], rc = sya[q], rd = syb[q];
            int t1 = 0, n1 = (direct || super) ? 0 : (((sw - 1) >> BLOCK_SHIFT) + 1) * (((sh - 1) >> BLOCK_SHIFT) + 1);
            unsigned todo1 = 0;
            int ta1 = 0, tb1 = -1, tc1 = 0, td1 = -1;
            // 64 x 64-cell tiles over the strip
            int t2 = 0, n2 = super ? (((sw - 1) >> SBLOCK_SHIFT) + 1) * (((sh - 1) >> SBLOCK_SHIFT) + 1) : 0;
            unsigned todo2 = 0;
            int ta2 = 0, tb2 = -1, tc2 = 0, td2 = -1;
            while (status == R_OK) {
                if (cells) {
                    cells = false;
                    scan_cells(ca, cb, cc, cd, prune);
                    continue;
                }
                if (todo1) {
                    const int src = __ffs(todo1) - 1;
                    todo1 &= todo1 - 1;
                    ca = __shfl_sync(0xffffffffu, ta1, src);
                    cb = __shfl_sync(0xffffffffu, tb1, src);
                    cc = __shfl_sync(0xffffffffu, tc1, src);
                    cd = __shfl_sync(0xffffffffu, td1, src);
                    prune = true;
                    cells = true;
                    continue;
                }
                if (t1 < n1) {
                    const int ti = t1 + lane;
                    bool live = false;
                    ta1 = 0, tb1 = -1, tc1 = 0, td1 = -1;
                    if (ti < n1) {
                        strip_tile(ti, q, ra, rb, rc, rd, BLOCK_SHIFT, ta1, tb1, tc1, td1);
                        live = occupied(A.bcount, S.block_base, S.bxsize, BLOCK_SHIFT, S, b.ocx, b.ocy, ta1, tb1, tc1,
                                        td1) &&
                               b.rect_reached(ta1, tb1, tc1, td1, fx, fy);
                    }
                    todo1 = __ballot_sync(0xffffffffu, live);
                    t1 += 32;
                    continue;
                }
                if (todo2) {
                    const int src = __ffs(todo2) - 1;
                    todo2 &= todo2 - 1;
                    ra = __shfl_sync(0xffffffffu, ta2, src);
                    rb = __shfl_sync(0xffffffffu, tb2, src);
                    rc = __shfl_sync(0xffffffffu, tc2, src);
                    rd = __shfl_sync(0xffffffffu, td2, src);
                    t1 = 0;
                    n1 = (((rb - ra) >> BLOCK_SHIFT) + 1) * (((rd - rc) >> BLOCK_SHIFT) + 1);
                    continue;
                }
                if (t2 < n2) {
                    const int ti = t2 + lane;
                    bool live = false;
                    ta2 = 0, tb2 = -1, tc2 = 0, td2 = -1;
                    if (ti < n2) {
                        strip_tile(ti, q, sxa[q], sxb[q], sya[q], syb[q], SBLOCK_SHIFT, ta2, tb2, tc2, td2);
                        live = occupied(A.bcount, S.sblock_base, S.sbxsize, SBLOCK_SHIFT, S, b.ocx, b.ocy, ta2, tb2,
                                        tc2, td2) &&
                               b.rect_reached(ta2, tb2, tc2, td2, fx, fy);
                    }
                    todo2 = __ballot_sync(0xffffffffu, live);
                    t2 += 32;
                    continue;
                }
                break;
            }
        }
        x0 = nx0;
        x1 = nx1;
        y0 = ny0;
        y1 = ny1;
    }
    if (status != R_OK) return status;
    for (int k = 0; k < b.m; ++k)
        if (b.R.idx(k) < 0) return R_UNBOUNDED;
    if (b.minimage && lane == 0) atomicOr(&A.st->err_flags, EF_MINIMAGE);
    return R_OK;
}

template <bool GEN>
// two blocks per SM: no register spills (a fourth of the ring state spilled at four blocks;
// measured: clustered 1M build -1.5%); the grid is sized to one wave of that residency
__global__ void __launch_bounds__(WARP_KERNEL_WARPS * 32, 2) k_build_warp(RingArgs A)
{
    __shared__ float4 se[WARP_KERNEL_CAP][WARP_KERNEL_WARPS];
    __shared__ float2 sv[WARP_KERNEL_CAP][WARP_KERNEL_WARPS];
    __shared__ int si[WARP_KERNEL_CAP][WARP_KERNEL_WARPS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    SmemRing<float, WARP_KERNEL_CAP, WARP_KERNEL_WARPS> ring{ se, sv, si, nullptr, wib };
    Ctr ctr = { 0, 0, 0, 0, 0, 0, 0 };
    unsigned pts = 0, heavy = 0;
    int maxr = 0;
    // a short work list is rebuilt here directly (a warp per point has a far shorter latency
    // than one thread per point, and few points cannot hide it); otherwise the deferred points
    const bool direct = A.worklist && item_count(A) <= A.warp_items;
    const int n = direct ? item_count(A) : min(*A.defer_count, A.npoints);
    const int *list = direct ? A.worklist : A.defer_list;
    if (direct && A.repair && blockIdx.x == 0 && threadIdx.x == 0 && n > 0) {
        atomicAdd(&A.st->repaired, (unsigned long long)n);
        atomicMax(&A.st->rounds, A.round + 1);
    }
    for (int item = blockIdx.x * WARP_KERNEL_WARPS + wib; item < n; item += gridDim.x * WARP_KERNEL_WARPS) {
        const int e = list[item];
        const int pid = e < 0 ? ~e : e;
        heavy += e < 0;
        const int slot = A.slot_of[pid];
        const int si = A.set_of ? A.set_of[slot] : 0;
        const SetDesc S = A.sets[si];
        const double2 p = A.cand_by_index ? A.pos[pid] : A.spos[slot];
        Builder<float, true, SmemRing<float, WARP_KERNEL_CAP, WARP_KERNEL_WARPS>, Ctr, 2, GEN> b(A, S, ring, ctr, p,
                                                                                              slot, A.sets + si);
        const int r = coop_run(b, lane);
        if (lane == 0) {
            pts++;
            if (r == R_OK) {
                finish(A, pid, ring, b.m, maxr);
            } else {
                atomicOr(&A.st->err_flags, r == R_CAPACITY ? EF_SLOW_OVERFLOW
                                          : r == R_UNBOUNDED ? EF_UNBOUNDED : EF_NONCONTIG);
                A.nn[pid] = 0;
            }
        }
        __syncwarp();
    }
    if (lane == 0 && pts) atomicAdd(&A.st->exact_points, (unsigned long long)pts);
    if (lane == 0 && heavy) atomicAdd(&A.st->heavy_points, (unsigned long long)heavy);
    flush_counters(A, ctr, 0, maxr);
}



// ------------------------------------------------------------------ local Delaunay test
// Flags every point whose fan is not certainly a piece of the Delaunay triangulation:
// a fan triangle that is not strictly CCW, a fan that does not wind exactly once, or a
// spoke (p, P_k) whose opposite vertex P_k+1 is not certainly outside the circle through
// (p, P_k-1, P_k).  The four vertices of a failing spoke's quadrilateral are queued (an
// edge flip changes all four rings).  Undecided filters count as failures.
__device__ __forceinline__ void warp_append(int *list, int *count, const int *items, int k)
{
    const int lane = threadIdx.x & 31;
    int incl = k;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    int total = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(count, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    int off = base + incl - k;
    for (int i = 0; i < k; ++i) list[off + i] = items[i];
}

constexpr int TEST_MAX_QUEUE = 24;
constexpr int TEST_MAX_EDGES = 6;

__device__ __forceinline__ void warp_append_edges(int2 *list, int *count, int cap, const int2 *items, int k,
                                                  int *overflow)
{
    const int lane = threadIdx.x & 31;
    int incl = k;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    int total = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(count, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    int off = base + incl - k;
    *overflow = 0;
    for (int i = 0; i < k; ++i) {
        if (off + i < cap) list[off + i] = items[i];
        else *overflow = 1;
    }
}

// One spoke (p, P_k) of a fan: triangle (p, P_k, P_k+1) strictly CCW and P_k+1 outside the
// circle through (p, P_k-1, P_k); counts the winding crossing and records failures
__device__ __forceinline__ void test_spoke(double2 prev, double2 cur, double2 nxt, int k, int rk, int i, bool flip,
                                           int &cross, int &nf, int *fail_k, bool &inverted, int2 *ev, int &ne)
{
    int o = orient32(__double2float_rn(cur.x), __double2float_rn(cur.y), __double2float_rn(nxt.x),
                     __double2float_rn(nxt.y));
    if (o == 0) o = orient64(cur.x, cur.y, nxt.x, nxt.y);
    int ic = incircle32(__double2float_rn(prev.x), __double2float_rn(prev.y), __double2float_rn(cur.x),
                        __double2float_rn(cur.y), __double2float_rn(nxt.x), __double2float_rn(nxt.y));
    if (ic == 0) ic = incircle64(prev.x, prev.y, cur.x, cur.y, nxt.x, nxt.y);
    if (cur.y < 0.0 && nxt.y >= 0.0) cross++;
    if (o <= 0 || ic >= 0) {
        if (nf < 3) fail_k[nf] = k;
        nf++;
    }
    inverted |= o <= 0;
    if (flip && o > 0 && ic >= 0 && i < rk) {
        if (ne < TEST_MAX_EDGES) ev[ne] = make_int2(i, rk);
        ne++;
    }
}

// Flip mode (A.flip_list set): a valid fan (every triangle strictly CCW, winding once) sends
// its illegal or undecided spokes (i, P_k) with i < P_k to the flip list (the flip stage
// decides them exactly); an invalid fan queues its point for rebuilding.
// four blocks per SM (64 registers): more warps in flight hide the neighbour gathers
// (measured: -4% repair time against three blocks at 73 registers)
template <bool GEN>
__global__ void __launch_bounds__(256, 4) k_test(TestArgs A)
{
    unsigned long long flagged = 0;
    const int ebase = *A.epoch_ptr + 1;
    const bool flip = A.flip_list != nullptr;
    float moved = 0.0f;   // largest distance outside the listing cell (when A.rcell_of is set)
    for (int base = blockIdx.x * blockDim.x; base < A.n; base += gridDim.x * blockDim.x) {
        // points taken in cell order (slot t -> point sidx[t]): the queue a warp appends is a
        // compact patch of cells, which keeps the repair rounds spatially coherent
        // flip mode: index order (rows, ring lengths and owner positions stream contiguously;
        // only the neighbour gathers are random)
        const int t = base + threadIdx.x;
        const int i = (t < A.n && A.sidx && !flip) ? A.sidx[t] : t;
        int q[TEST_MAX_QUEUE];
        int nq = 0;
        int2 ev[TEST_MAX_EDGES];
        int ne = 0;
        bool inverted = false;
        if (t < A.n && A.rcell_of) {
            const SetDesc S = A.sets[A.set_of ? A.set_of[i] : 0];
            const double2 p = A.pos[i];
            const bool bad_in = GEN ? !(isfinite(p.x) && isfinite(p.y))
                                    : !(p.x >= 0.0 && p.x < S.Lx && p.y >= 0.0 && p.y < S.Ly);
            if (bad_in) atomicOr(&A.st->err_flags, EF_BAD_INPUT);
            moved = fmaxf(moved, outside_cell<GEN>(S, A.rcell_of[i], p));
        }
        if (t < A.n) {
            int m = A.nn[i];
            bool bad = (m < 3 || m > A.stride);
            const int *row = A.tri + (size_t)i * A.stride;
            int fail_k[3] = { -1, -1, -1 };
            int nf = 0;
            if (!bad) {
                for (int k = 0; k < m; ++k) {
                    int r = row[k];
                    if (r < 0 || r >= A.n || r == i) bad = true;
                }
                if (!bad) {
                const SetDesc S = A.sets[A.set_of ? A.set_of[i] : 0];
                double2 p = (A.sidx && !flip) ? A.spos[t] : A.pos[i];
                double2 q0 = __ldg(&A.pos[row[0]]), ql = __ldg(&A.pos[row[m - 1]]);
                double2 o0 = GEN ? gen_off(q0, p, S)
                                 : make_double2(wrap_off(q0.x, p.x, S.Lx, S.hLx), wrap_off(q0.y, p.y, S.Ly, S.hLy));
                double2 prev = GEN ? gen_off(ql, p, S)
                                   : make_double2(wrap_off(ql.x, p.x, S.Lx, S.hLx), wrap_off(ql.y, p.y, S.Ly, S.hLy));
                double2 cur = o0;
                int cross = 0;
                // neighbour positions gathered two spokes ahead of their use
                double2 qa = __ldg(&A.pos[row[1 < m ? 1 : 0]]), qb = __ldg(&A.pos[row[2 < m ? 2 : 0]]);
                for (int k = 0; k < m; ++k) {
                    const double2 qn = qa;
                    qa = qb;
                    if (k + 3 < m) qb = __ldg(&A.pos[row[k + 3]]);
                    double2 nxt;
                    if (k + 1 < m) {
                        nxt = GEN ? gen_off(qn, p, S)
                                  : make_double2(wrap_off(qn.x, p.x, S.Lx, S.hLx), wrap_off(qn.y, p.y, S.Ly, S.hLy));
                    } else {
                        nxt = o0;
                    }
                    test_spoke(prev, cur, nxt, k, row[k], i, flip, cross, nf, fail_k, inverted, ev, ne);
                    prev = cur;
                    cur = nxt;
                }
                if (cross != 1) bad = true;
                }
            }
            if (flip) {
                // invalid fan (or more illegal spokes than the edge buffer): rebuild the point
                if (bad || inverted || ne > TEST_MAX_EDGES) {
                    if (atomicMax(&A.mark[i], ebase) < ebase) q[nq++] = i;
                    ne = 0;
                }
            } else if (bad || nf > 0) {
                if (atomicMax(&A.mark[i], ebase) < ebase) q[nq++] = i;
                if (!bad) {
                    // a spoke failure: its quadrilateral; more than three failures: the whole fan
                    if (nf <= 3) {
                        for (int f = 0; f < nf; ++f) {
                            int k = fail_k[f];
                            int js[3] = { row[k == 0 ? m - 1 : k - 1], row[k], row[k + 1 == m ? 0 : k + 1] };
                            for (int t = 0; t < 3; ++t)
                                if (nq < TEST_MAX_QUEUE && atomicMax(&A.mark[js[t]], ebase) < ebase)
                                    q[nq++] = js[t];
                        }
                    } else {
                        for (int k = 0; k < m; ++k)
                            if (nq < TEST_MAX_QUEUE && atomicMax(&A.mark[row[k]], ebase) < ebase)
                                q[nq++] = row[k];
                    }
                }
            }
        }
        flagged += nq;
        if (flip) {
            int overflow = 0;
            warp_append_edges(A.flip_list, A.flip_count, A.flip_cap, ev, ne, &overflow);
            if (overflow && atomicMax(&A.mark[i], ebase) < ebase) {
                q[nq++] = i;   // list full: the point's spokes are settled by rebuilding it
                flagged++;
            }
        }
        warp_append(A.list, A.list_count, q, nq);
    }
    for (int o = 16; o > 0; o >>= 1) flagged += __shfl_down_sync(0xffffffffu, flagged, o);
    if ((threadIdx.x & 31) == 0 && flagged) atomicAdd(&A.st->flagged, flagged);
    for (int o = 16; o > 0; o >>= 1) moved = fmaxf(moved, __shfl_down_sync(0xffffffffu, moved, o));
    if ((threadIdx.x & 31) == 0 && moved > 0.0f)
        atomicMax(reinterpret_cast<int *>(&A.st->skin_measured), __float_as_int(moved));
}

// ------------------------------------------------------------------------- launchers
template <typename T, int CAP, int BLOCK, bool GEN = false>
static cudaError_t launch_build_t(const RingArgs &a, int sms, cudaStream_t s)
{
    int blocks;
    if (a.worklist) {
        int want = (a.n_items + BLOCK - 1) / BLOCK;
        blocks = want < sms * 32 ? want : sms * 32;
    } else {
        blocks = (a.n_items + BLOCK - 1) / BLOCK;
    }
    if (blocks < 1) blocks = 1;
    if (a.cand_by_index) k_build<T, CAP, BLOCK, true, GEN><<<blocks, BLOCK, 0, s>>>(a);
    else k_build<T, CAP, BLOCK, false, GEN><<<blocks, BLOCK, 0, s>>>(a);
    return cudaGetLastError();
}

// kernel shapes the autotuner chooses from: (ring capacity on chip, threads per block, lanes
// per point); index 0 is the default.  Shapes 5 and 6: a group of 4 / 8 lanes per point
// (dgt_group.cu)
static const int kShapeCap[KERNEL_SHAPES] = { 14, 12, 16, 14, 12, 14, 14 };
static const int kShapeBlock[KERNEL_SHAPES] = { 64, 64, 64, 32, 32, 64, 64 };
static const int kShapeLanes[KERNEL_SHAPES] = { 1, 1, 1, 1, 1, 4, 8 };

int kernel_shape_cap(int shape) { return (shape >= 0 && shape < KERNEL_SHAPES) ? kShapeCap[shape] : -1; }
int kernel_shape_block(int shape) { return (shape >= 0 && shape < KERNEL_SHAPES) ? kShapeBlock[shape] : -1; }

cudaError_t launch_build(const RingArgs &a, int mode, int sms, int shape, cudaStream_t s)
{
    if (a.n_items <= 0) return cudaSuccess;
    if (shape >= 0 && shape < KERNEL_SHAPES && kShapeLanes[shape] > 1)
        return launch_build_group(a, mode, sms, kShapeLanes[shape], s);
    if (a.general) {
        // general boxes: the default shape only (rings past its capacity go to the warp kernel)
        if (mode == MODE_F64) return launch_build_t<double, 14, 64, true>(a, sms, s);
        return launch_build_t<float, 14, 64, true>(a, sms, s);
    }
    if (mode == MODE_F64) return launch_build_t<double, 14, 64>(a, sms, s);
    switch (shape) {
    case 1: return launch_build_t<float, 12, 64>(a, sms, s);
    case 2: return launch_build_t<float, 16, 64>(a, sms, s);
    case 3: return launch_build_t<float, 14, 32>(a, sms, s);
    case 4: return launch_build_t<float, 12, 32>(a, sms, s);
    default: return launch_build_t<float, 14, 64>(a, sms, s);
    }
}

cudaError_t launch_deferred(const RingArgs &a, int sms, cudaStream_t s)
{
    if (a.general) k_build_warp<true><<<max(sms, 1) * 2, WARP_KERNEL_WARPS * 32, 0, s>>>(a);
    else k_build_warp<false><<<max(sms, 1) * 2, WARP_KERNEL_WARPS * 32, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_test(const TestArgs &a, cudaStream_t s)
{
    if (a.n <= 0) return cudaSuccess;
    int blocks = (a.n + 255) / 256;
    if (a.general) k_test<true><<<blocks, 256, 0, s>>>(a);
    else k_test<false><<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// The points of the first rebuild round take their current ring neighbours along: a rebuilt
// point's old and new neighbours are what the consistency checks would queue for the next
// round, and a round costs about the same for a few points as for a wave of them.  Only a
// list of at most max_items / 8 points is expanded (the result stays within one wave).
__global__ void __launch_bounds__(256) k_expand(int *list, int *count, int cap, const int *tri, const int *nn,
                                                int stride, int n, int *mark, const int *epoch_ptr, int max_items)
{
    const int ebase = *epoch_ptr + 1;
    const int n0 = min(*count, cap);
    if (n0 > max_items / 8) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n0; t += gridDim.x * blockDim.x) {
        const int i = list[t];
        if (i < 0 || i >= n) continue;
        const int m = nn[i];
        if (m < 1 || m > stride) continue;
        const int *row = tri + (size_t)i * stride;
        for (int k = 0; k < m; ++k) {
            const int j = row[k];
            if (j < 0 || j >= n) continue;
            if (atomicMax(&mark[j], ebase) < ebase) {
                const int at = atomicAdd(count, 1);
                if (at < cap) list[at] = j;
            }
        }
    }
}

cudaError_t launch_expand(int *list, int *count, int cap, const int *tri, const int *nn, int stride, int n,
                          int *mark, const int *epoch_ptr, int sms, cudaStream_t s)
{
    // one wave of the per-thread rebuild kernel: 8 blocks of 64 threads per SM
    k_expand<<<max(sms, 1) * 4, 256, 0, s>>>(list, count, cap, tri, nn, stride, n, mark, epoch_ptr,
                                             max(sms, 1) * 8 * 64);
    return cudaGetLastError();
}

__global__ void k_call_end(DevCtl *ctl, DevStatus *st, int rounds, int advance_step)
{
    if (advance_step) ctl->step += 1;
    int f = st->err_flags;
    if (rounds > 0) {
        if (st->list_count[rounds & 1] > 0) {
            f |= EF_NOT_CONVERGED;
            st->err_flags |= EF_NOT_CONVERGED;
        }
        ctl->epoch += rounds + 1;
        ctl->calls += 1;
    }
    ctl->sticky |= f;
}

cudaError_t launch_call_end(DevCtl *ctl, DevStatus *st, int rounds, cudaStream_t s, bool advance_step)
{
    k_call_end<<<1, 1, 0, s>>>(ctl, st, rounds, advance_step ? 1 : 0);
    return cudaGetLastError();
}

__global__ void k_restride(const int *src, int os, int *dst, int ns, const int *nn, int n)
{
    int i = blockIdx.y * gridDim.x + blockIdx.x;
    if (i >= n) return;
    int m = nn ? min(nn[i], min(os, ns)) : min(os, ns);
    for (int k = threadIdx.x; k < ns; k += blockDim.x) dst[(size_t)i * ns + k] = k < m ? src[(size_t)i * os + k] : 0;
}

cudaError_t launch_restride(const int *src, int os, int *dst, int ns, const int *nn, int n, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    dim3 g(n < 65535 ? n : 65535, (n + 65534) / 65535);
    k_restride<<<g, 32, 0, s>>>(src, os, dst, ns, nn, n);
    return cudaGetLastError();
}

}  // namespace dgt

// One-ring construction with a group of G lanes per point (G = 4 or 8: 32 / G points per warp).
//
// The per-point construction is the one of dgt_ring.cu (the reference's localized one-ring:
// virtual corners, insertion of candidates whose bisector cuts the polygon, certification
// by the cells the Voronoi-vertex circles reach; DelaunayGPU.cu:318-608, :680-943), with
// the ring of a point shared by its group in shared memory and the work inside a point
// spread over the group's lanes:
//
//  - cells are taken as row segments (a run of cells of one grid row is one contiguous range
//    of cell-order slots), G segments at a time, one per lane; the phase's candidates are
//    then dealt out G at a time (group prefix sum over the segments' counts, a binary
//    search by shuffles for each lane's segment);
//  - each lane classifies its candidate against every edge circle of the current ring;
//  - while some candidates conflict, the nearest one is inserted (the group replaces the
//    conflict arc together: each lane moves its share of the ring entries, three lanes write
//    the new vertex and the two new edge circles); the other conflicting lanes keep their
//    decisions for the edges that survive (same circles) and test only the two new ones.
//    Candidates that did not conflict stay outside: the union of the circles through p of a
//    star-shaped ring only shrinks under insertion.
//
// Every loop is warp-uniform (lanes of finished groups ride along predicated off), so the
// warp stays converged; the shuffles are width-G shuffles of the full warp.  Output, repair
// bookkeeping and deferral to the warp-per-point kernel are those of the per-thread kernel
// (finish(), run by the group's first lane).
#include "dgt_builder.cuh"

namespace dgt {

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <int G> __device__ __forceinline__ int gshfl(int v, int src) { return __shfl_sync(FULL, v, src, G); }
template <int G> __device__ __forceinline__ unsigned gshfl(unsigned v, int src) { return __shfl_sync(FULL, v, src, G); }
template <int G> __device__ __forceinline__ float gshfl(float v, int src) { return __shfl_sync(FULL, v, src, G); }
template <int G> __device__ __forceinline__ double gshfl(double v, int src) { return __shfl_sync(FULL, v, src, G); }
template <int G> __device__ __forceinline__ unsigned long long gshfl(unsigned long long v, int src)
{
    return __shfl_sync(FULL, v, src, G);
}

// this lane's group's bits of a warp vote (bit i = lane i of the group)
template <int G> __device__ __forceinline__ unsigned gvote(bool p)
{
    const unsigned b = __ballot_sync(FULL, p);
    const int base = (threadIdx.x & 31) & ~(G - 1);
    return (b >> base) & ((1u << G) - 1u);
}

// nearest-first key: the candidate's squared distance (non-negative float: its bit pattern
// orders like the value) with the lane in the low bits
template <int G> __device__ __forceinline__ unsigned near_key(float nd, int glane)
{
    return (__float_as_uint(nd) & ~(unsigned)(G - 1)) | (unsigned)glane;
}

// The group inserts candidate (d, id) whose conflicting edges are `mask` (the same on every
// lane of the group; `go` false: nothing to insert, the lanes only take part in the syncs).
// Returns R_OK / R_NONCONTIG / R_CAPACITY (uniform in the group); s, e: the first and last
// conflicting edge, c their count, ns the new index of the first new edge.
template <int G, class B>
__device__ __forceinline__ int grp_insert(B &b, bool go, int glane, typename B::V2 d, int id,
                                          typename B::Mask mask, int &s, int &e, int &ns)
{
    typedef typename B::V2 V2;
    typedef typename B::E4 E4;
    typedef typename B::Real T;
    constexpr int CAP = B::RingT::cap;
    const int m = b.m;
    int c;
    const bool arc = B::conflict_arc(mask, m, s, e, c);
    int r = R_OK;
    if (go && !arc) r = R_NONCONTIG;
    const int mnew = m - c + 2;
    if (go && r == R_OK && mnew > CAP) r = R_CAPACITY;
    go = go && r == R_OK;
    ns = s <= e ? s : s - e - 1;
    E4 ca, cb;
    if (go) {
        const V2 vs = b.R.vert(s), ve = b.R.vert(e + 1 == m ? 0 : e + 1);
        ca = make_circ<T>(vs.x, vs.y, d.x, d.y);
        cb = make_circ<T>(d.x, d.y, ve.x, ve.y);
    }
    // entries that move: read them all, then write them (the old and new places overlap)
    constexpr int PER = (CAP + G - 1) / G;
    E4 te[PER];
    V2 tv[PER];
    int ti[PER], dst[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int k = glane + q * G;
        dst[q] = -1;
        if (go && k < m) {
            int nk = -1;
            if (s <= e) nk = k > e ? k + 2 - c : -1;   // k <= s stays where it is, s < k <= e goes
            else nk = (k > e && k <= s) ? k - (e + 1) : -1;
            if (nk >= 0 && nk != k) {
                dst[q] = nk;
                te[q] = b.R.edge(k);
                tv[q] = b.R.vert(k);
                ti[q] = b.R.idx(k);
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        if (dst[q] >= 0) {
            b.R.set_edge(dst[q], te[q]);
            b.R.set_vert(dst[q], tv[q], ti[q]);
        }
    }
    __syncwarp();
    if (go) {
        if (glane == 0) b.R.set_edge(ns, ca);
        if (glane == 1) b.R.set_vert(ns + 1, d, id);
        if (glane == 2) b.R.set_edge(ns + 1, cb);
        if (glane == 0) b.ctr.add_ins();
        b.m = mnew;
        const T rn = ca.w > cb.w ? ca.w : cb.w;
        const T r2n = B::r2_of(rn);
        if (!(r2n <= b.r2max)) b.r2max = r2n;   // an infinite circle disables the prefilter
    }
    __syncwarp();
    return r;
}

// The construction of one point per group.  Every lane of the warp calls it (warp votes and
// full-warp shuffles inside); `act` is false for groups without a point.  Returns R_OK or
// the reason the point goes elsewhere, the same on every lane of the group.
template <int G, class B>
__device__ int grp_build(B &b, const bool act, const int glane)
{
    typedef typename B::Mask Mask;
    typedef typename B::V2 V2;
    const RingArgs &A = b.A;
    const SetDesc &S = b.S;
    if (act && glane == 0) b.init_ring();
    __syncwarp();
    b.init_local();
    const double2 fp = cell_pos<B::general>(S, b.p);
    const double fx = fp.x - (double)b.ocx, fy = fp.y - (double)b.ocy;
    int x0 = 0, x1 = -1, y0 = 0, y1 = -1;   // the scanned rectangle (relative cells; none yet)
    const int max_phase = S.xsize + S.ysize + 8;
    bool done = !act;
    int status = R_OK;
    for (int phase = 0;; ++phase) {
        bool live = !done && status == R_OK;
        int gx0 = x0, gx1 = x1, gy0 = y0, gy1 = y1;
        if (live && phase >= max_phase) {
            done = true;
            live = false;
        }
        if (live && phase == 0) {
            // the own cell
            gx0 = gx1 = gy0 = gy1 = 0;
        } else if (live) {
            // certification: grow towards the cells the edge circles reach, one per side (a
            // ring that still holds virtual corners takes the whole 3x3 block; a ring whose
            // circles lie inside the own cell, as in dense clusters, stops there)
            int lx, hx, ly, hy;
            if (!b.need_rect(fx, fy, lx, hx, ly, hy)) {
                lx = ly = -(1 << 28);
                hx = hy = (1 << 28);
            }
            if (lx < x0 && gx1 - gx0 + 1 < S.xsize) gx0--;
            if (hx > x1 && gx1 - gx0 + 1 < S.xsize) gx1++;
            if (ly < y0 && gy1 - gy0 + 1 < S.ysize) gy0--;
            if (hy > y1 && gy1 - gy0 + 1 < S.ysize) gy1++;
            if (gx0 == x0 && gx1 == x1 && gy0 == y0 && gy1 == y1) {
                done = true;
                live = false;
            }
        }
        if (!__any_sync(FULL, live)) break;
        // the phase's new cells as row segments [rxa, rxb] x {ry}: phase 0 the own cell; later
        // the left and right columns over the old rows (a segment per cell), then the rows
        // below and above over the new columns
        const int w = gx1 - gx0 + 1;
        int nl = 0, nr = 0, nb = 0, nt = 0, nseg = 0, ncells = 0;
        if (live) {
            if (phase == 0) {
                nseg = 1;
                ncells = 1;
            } else {
                nl = gx0 < x0 ? y1 - y0 + 1 : 0;
                nr = gx1 > x1 ? y1 - y0 + 1 : 0;
                nb = gy0 < y0 ? 1 : 0;
                nt = gy1 > y1 ? 1 : 0;
                nseg = nl + nr + nb + nt;
                ncells = nl + nr + (nb + nt) * w;
            }
            if (glane == 0) {
                b.ctr.add_cells((unsigned)ncells);
                b.R.work() += ncells;
            }
        }
        for (int c0 = 0; __any_sync(FULL, c0 < nseg); c0 += G) {
            // this lane's segment: up to two slot ranges (a row run across the periodic seam)
            const int sg = c0 + glane;
            int st1 = 0, n1 = 0, st2 = 0, n2 = 0;
            if (sg < nseg) {
                int ry, rxa, rxb;
                if (phase == 0) {
                    ry = rxa = rxb = 0;
                } else if (sg < nl) {
                    ry = y0 + sg;
                    rxa = rxb = x0 - 1;
                } else if (sg < nl + nr) {
                    ry = y0 + sg - nl;
                    rxa = rxb = x1 + 1;
                } else {
                    ry = (sg < nl + nr + nb) ? y0 - 1 : y1 + 1;
                    rxa = gx0;
                    rxb = gx1;
                }
                const int cy = wrapi(b.ocy + ry, S.ysize);
                const int ax = wrapi(b.ocx + rxa, S.xsize), len = rxb - rxa + 1;
                const int row = S.cell_base + cy * S.xsize;
                if (ax + len <= S.xsize) {
                    st1 = __ldg(&A.cstart[row + ax]);
                    n1 = __ldg(&A.cstart[row + ax + len]) - st1;
                } else {
                    st1 = __ldg(&A.cstart[row + ax]);
                    n1 = __ldg(&A.cstart[row + S.xsize]) - st1;
                    st2 = __ldg(&A.cstart[row]);
                    n2 = __ldg(&A.cstart[row + ax + len - S.xsize]) - st2;
                }
            }
            const int cnt = n1 + n2;
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < G; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o, G);
                if (glane >= o) incl += v;
            }
            const int total = gshfl<G>(incl, G - 1), excl = incl - cnt;
            if (live && glane == 0) b.R.work() += total;
            for (int j0 = 0; __any_sync(FULL, j0 < total); j0 += G) {
                const int j = j0 + glane;
                const bool have = live && status == R_OK && j < total;
                // the lane whose segment holds candidate j: the last one starting at or before j
                int o = 0;
#pragma unroll
                for (int step = G / 2; step > 0; step >>= 1) {
                    const int ex = gshfl<G>(excl, o + step);
                    if (ex <= j) o += step;
                }
                // (every shuffle on every lane: a shuffle taken by only some lanes reads garbage)
                const int q = j - gshfl<G>(excl, o);
                const int on1 = gshfl<G>(n1, o), ost1 = gshfl<G>(st1, o), ost2 = gshfl<G>(st2, o);
                const int sl = q < on1 ? ost1 + q : ost2 + (q - on1);
                // classify against the current ring
                V2 d = B::PR::mk2(0, 0);
                double2 d64 = make_double2(0.0, 0.0);
                Mask mask = 0;
                int rc = R_OK;
                if (have) rc = b.classify(sl, d, mask, d64);
                if (gvote<G>(rc != R_OK)) {
                    status = R_EXACT;
                    mask = 0;
                }
                bool want = have && status == R_OK && mask != 0;
                while (__any_sync(FULL, want)) {
                    // the nearest conflicting candidate of each group goes in
                    unsigned key = want ? near_key<G>((float)(d.x * d.x + d.y * d.y), glane) : 0xffffffffu;
#pragma unroll
                    for (int o2 = G / 2; o2 > 0; o2 >>= 1) key = min(key, __shfl_xor_sync(FULL, key, o2, G));
                    const bool ins = key != 0xffffffffu;
                    const int win = (int)(key & (unsigned)(G - 1));
                    const V2 dw = B::PR::mk2(gshfl<G>(d.x, win), gshfl<G>(d.y, win));
                    const Mask mw = (Mask)gshfl<G>((unsigned)mask, win);
                    int id = (want && glane == win) ? __ldg(&A.sidx[sl]) : 0;
                    id = gshfl<G>(id, win);
                    int s, e, ns;
                    const int ir = grp_insert<G>(b, ins, glane, dw, id, mw, s, e, ns);
                    if (ins && ir != R_OK) {
                        status = ir;
                        want = false;
                    }
                    if (glane == win) want = false;
                    int rr = R_OK;
                    if (want) {
                        // edges outside the inserted arc keep their circles (and decisions)
                        int ns2;
                        Mask nmk = B::remap_mask(mask, s, e, ns2);
                        const int i0 = b.test_edge(ns, d, d64);
                        const int i1 = b.test_edge(ns + 1, d, d64);
                        if (i0 < 0 || i1 < 0) rr = R_EXACT;
                        nmk |= (Mask)(i0 > 0) << ns;
                        nmk |= (Mask)(i1 > 0) << (ns + 1);
                        mask = nmk;
                    }
                    if (gvote<G>(rr != R_OK)) {
                        status = R_EXACT;
                        want = false;
                    }
                    want = want && mask != 0;
                }
            }
        }
        __syncwarp();   // the group's work count, written by its first lane
        if (live) {
            // over the work budget: the warp-per-point kernel takes the point over
            if (status == R_OK && b.R.work() > A.work_budget) status = R_HEAVY;
            x0 = gx0;
            x1 = gx1;
            y0 = gy0;
            y1 = gy1;
        }
        if (__all_sync(FULL, done || status != R_OK)) break;
    }
    if (!act) return R_OK;
    if (status != R_OK) return status;
    for (int k = 0; k < b.m; ++k)
        if (b.R.idx(k) < 0) return R_UNBOUNDED;
    if (b.minimage && glane == 0) atomicOr(&A.st->err_flags, EF_MINIMAGE);
    return R_OK;
}

}  // namespace

// G lanes per point, BLOCK / G points per block; ring of CAP entries per point in shared
// memory; IDX: candidate and own positions through the index (repair rounds), else from the
// cell-order copy (global build); GEN: general periodic box
template <typename T, int CAP, int G, int BLOCK, bool IDX, bool GEN>
__global__ void __launch_bounds__(BLOCK) k_build_grp(RingArgs A)
{
    typedef typename Prec<T>::T4 E4;
    typedef typename Prec<T>::T2 V2;
    constexpr int NG = BLOCK / G;
    __shared__ E4 se[CAP][NG];
    __shared__ V2 sv[CAP][NG];
    __shared__ int si[CAP][NG];
    __shared__ int swork[NG];
    __shared__ unsigned srare[5][BLOCK];
    const int glane = threadIdx.x & (G - 1), grp = threadIdx.x / G;
    SmemRing<T, CAP, NG> ring{ se, sv, si, swork, grp };
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
    for (int base = blockIdx.x * NG; base < n; base += gridDim.x * NG) {
        const int t = base + grp;
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
        const int si_ = (act && A.set_of) ? __ldg(&A.set_of[slot]) : 0;
        const SetDesc S = A.sets[si_];
        const double2 p = !act ? make_double2(0.0, 0.0) : (IDX ? __ldg(&A.pos[pid]) : __ldg(&A.spos[slot]));
        Builder<T, false, SmemRing<T, CAP, NG>, SmemCtr<BLOCK>, IDX ? 1 : 0, GEN> b(A, S, ring, ctr, p, slot,
                                                                                  A.sets + si_);
        const int r = grp_build<G>(b, act, glane);
        if (act && glane == 0) {
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
        __syncwarp();
    }
    flush_counters(A, ctr.total(), pts, maxr);
}

template <typename T, int CAP, int G, int BLOCK, bool GEN>
static cudaError_t launch_grp_t(const RingArgs &a, int sms, cudaStream_t s)
{
    constexpr int NG = BLOCK / G;
    int blocks;
    if (a.worklist) {
        const int want = (a.n_items + NG - 1) / NG;
        blocks = want < sms * 32 ? want : sms * 32;
    } else {
        blocks = (a.n_items + NG - 1) / NG;
    }
    if (blocks < 1) blocks = 1;
    if (a.cand_by_index) k_build_grp<T, CAP, G, BLOCK, true, GEN><<<blocks, BLOCK, 0, s>>>(a);
    else k_build_grp<T, CAP, G, BLOCK, false, GEN><<<blocks, BLOCK, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_build_group(const RingArgs &a, int mode, int sms, int lanes, cudaStream_t s)
{
    if (a.n_items <= 0) return cudaSuccess;
    if (a.general) {
        if (mode == MODE_F64) return launch_grp_t<double, 14, 8, 64, true>(a, sms, s);
        return lanes == 4 ? launch_grp_t<float, 14, 4, 64, true>(a, sms, s)
                          : launch_grp_t<float, 14, 8, 64, true>(a, sms, s);
    }
    if (mode == MODE_F64) {
        return lanes == 4 ? launch_grp_t<double, 14, 4, 64, false>(a, sms, s)
                          : launch_grp_t<double, 14, 8, 64, false>(a, sms, s);
    }
    return lanes == 4 ? launch_grp_t<float, 14, 4, 64, false>(a, sms, s)
                      : launch_grp_t<float, 14, 8, 64, false>(a, sms, s);
}

}  // namespace dgt

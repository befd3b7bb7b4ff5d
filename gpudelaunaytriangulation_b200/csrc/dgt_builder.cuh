// The per-point one-ring builder shared by the construction kernels (dgt_ring.cu: one thread
// per point, and the warp per point of the deferred path; dgt_group.cu: a group of lanes per
// point): ring storage policies, the candidate classification against the ring's edge
// circles, insertion, certification of the scanned cell rectangle, and the output /
// repair bookkeeping of a finished ring.  See dgt_ring.cu for the construction itself.
#pragma once
#include "dgt_internal.cuh"
#include "dgt_predicates.cuh"
#include "dgt_rowreg.cuh"

namespace dgt {

enum { R_OK = 0, R_CAPACITY = 1, R_EXACT = 2, R_UNBOUNDED = 3, R_NONCONTIG = 4, R_HEAVY = 5 };

// statistics of one thread
struct Ctr {
    unsigned cand, tests, u32, u64, ins, mism, cells;
    __device__ __forceinline__ void add_u32() { u32++; }
    __device__ __forceinline__ void add_u64() { u64++; }
    __device__ __forceinline__ void add_ins() { ins++; }
    __device__ __forceinline__ void add_mism(unsigned v) { mism += v; }
    __device__ __forceinline__ void add_cells() { cells++; }
    __device__ __forceinline__ void add_cells(unsigned v) { cells += v; }
    __device__ __forceinline__ Ctr total() const { return *this; }
};
// the same, with the rarely bumped counters in shared memory (one column per thread): the
// per-thread kernel's registers are what limits its occupancy
template <int BLOCK>
struct SmemCtr {
    unsigned cand, tests;
    unsigned (*rare)[BLOCK];   // rows: u32, u64, ins, mism, cells
    __device__ __forceinline__ void add_u32() { rare[0][threadIdx.x]++; }
    __device__ __forceinline__ void add_u64() { rare[1][threadIdx.x]++; }
    __device__ __forceinline__ void add_ins() { rare[2][threadIdx.x]++; }
    __device__ __forceinline__ void add_mism(unsigned v) { rare[3][threadIdx.x] += v; }
    __device__ __forceinline__ void add_cells() { rare[4][threadIdx.x]++; }
    __device__ __forceinline__ void add_cells(unsigned v) { rare[4][threadIdx.x] += v; }
    __device__ __forceinline__ Ctr total() const
    {
        const int t = threadIdx.x;
        return Ctr{ cand, tests, rare[0][t], rare[1][t], rare[2][t], rare[3][t], rare[4][t] };
    }
};

// ---------------------------------------------------------------- ring storage policies
template <typename T, int CAP, int BLOCK>
struct SmemRing {
    typedef typename Prec<T>::T4 E4;
    typedef typename Prec<T>::T2 V2;
    E4 (*e)[BLOCK];
    V2 (*v)[BLOCK];
    int (*id)[BLOCK];
    int *wk;   // per-thread scan work of the current point (per-thread kernel only)
    int t;
    static constexpr int cap = CAP;
    __device__ __forceinline__ int &work() { return wk[t]; }
    __device__ __forceinline__ E4 edge(int k) const { return e[k][t]; }
    __device__ __forceinline__ V2 vert(int k) const { return v[k][t]; }
    __device__ __forceinline__ int idx(int k) const { return id[k][t]; }
    __device__ __forceinline__ void set_edge(int k, E4 x) { e[k][t] = x; }
    __device__ __forceinline__ void set_vert(int k, V2 x, int i) { v[k][t] = x; id[k][t] = i; }
    __device__ __forceinline__ void move(int dst, int src)
    {
        e[dst][t] = e[src][t];
        v[dst][t] = v[src][t];
        id[dst][t] = id[src][t];
    }
};

template <int CAP> struct MaskT { typedef unsigned int type; };
template <> struct MaskT<64> { typedef unsigned long long type; };
__device__ __forceinline__ int popc_(unsigned int x) { return __popc(x); }
__device__ __forceinline__ int popc_(unsigned long long x) { return __popcll(x); }
__device__ __forceinline__ int ffs_(unsigned int x) { return __ffs(x); }
__device__ __forceinline__ int ffs_(unsigned long long x) { return __ffsll(x); }

// i in [-n, 2n): one correction brings it into [0, n)
__device__ __forceinline__ int wrapi(int i, int n)
{
    return i < 0 ? i + n : (i >= n ? i - n : i);
}

template <typename T>
__device__ __forceinline__ typename Prec<T>::T2 corner(int c, T V)
{
    return Prec<T>::mk2((c == 0 || c == 3) ? V : -V, (c < 2) ? V : -V);
}

// ------------------------------------------------------- out-of-line rare paths (small hot loop)
// double offset of ring entry `id` relative to p
__device__ __forceinline__ double2 off64(const double2 *pos, double2 p, double Lx, double hLx, double Ly,
                                         double hLy, float V, int id)
{
    if (id >= 0) {
        double2 q = __ldg(&pos[id]);
        return make_double2(wrap_off(q.x, p.x, Lx, hLx), wrap_off(q.y, p.y, Ly, hLy));
    }
    int c = -id - 1;   // virtual corners 0:(V,V) 1:(-V,V) 2:(-V,-V) 3:(V,-V)
    double v = (double)V;
    return make_double2((c == 0 || c == 3) ? v : -v, (c < 2) ? v : -v);
}

// float64 in-circle of d against edge (ia, ib); with exact: exact sign when float64 cannot
// decide.  Returns +1/-1 decided in float64, +2/-2 decided exactly, 0 undecided.
template <bool EXACT>
__device__ __noinline__ int recheck64(const double2 *pos, double2 p, double Lx, double hLx, double Ly,
                                      double hLy, float V, int ia, int ib, double dx, double dy)
{
    double2 a = off64(pos, p, Lx, hLx, Ly, hLy, V, ia), b = off64(pos, p, Lx, hLx, Ly, hLy, V, ib);
    int r = incircle64(a.x, a.y, b.x, b.y, dx, dy);
    if (r != 0 || !EXACT) return r;
    r = incircle_exact(a.x, a.y, b.x, b.y, dx, dy);
    return r > 0 ? 2 : -2;   // on the circle: not strictly inside
}

// check mode: 1 when float64 certainly contradicts the filter's decision `inside`
static __device__ __noinline__ int check64(const double2 *pos, double2 p, double Lx, double hLx, double Ly, double hLy,
                                    float V, int ia, int ib, double dx, double dy, int inside)
{
    double2 a = off64(pos, p, Lx, hLx, Ly, hLy, V, ia), b = off64(pos, p, Lx, hLx, Ly, hLy, V, ib);
    int r = incircle64(a.x, a.y, b.x, b.y, dx, dy);
    return (inside && r < 0) || (!inside && r > 0) ? 1 : 0;
}

// circle of edge (ia, ib) in double (make_circ layout)
static __device__ __noinline__ double4 circle64(const double2 *pos, double2 p, double Lx, double hLx, double Ly,
                                         double hLy, float V, int ia, int ib)
{
    double2 a = off64(pos, p, Lx, hLx, Ly, hLy, V, ia), b = off64(pos, p, Lx, hLx, Ly, hLy, V, ib);
    return make_circ<double>(a.x, a.y, b.x, b.y);
}

// the same three for a general box (S: the set's descriptor in global memory)
__device__ __forceinline__ double2 off64g(const double2 *pos, double2 p, const SetDesc *S, int id)
{
    if (id >= 0) return gen_off(__ldg(&pos[id]), p, *S);
    int c = -id - 1;
    double v = (double)S->V;
    return make_double2((c == 0 || c == 3) ? v : -v, (c < 2) ? v : -v);
}
template <bool EXACT>
__device__ __noinline__ int recheck64g(const double2 *pos, double2 p, const SetDesc *S, int ia, int ib, double dx,
                                       double dy)
{
    double2 a = off64g(pos, p, S, ia), b = off64g(pos, p, S, ib);
    int r = incircle64(a.x, a.y, b.x, b.y, dx, dy);
    if (r != 0 || !EXACT) return r;
    r = incircle_exact(a.x, a.y, b.x, b.y, dx, dy);
    return r > 0 ? 2 : -2;
}
static __device__ __noinline__ int check64g(const double2 *pos, double2 p, const SetDesc *S, int ia, int ib, double dx,
                                     double dy, int inside)
{
    double2 a = off64g(pos, p, S, ia), b = off64g(pos, p, S, ib);
    int r = incircle64(a.x, a.y, b.x, b.y, dx, dy);
    return (inside && r < 0) || (!inside && r > 0) ? 1 : 0;
}
static __device__ __noinline__ double4 circle64g(const double2 *pos, double2 p, const SetDesc *S, int ia, int ib)
{
    double2 a = off64g(pos, p, S, ia), b = off64g(pos, p, S, ib);
    return make_circ<double>(a.x, a.y, b.x, b.y);
}

// ------------------------------------------------------------------- the construction
// CAND: where candidate positions come from -- 0 the cell-order copy (current after a
// binning), 1 the caller's positions through the index (repair: the cell lists may be older
// than the positions), 2 chosen at run time by A.cand_by_index.  GEN: general periodic box
// (offsets, cells and certification in the box's fractional frame; Sg: the set's descriptor
// in global memory, for the out-of-line float64 paths)
// own-cell points up to which a warp's first phase takes the whole 3x3 block (measured on 4M
// uniform points: 2 -> 6.64 ms, 4 -> 5.87, 8 -> 5.79, 16 -> 5.79, against 6.00 ms own cell
// first; a lane-by-lane choice at 4 made the clustered mixture 2% slower)
constexpr int BLOCK_FIRST_MAX = 8;
template <typename T, bool EXACT, class Ring, class C = Ctr, int CAND = 2, bool GEN = false>
struct Builder {
    static constexpr bool general = GEN;
    typedef T Real;
    typedef Ring RingT;
    typedef Prec<T> PR;
    typedef typename PR::T4 E4;
    typedef typename PR::T2 V2;
    typedef typename MaskT<Ring::cap>::type Mask;

    const RingArgs &A;
    const SetDesc &S;
    const SetDesc *Sg;
    Ring &R;
    C &ctr;
    double2 p;
    int slot;
    int m;
    T r2max;
    int ocx, ocy;
    bool minimage = false;   // the certified circles reach past half the box

    __device__ Builder(const RingArgs &a, const SetDesc &s, Ring &r, C &c, double2 pp, int sl,
                       const SetDesc *sg = nullptr)
        : A(a), S(s), Sg(sg), R(r), ctr(c), p(pp), slot(sl), m(0), r2max((T)0), ocx(0), ocy(0) {}

    // r2max bounds |d|^2 for any d inside some edge circle (a circle through the origin of
    // radius <= rc lies within 2 rc of it): the candidate prefilter.  Exact maximum here;
    // inserts only fold in their two new circles (still an upper bound: the other circles
    // are unchanged), and the exact value is restored where the edges are walked anyway.
    __device__ __forceinline__ static T r2_of(T rc) { return (T)4 * rc * rc * ((T)1 + (T)64 * PR::u()); }
    __device__ void refresh_r2max()
    {
        T mx = (T)0;
        for (int k = 0; k < m; ++k) {
            T rc = R.edge(k).w;
            mx = rc > mx ? rc : mx;
        }
        r2max = r2_of(mx);
    }

    // the square of virtual corners (ring storage only)
    __device__ void init_ring()
    {
        T V = (T)S.V;
        for (int c = 0; c < 4; ++c) R.set_vert(c, corner<T>(c, V), -1 - c);
        for (int c = 0; c < 4; ++c) {
            V2 a = corner<T>(c, V), b = corner<T>((c + 1) & 3, V);
            R.set_edge(c, make_circ<T>(a.x, a.y, b.x, b.y));
        }
    }
    // per-thread state of a fresh ring (reads the ring storage)
    __device__ void init_local()
    {
        if (!EXACT) R.work() = 0;
        m = 4;
        refresh_r2max();
        const double2 f = cell_pos<GEN>(S, p);
        int cx = (int)floor(f.x), cy = (int)floor(f.y);
        ocx = min(max(cx, 0), S.xsize - 1);
        ocy = min(max(cy, 0), S.ysize - 1);
    }
    __device__ void init()
    {
        init_ring();
        init_local();
    }

    // float64 (then, on the exact path, exact) decision for edge k against candidate d:
    // +1 conflict, -1 none, 0 undecided (only without EXACT)
    __device__ __forceinline__ int recheck(int k, double2 d64)
    {
        int ia = R.idx(k), ib = R.idx(k + 1 == m ? 0 : k + 1);
        int r = GEN ? recheck64g<EXACT>(A.pos, p, Sg, ia, ib, d64.x, d64.y)
                    : recheck64<EXACT>(A.pos, p, S.Lx, S.hLx, S.Ly, S.hLy, S.V, ia, ib, d64.x, d64.y);
        if (r == 2 || r == -2 || r == 0) ctr.add_u64();
        return r > 0 ? 1 : (r < 0 ? -1 : 0);
    }

    __device__ int insert(V2 d, int id, Mask mask)
    {
        Mask full = (m == 64) ? ~(Mask)0 : (((Mask)1 << m) - 1);
        Mask nm = ~mask & full;
        Mask rl = ((nm << 1) | (nm >> (m - 1))) & full;
        Mask rr = ((nm >> 1) | (nm << (m - 1))) & full;
        Mask starts = mask & rl, ends = mask & rr;
        if (mask == full || popc_(starts) != 1) return R_NONCONTIG;
        int s = ffs_(starts) - 1, e = ffs_(ends) - 1, c = popc_(mask);
        int mnew = m - c + 2;
        if (mnew > Ring::cap) return R_CAPACITY;
        V2 vs = R.vert(s), ve = R.vert(e + 1 == m ? 0 : e + 1);
        E4 ca = make_circ<T>(vs.x, vs.y, d.x, d.y);
        E4 cb = make_circ<T>(d.x, d.y, ve.x, ve.y);
        int ns;
        if (s <= e) {
            int delta = 2 - c;
            if (delta > 0) {
                for (int k = m - 1; k >= e + 1; --k) R.move(k + 1, k);
            } else if (delta < 0) {
                for (int k = e + 1; k < m; ++k) R.move(k + delta, k);
            }
            ns = s;
        } else {
            for (int k = e + 1; k <= s; ++k) R.move(k - (e + 1), k);
            ns = s - e - 1;
        }
        R.set_edge(ns, ca);
        R.set_vert(ns + 1, d, id);
        R.set_edge(ns + 1, cb);
        m = mnew;
        ctr.add_ins();
        const T rn = ca.w > cb.w ? ca.w : cb.w;
        const T r2n = r2_of(rn);
        if (!(r2n <= r2max)) r2max = r2n;   // an infinite (unbounded) circle disables the prefilter
        return R_OK;
    }

    // one candidate (cell-order slot sl) against every ring edge: `mask` gets the edges whose
    // circle holds it strictly inside (undecided filters settled by recheck); d its offset
    __device__ __forceinline__ int classify(int sl, V2 &d, Mask &mask)
    {
        double2 d64;
        return classify(sl, d, mask, d64);
    }
    // the same, also giving the candidate's double offset (for later rechecks)
    __device__ __forceinline__ int classify(int sl, V2 &d, Mask &mask, double2 &d64)
    {
        mask = 0;
        d64 = make_double2(0.0, 0.0);
        if (sl == slot) return R_OK;
        // repair calls read candidates through the index: the cell-order copy may be older
        // than the positions (cell lists kept from the last binning)
        const bool by_index = CAND == 1 || (CAND == 2 && A.cand_by_index);
        double2 q = by_index ? __ldg(&A.pos[__ldg(&A.sidx[sl])]) : __ldg(&A.spos[sl]);
        // general box: the matrices are read through the descriptor in global memory (L1
        // hits) rather than held in registers across the scan
        d64 = GEN ? gen_off(q, p, *Sg)
                  : make_double2(wrap_off(q.x, p.x, S.Lx, S.hLx), wrap_off(q.y, p.y, S.Ly, S.hLy));
        if (d64.x == 0.0 && d64.y == 0.0) return R_OK;   // coincident point
        ctr.cand++;
        d = PR::mk2(PR::from64(d64.x), PR::from64(d64.y));
        T nd = d.x * d.x + d.y * d.y;
        if (nd > r2max) return R_OK;
        T ad = sqrt_up(nd);   // only scales the bound: an upper value is safe
        T kb = (T)8 * PR::u() * nd + PR::tiny();
        Mask open = 0;
        // two edges per trip: their loads and tests overlap (measured: -4% build time)
#pragma unroll 2
        for (int k = 0; k < m; ++k) {
            E4 e = R.edge(k);
            T sv = fma(d.x, e.x, fma(d.y, e.y, -nd));
            T bd = fma(ad, e.z, kb);
            mask |= (Mask)(sv > bd) << k;
            open |= (Mask)(sv <= bd && sv >= -bd) << k;
        }
        ctr.tests += m;
        if (open) {
            for (int k = 0; k < m; ++k) {
                if (!((open >> k) & 1)) continue;
                ctr.add_u32();
                int r = recheck(k, d64);
                if (r == 0) return R_EXACT;
                if (r > 0) mask |= (Mask)1 << k;
            }
        }
        if (A.check) {
            for (int k = 0; k < m; ++k) {
                if ((open >> k) & 1) continue;
                int ia = R.idx(k), ib = R.idx(k + 1 == m ? 0 : k + 1);
                ctr.add_mism(GEN ? check64g(A.pos, p, Sg, ia, ib, d64.x, d64.y, (int)((mask >> k) & 1))
                                 : check64(A.pos, p, S.Lx, S.hLx, S.Ly, S.hLy, S.V, ia, ib, d64.x, d64.y,
                                           (int)((mask >> k) & 1)));
            }
        }
        return R_OK;
    }

    // One ring edge k against candidate d (float offset) / d64 (double offset): 1 strictly
    // inside its circle, 0 not, -1 undecided even in float64 (only without EXACT).  The
    // filter of classify for a single edge, with the same recheck and check-mode accounting.
    __device__ __forceinline__ int test_edge(int k, V2 d, double2 d64)
    {
        const T nd = d.x * d.x + d.y * d.y;
        const T ad = sqrt_up(nd);
        const T kb = (T)8 * PR::u() * nd + PR::tiny();
        const E4 e = R.edge(k);
        const T sv = fma(d.x, e.x, fma(d.y, e.y, -nd));
        const T bd = fma(ad, e.z, kb);
        ctr.tests++;
        if (sv > bd || sv < -bd) {
            const int in = sv > bd ? 1 : 0;
            if (A.check) {
                const int ia = R.idx(k), ib = R.idx(k + 1 == m ? 0 : k + 1);
                ctr.add_mism(GEN ? check64g(A.pos, p, Sg, ia, ib, d64.x, d64.y, in)
                                 : check64(A.pos, p, S.Lx, S.hLx, S.Ly, S.hLy, S.V, ia, ib, d64.x, d64.y, in));
            }
            return in;
        }
        ctr.add_u32();
        const int r = recheck(k, d64);
        return r == 0 ? -1 : (r > 0 ? 1 : 0);
    }

    // The conflict arc of `mask` on a ring of m entries: first edge s, last edge e (s > e when
    // it wraps past the end), count c; false when the conflicting edges are not one arc.
    __device__ __forceinline__ static bool conflict_arc(Mask mask, int m, int &s, int &e, int &c)
    {
        const Mask full = (m == 8 * (int)sizeof(Mask)) ? ~(Mask)0 : (((Mask)1 << m) - 1);
        const Mask nm = ~mask & full;
        const Mask rl = ((nm << 1) | (nm >> (m - 1))) & full;
        const Mask rr = ((nm >> 1) | (nm << (m - 1))) & full;
        const Mask starts = mask & rl, ends = mask & rr;
        s = ffs_(starts) - 1;
        e = ffs_(ends) - 1;
        c = popc_(mask);
        return mask != full && popc_(starts) == 1;
    }
    // After inserting a candidate over arc [s, e]: another candidate's decisions for the
    // edges that survive (same circles) at their new indices; the two new edges start at
    // the returned index (their bits are left clear).
    __device__ __forceinline__ static Mask remap_mask(Mask mk, int s, int e, int &ns)
    {
        if (s <= e) {
            ns = s;
            const Mask low = s == 0 ? (Mask)0 : ((((Mask)1 << s) - 1) & mk);
            return low | ((mk >> (e + 1)) << (s + 2));
        }
        ns = s - e - 1;
        const Mask keep = ns == 0 ? (Mask)0 : (((Mask)1 << ns) - 1);
        return (mk >> (e + 1)) & keep;
    }

    // one candidate: classify, insert on conflict
    __device__ __forceinline__ int candidate(int sl)
    {
        V2 d;
        Mask mask;
        int r = classify(sl, d, mask);
        if (r != R_OK || !mask) return r;
        return insert(d, __ldg(&A.sidx[sl]), mask);
    }

    // Growth of the scanned rectangle from [x0,x1]x[y0,y1] to [nx0,nx1]x[ny0,ny1] by at most
    // one column / row per side; its new cells are the left column, the right column (over
    // the old rows), then the bottom and top rows (over the new columns).  own: the single
    // cell (0,0) of the first phase.
    struct Growth {
        int x0, x1, y0, y1, nx0, nx1, ny0, ny1, nl, nr, nb, nt;
        bool own, block;
    };
    __device__ __forceinline__ static Growth growth(int x0, int x1, int y0, int y1, int nx0, int nx1, int ny0,
                                                    int ny1, bool own, bool block = false)
    {
        Growth g{ x0, x1, y0, y1, nx0, nx1, ny0, ny1, 0, 0, 0, 0, own, block };
        if (own || block) return g;
        g.nl = nx0 < x0 ? (y1 - y0 + 1) : 0;
        g.nr = nx1 > x1 ? (y1 - y0 + 1) : 0;
        g.nb = ny0 < y0 ? (nx1 - nx0 + 1) : 0;
        g.nt = ny1 > y1 ? (nx1 - nx0 + 1) : 0;
        return g;
    }
    __device__ __forceinline__ static void growth_cell(const Growth &g, int ci, int &rx, int &ry)
    {
        if (g.own) { rx = 0; ry = 0; return; }
        if (g.block) {
            // the 3x3 block: own cell, edge neighbours, corners (2-bit codes of x + 1, y + 1)
            rx = (int)((0x8949u >> (2 * ci)) & 3u) - 1;
            ry = (int)((0x2895u >> (2 * ci)) & 3u) - 1;
            return;
        }
        if (ci < g.nl) { rx = g.x0 - 1; ry = g.y0 + ci; return; }
        ci -= g.nl;
        if (ci < g.nr) { rx = g.x1 + 1; ry = g.y0 + ci; return; }
        ci -= g.nr;
        if (ci < g.nb) { rx = g.nx0 + ci; ry = g.y0 - 1; return; }
        ci -= g.nb;
        rx = g.nx0 + ci;
        ry = g.y1 + 1;
    }

    // every candidate of the growth's cells.  The lanes of a warp advance in lockstep, one
    // candidate each per step (a warp vote closes every step), so the candidate code runs
    // with all lanes that still have candidates.  Every lane of the warp must call this;
    // `live` is false for lanes with nothing to scan.
    __device__ __forceinline__ int scan(const Growth &g, bool live)
    {
        const int ncell = !live ? 0 : (g.own ? 1 : (g.block ? 9 : g.nl + g.nr + g.nb + g.nt));
        int ci = 0, sl = 0, se = 0, status = R_OK;
        // the ranges of cells ci and ci + 1 are loaded ahead of their use, so a lane moving
        // to its next cell rarely waits on the load (measured: -1.7% build time)
        int asl = 0, ase = 0, bsl = 0, bse = 0;
        auto fetch = [&](int k, int &fs, int &fe) {
            int rx, ry;
            growth_cell(g, k, rx, ry);
            const int cx = wrapi(ocx + rx, S.xsize), cy = wrapi(ocy + ry, S.ysize);
            const int c = S.cell_base + cy * S.xsize + cx;
            fs = __ldg(&A.cstart[c]);
            fe = __ldg(&A.cstart[c + 1]);
        };
        if (ncell > 0) fetch(0, asl, ase);
        if (ncell > 1) fetch(1, bsl, bse);
        for (;;) {
            bool have = false;
            if (status == R_OK) {
                while (sl >= se && ci < ncell) {
                    sl = asl;
                    se = ase;
                    asl = bsl;
                    ase = bse;
                    ctr.add_cells();
                    if (!EXACT) R.work() += 1 + se - sl;   // checked against the budget per phase
                    if (++ci + 1 < ncell) fetch(ci + 1, bsl, bse);
                }
                have = sl < se;
            }
            if (!__any_sync(0xffffffffu, have)) break;
            if (have) {
                int r = candidate(sl++);
                if (r != R_OK) status = r;
            }
        }
        return status;
    }

    // Certification: cells (relative to the own cell) covering the union of the edge circles'
    // bounding boxes.  Returns false when some circle cannot be bounded (whole box needed).
    __device__ bool need_rect(double fx, double fy, int &lx, int &hx, int &ly, int &hy)
    {
        if (GEN) return need_rect_gen(fx, fy, lx, hx, ly, hy);
        double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
        T mx = (T)0;
        bool finite = true;
        for (int k = 0; k < m; ++k) {
            E4 e = R.edge(k);
            double cx, cy, rc;
            mx = e.w > mx ? e.w : mx;
            finite &= e.w < PR::inf();
            if (e.w < PR::inf()) {
                cx = 0.5 * (double)e.x;
                cy = 0.5 * (double)e.y;
                rc = (double)e.w;
            } else {
                int ia = R.idx(k), ib = R.idx(k + 1 == m ? 0 : k + 1);
                double4 c = circle64(A.pos, p, S.Lx, S.hLx, S.Ly, S.hLy, S.V, ia, ib);
                if (!(c.w < Prec<double>::inf())) {
                    minimage = true;
                    return false;
                }
                cx = 0.5 * c.x;
                cy = 0.5 * c.y;
                rc = c.w;
            }
            xmin = fmin(xmin, cx - rc);
            xmax = fmax(xmax, cx + rc);
            ymin = fmin(ymin, cy - rc);
            ymax = fmax(ymax, cy + rc);
        }
        if (finite) r2max = r2_of(mx);   // the exact prefilter bound, restored for free
        // judged on the circles of the latest ring only (the final one when the scan ends)
        minimage = xmin < -S.hLx || xmax > S.hLx || ymin < -S.hLy || ymax > S.hLy;
        // cell lists older than the positions: a point may sit up to `sk` cells from the cell
        // that lists it
        const double sk = A.skin ? (double)*A.skin : 0.0;
        double a0 = fx + xmin * S.icw - sk, a1 = fx + xmax * S.icw + sk;
        double b0 = fy + ymin * S.ich - sk, b1 = fy + ymax * S.ich + sk;
        a0 -= 1e-9 * (1.0 + fabs(a0));
        a1 += 1e-9 * (1.0 + fabs(a1));
        b0 -= 1e-9 * (1.0 + fabs(b0));
        b1 += 1e-9 * (1.0 + fabs(b1));
        lx = (int)fmax(floor(a0), -1e8);
        hx = (int)fmin(floor(a1), 1e8);
        ly = (int)fmax(floor(b0), -1e8);
        hy = (int)fmin(floor(b1), 1e8);
        return true;
    }

    // General box: the same in cell units.  A circle (c, rc) maps to an ellipse in cell
    // coordinates, centred at g c, whose bounding box spans rc times the row norms of g.
    __device__ bool need_rect_gen(double fx, double fy, int &lx, int &hx, int &ly, int &hy)
    {
        double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
        T mx = (T)0;
        bool finite = true;
        for (int k = 0; k < m; ++k) {
            E4 e = R.edge(k);
            double cx, cy, rc;
            mx = e.w > mx ? e.w : mx;
            finite &= e.w < PR::inf();
            if (e.w < PR::inf()) {
                cx = 0.5 * (double)e.x;
                cy = 0.5 * (double)e.y;
                rc = (double)e.w;
            } else {
                int ia = R.idx(k), ib = R.idx(k + 1 == m ? 0 : k + 1);
                double4 c = circle64g(A.pos, p, Sg, ia, ib);
                if (!(c.w < Prec<double>::inf())) {
                    minimage = true;
                    return false;
                }
                cx = 0.5 * c.x;
                cy = 0.5 * c.y;
                rc = c.w;
            }
            const double uc = S.g11 * cx + S.g12 * cy, vc = S.g21 * cx + S.g22 * cy;
            const double hu = rc * S.gnx, hv = rc * S.gny;
            umin = fmin(umin, uc - hu);
            umax = fmax(umax, uc + hu);
            vmin = fmin(vmin, vc - hv);
            vmax = fmax(vmax, vc + hv);
        }
        if (finite) r2max = r2_of(mx);
        // fractional offsets are unique within half the box per axis (hxs, hys cells)
        minimage = umin < -S.hxs || umax > S.hxs || vmin < -S.hys || vmax > S.hys;
        const double sk = A.skin ? (double)*A.skin : 0.0;
        double a0 = fx + umin - sk, a1 = fx + umax + sk;
        double b0 = fy + vmin - sk, b1 = fy + vmax + sk;
        a0 -= 1e-9 * (1.0 + fabs(a0));
        a1 += 1e-9 * (1.0 + fabs(a1));
        b0 -= 1e-9 * (1.0 + fabs(b0));
        b1 += 1e-9 * (1.0 + fabs(b1));
        lx = (int)fmax(floor(a0), -1e8);
        hx = (int)fmin(floor(a1), 1e8);
        ly = (int)fmax(floor(b0), -1e8);
        hy = (int)fmin(floor(b1), 1e8);
        return true;
    }

    // Whether the cell (rx, ry) (relative to the own cell) may hold a point strictly inside
    // some edge circle: its rectangle, widened by a margin far above the rounding of cell
    // indices and offsets, meets a disc (c~, rc) that contains the exact circle.  Cells
    // across the minimum-image seam are always reached.  A cell not reached stays so: the
    // union of the circles through p of a star-shaped ring only shrinks under insertion (a
    // disc through p centred in the convex Voronoi cell lies in the union of the discs centred
    // at the cell's vertices, because d - c, |d - c|^2 - |p - c|^2 is affine in c).
    __device__ bool cell_reached(int rx, int ry, double fx, double fy)
    {
        return rect_reached(rx, rx, ry, ry, fx, fy);
    }
    // the same for the cells [rx0, rx1] x [ry0, ry1] together
    __device__ bool rect_reached(int rx0, int rx1, int ry0, int ry1, double fx, double fy)
    {
        if (GEN) return rect_reached_gen(rx0, rx1, ry0, ry1, fx, fy);
        const double mg = 1e-9;
        const double sk = A.skin ? (double)*A.skin : 0.0;   // see need_rect
        double a0 = (double)rx0 - fx - sk, a1 = (double)rx1 - fx + 1.0 + sk;
        double b0 = (double)ry0 - fy - sk, b1 = (double)ry1 - fy + 1.0 + sk;
        a0 = (a0 - mg * (1.0 + fabs(a0))) * S.cw;
        a1 = (a1 + mg * (1.0 + fabs(a1))) * S.cw;
        b0 = (b0 - mg * (1.0 + fabs(b0))) * S.ch;
        b1 = (b1 + mg * (1.0 + fabs(b1))) * S.ch;
        if (a0 < -S.hLx || a1 > S.hLx || b0 < -S.hLy || b1 > S.hLy) return true;
        for (int k = 0; k < m; ++k) {
            E4 e = R.edge(k);
            if (!(e.w < PR::inf())) return true;
            double cx = 0.5 * (double)e.x, cy = 0.5 * (double)e.y, rc = (double)e.w * (1.0 + mg);
            double dx = fmax(fmax(a0 - cx, cx - a1), 0.0), dy = fmax(fmax(b0 - cy, cy - b1), 0.0);
            if (dx * dx + dy * dy <= rc * rc) return true;
        }
        return false;
    }
    // general box: the cells against each circle's ellipse bounding box in cell units (a
    // superset of the ellipse, so a cell judged unreached is unreached)
    __device__ bool rect_reached_gen(int rx0, int rx1, int ry0, int ry1, double fx, double fy)
    {
        const double mg = 1e-9;
        const double sk = A.skin ? (double)*A.skin : 0.0;
        double a0 = (double)rx0 - fx - sk, a1 = (double)rx1 - fx + 1.0 + sk;
        double b0 = (double)ry0 - fy - sk, b1 = (double)ry1 - fy + 1.0 + sk;
        a0 -= mg * (1.0 + fabs(a0));
        a1 += mg * (1.0 + fabs(a1));
        b0 -= mg * (1.0 + fabs(b0));
        b1 += mg * (1.0 + fabs(b1));
        if (a0 < -S.hxs || a1 > S.hxs || b0 < -S.hys || b1 > S.hys) return true;
        for (int k = 0; k < m; ++k) {
            E4 e = R.edge(k);
            if (!(e.w < PR::inf())) return true;
            const double cx = 0.5 * (double)e.x, cy = 0.5 * (double)e.y, rc = (double)e.w * (1.0 + mg);
            const double uc = S.g11 * cx + S.g12 * cy, vc = S.g21 * cx + S.g22 * cy;
            const double hu = rc * S.gnx, hv = rc * S.gny;
            if (uc + hu >= a0 && uc - hu <= a1 && vc + hv >= b0 && vc - hv <= b1) return true;
        }
        return false;
    }

    // Called by every lane of the warp (warp votes inside); `active` false for lanes
    // without a point.  Returns R_OK / error for active lanes.
    __device__ int run(bool active)
    {
        init();
        const double2 fp = cell_pos<GEN>(S, p);
        const double fx = fp.x - (double)ocx, fy = fp.y - (double)ocy;
        int x0 = 0, x1 = 0, y0 = 0, y1 = 0;
        const int max_phase = S.xsize + S.ysize + 8;
        bool done = !active;
        int status = R_OK;
        // global builds whose warp sees only sparse own cells scan the whole 3x3 block in the
        // first phase: one lockstep phase in place of two, the own cell's being short and
        // unevenly filled across the lanes (4M uniform points: 6.00 -> 5.79 ms; the choice is
        // per warp because lanes in different first phases diverge, and repair rounds keep
        // the own cell first: their rebuild rounds ran 2% slower with it)
        bool sparse = true;
        if (CAND == 0 && active) {
            const int c0 = S.cell_base + ocy * S.xsize + ocx;
            sparse = S.xsize >= 3 && S.ysize >= 3 && __ldg(&A.cstart[c0 + 1]) - __ldg(&A.cstart[c0]) <= BLOCK_FIRST_MAX;
        }
        const bool block0 = CAND == 0 && __all_sync(0xffffffffu, sparse);
        for (int phase = 0;; ++phase) {
            bool live = !done && status == R_OK;
            int gx0 = x0, gx1 = x1, gy0 = y0, gy1 = y1;
            if (live && phase >= max_phase) {
                done = true;
                live = false;
            }
            // every phase after the own cell grows towards the cells the circles reach (one
            // per side): a ring that still holds virtual corners takes the whole 3x3 block next,
            // a ring whose circles already lie inside the own cell (dense clusters) stops there
            if (live && phase >= 1) {
                int lx, hx, ly, hy;
                if (!need_rect(fx, fy, lx, hx, ly, hy)) {
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
            if (phase == 0 && block0) {
                gx0 = gy0 = -1;
                gx1 = gy1 = 1;
            }
            int r = scan(growth(x0, x1, y0, y1, gx0, gx1, gy0, gy1, phase == 0 && !block0, phase == 0 && block0),
                         live);
            if (live) {
                if (r != R_OK) status = r;
                // over the work budget: the warp-per-point kernel takes the point over
                if (!EXACT && status == R_OK && R.work() > A.work_budget) status = R_HEAVY;
                x0 = gx0; x1 = gx1; y0 = gy0; y1 = gy1;
            }
            if (__all_sync(0xffffffffu, done || status != R_OK)) break;
        }
        if (!active) return R_OK;
        if (status != R_OK) return status;
        for (int k = 0; k < m; ++k)
            if (R.idx(k) < 0) return R_UNBOUNDED;
        if (minimage) atomicOr(&A.st->err_flags, EF_MINIMAGE);
        return R_OK;
    }
};

// ------------------------------------------------------------- output + repair bookkeeping
__device__ __forceinline__ void enqueue_next(const RingArgs &A, int ebase, int ep, int j)
{
    if (atomicMax(&A.mark[j], ep + 1) < ebase) A.next_list[atomicAdd(A.next_count, 1)] = j;
}

template <class Ring>
__device__ void finish(const RingArgs &A, int pid, Ring &R, int m, int &maxr)
{
    const int ebase = A.repair ? *A.epoch_ptr + 1 : 0;
    const int ep = ebase + A.round;
    maxr = max(maxr, m);
    int *row = A.tri + (size_t)pid * A.stride;
    if (A.repair && m <= RR) {
        // consistency of the rebuilt ring with the rings it touches (see enqueue rules in
        // dgt_api.cu: points rebuilt in this call are exact; an untouched point must either
        // list pid with the matching neighbours on both sides or be rebuilt too).  Register
        // form: the old row, the neighbours' marks and ring lengths are loaded at once, each
        // neighbour row with one vector load.
        const int om = A.nn[pid];
        Ring16 old, nb;
        row_load(row, A.stride, old);
#pragma unroll
        for (int k = 0; k < RR; ++k) nb.r[k] = k < m ? R.idx(k) : -1;
        int mk[RR], mn[RR];
#pragma unroll
        for (int k = 0; k < RR; ++k) {
            mk[k] = k < m ? A.mark[nb.r[k]] : ebase;
            mn[k] = k < m ? A.nn[nb.r[k]] : 0;
        }
        if (om >= 1 && om <= min(A.stride, RR)) {
#pragma unroll
            for (int k = 0; k < RR; ++k) {
                const int o = old.r[k];
                bool kept = k >= om;
#pragma unroll
                for (int t = 0; t < RR; ++t) kept |= (t < m && nb.r[t] == o);
                if (!kept && o >= 0 && o < A.npoints) enqueue_next(A, ebase, ep, o);
            }
        } else if (om >= 1 && om <= A.stride) {
            for (int k = 0; k < om; ++k) {
                const int o = row[k];
                bool kept = false;
                for (int t = 0; t < m; ++t) kept |= (R.idx(t) == o);
                if (!kept && o >= 0 && o < A.npoints) enqueue_next(A, ebase, ep, o);
            }
        }
#pragma unroll
        for (int k = 0; k < RR; ++k) {
            if (k >= m || mk[k] >= ebase) continue;
            const int pred = k == 0 ? R.idx(m - 1) : nb.r[k > 0 ? k - 1 : 0];
            const int succ = k + 1 < m ? nb.r[k + 1 < RR ? k + 1 : 0] : nb.r[0];
            bool ok = mn[k] >= 3 && mn[k] <= min(A.stride, RR);
            if (ok) {
                Ring16 rn;
                row_load(A.tri + (size_t)nb.r[k] * A.stride, A.stride, rn);
                int pr, sc;
                ok = ring_find(rn, mn[k], pid, pr, sc) >= 0 && pr == succ && sc == pred;
            } else if (mn[k] >= 3 && mn[k] <= A.stride) {
                const int *rr = A.tri + (size_t)nb.r[k] * A.stride;
                const int l = mn[k];
                int pos = -1;
                for (int t = 0; t < l; ++t)
                    if (rr[t] == pid) pos = t;
                ok = pos >= 0 && rr[pos == 0 ? l - 1 : pos - 1] == succ && rr[pos + 1 == l ? 0 : pos + 1] == pred;
            }
            if (!ok) enqueue_next(A, ebase, ep, nb.r[k]);
        }
    } else if (A.repair) {
        int om = A.nn[pid];
        if (om >= 1 && om <= A.stride) {
            for (int k = 0; k < om; ++k) {
                int o = row[k];
                bool kept = false;
                for (int t = 0; t < m; ++t) kept |= (R.idx(t) == o);
                if (!kept && o >= 0 && o < A.npoints) enqueue_next(A, ebase, ep, o);
            }
        }
        for (int k = 0; k < m; ++k) {
            int nb = R.idx(k);
            if (A.mark[nb] >= ebase) continue;
            int pred = R.idx(k == 0 ? m - 1 : k - 1), succ = R.idx(k + 1 == m ? 0 : k + 1);
            int mn = A.nn[nb];
            bool ok = (mn >= 3 && mn <= A.stride);
            if (ok) {
                const int *rn = A.tri + (size_t)nb * A.stride;
                int pos = -1;
                for (int t = 0; t < mn; ++t)
                    if (rn[t] == pid) pos = t;
                ok = pos >= 0 && rn[pos == 0 ? mn - 1 : pos - 1] == succ && rn[pos + 1 == mn ? 0 : pos + 1] == pred;
            }
            if (!ok) enqueue_next(A, ebase, ep, nb);
        }
    }
    if (m > A.stride) {
        atomicMax(&A.st->need_stride, m);
        A.nn[pid] = 0;   // row left unwritten: mark the ring invalid
        return;
    }
    int best = 0, bv = R.idx(0);
    for (int k = 1; k < m; ++k) {
        int v = R.idx(k);
        if (v < bv) { bv = v; best = k; }
    }
    for (int k = 0; k < m; ++k) {
        int src = best + k;
        if (src >= m) src -= m;
        row[k] = R.idx(src);
    }
    A.nn[pid] = m;
}

__device__ __forceinline__ void flush_counters(const RingArgs &A, const Ctr &c, unsigned pts, int maxr)
{
    unsigned long long v[8] = { pts, c.cand, c.tests, c.u32, c.u64, c.ins, c.mism, c.cells };
    for (int i = 0; i < 8; ++i)
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
    for (int o = 16; o > 0; o >>= 1) maxr = max(maxr, __shfl_down_sync(0xffffffffu, maxr, o));
    if ((threadIdx.x & 31) == 0) {
        if (v[0]) atomicAdd(&A.st->points, v[0]);
        if (v[1]) atomicAdd(&A.st->candidates, v[1]);
        if (v[2]) atomicAdd(&A.st->tests, v[2]);
        if (v[3]) atomicAdd(&A.st->f32_undecided, v[3]);
        if (v[4]) atomicAdd(&A.st->f64_undecided, v[4]);
        if (v[5]) atomicAdd(&A.st->insertions, v[5]);
        if (v[6]) atomicAdd(&A.st->mismatches, v[6]);
        if (v[7]) atomicAdd(&A.st->cells, v[7]);
        if (maxr > 0) atomicMax(&A.st->max_ring, maxr);
    }
}

__device__ __forceinline__ int item_count(const RingArgs &A)
{
    if (!A.worklist) return A.n_items;
    int c = *A.worklist_count;
    return c < A.n_items ? c : A.n_items;
}


}  // namespace dgt

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
__device__ __noinline__ int check64(const double2 *pos, double2 p, double Lx, double hLx, double Ly, double hLy,
                                    float V, int ia, int ib, double dx, double dy, int inside)
{
    double2 a = off64(pos, p, Lx, hLx, Ly, hLy, V, ia), b = off64(pos, p, Lx, hLx, Ly, hLy, V, ib);
    int r = incircle64(a.x, a.y, b.x, b.y, dx, dy);
    return (inside && r < 0) || (!inside && r > 0) ? 1 : 0;
}

// circle of edge (ia, ib) in double (make_circ layout)
__device__ __noinline__ double4 circle64(const double2 *pos, double2 p, double Lx, double hLx, double Ly,
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
__device__ __noinline__ int check64g(const double2 *pos, double2 p, const SetDesc *S, int ia, int ib, double dx,
                                     double dy, int inside)
{
    double2 a = off64g(pos, p, S, ia), b = off64g(pos, p, S, ib);
    int r = incircle64(a.x, a.y, b.x, b.y, dx, dy);
    return (inside && r < 0) || (!inside && r > 0) ? 1 : 0;
}
__device__ __noinline__ double4 circle64g(const double2 *pos, double2 p, const SetDesc *S, int ia, int ib)
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
template <typename T, bool EXACT, class Ring, class C = Ctr, int CAND = 2, bool GEN = false>
struct Builder {
    static constexpr bool general = GEN;
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
        mask = 0;
        if (sl == slot) return R_OK;
        // repair calls read candidates through the index: the cell-order copy may be older
        // than the positions (cell lists kept from the last binning)
        const bool by_index = CAND == 1 || (CAND == 2 && A.cand_by_index);
        double2 q = by_index ? __ldg(&A.pos[__ldg(&A.sidx[sl])]) : __ldg(&A.spos[sl]);
        // general box: the matrices are read through the descriptor in global memory (L1
        // hits) rather than held in registers across the scan
        double2 d64 = GEN ? gen_off(q, p, *Sg)
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
        bool own;
    };
    __device__ __forceinline__ static Growth growth(int x0, int x1, int y0, int y1, int nx0, int nx1, int ny0,
                                                    int ny1, bool own)
    {
        Growth g{ x0, x1, y0, y1, nx0, nx1, ny0, ny1, 0, 0, 0, 0, own };
        if (own) return g;
        g.nl = nx0 < x0 ? (y1 - y0 + 1) : 0;
        g.nr = nx1 > x1 ? (y1 - y0 + 1) : 0;
        g.nb = ny0 < y0 ? (nx1 - nx0 + 1) : 0;
        g.nt = ny1 > y1 ? (nx1 - nx0 + 1) : 0;
        return g;
    }
    __device__ __forceinline__ static void growth_cell(const Growth &g, int ci, int &rx, int &ry)
    {
        if (g.own) { rx = 0; ry = 0; return; }
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
        const int ncell = !live ? 0 : (g.own ? 1 : g.nl + g.nr + g.nb + g.nt);
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
        for (int phase = 0;; ++phase) {
            bool live = !done && status == R_OK;
            int gx0 = x0, gx1 = x1, gy0 = y0, gy1 = y1;
            if (live && phase >= max_phase) {
                done = true;
                live = false;
            }
            if (live && phase == 1) {
                refresh_r2max();   // after the own cell's insertions
                // the 3x3 block (fewer columns / rows on grids narrower than 3 cells)
                gx0 = S.xsize >= 3 ? -1 : 0;
                gx1 = S.xsize >= 2 ? 1 : 0;
                gy0 = S.ysize >= 3 ? -1 : 0;
                gy1 = S.ysize >= 2 ? 1 : 0;
            } else if (live && phase > 1) {
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
            int r = scan(growth(x0, x1, y0, y1, gx0, gx1, gy0, gy1, phase == 0), live);
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
                slot = t;
                pid = __ldg(&A.sidx[t]);
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
// filter, float64 recheck, exact residue, 64 entries), take 32 new cells at a time (dropping empty occupancy
// blocks and cells that no current circle reaches) and 32 candidates at a time.  One lane inserts; lanes whose
// candidates conflicted test them again against the new ring (a candidate outside every
// circle stays outside, see cell_reached).  The scanned rectangle grows one cell per side
// while the ring keeps changing, by half its extent while virtual corners are left, and
// straight to the circles' cells once a layer changed nothing.
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
    int status = R_OK;
    const int max_phase = S.xsize + S.ysize + 8;

    // one candidate per lane (have): classify all, then insert the conflicting ones one at a
    // time (the others re-test against each new ring)
    auto settle = [&](int sl, bool have) {
        V2 d = B::PR::mk2(0, 0);
        Mask mask = 0;
        if (have) b.classify(sl, d, mask);
        unsigned want = __ballot_sync(0xffffffffu, have && mask != 0);
        while (want) {
            const int leader = __ffs(want) - 1;
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
            const bool again = ((want >> lane) & 1u) && lane != leader;
            mask = 0;
            if (again) b.classify(sl, d, mask);
            want = __ballot_sync(0xffffffffu, again && mask != 0);
        }
    };
    // every candidate of the cells [xa, xb] x [ya, yb] (relative to the own cell): 32 cells
    // at a time, one per lane (empty occupancy blocks dropped, and with `prune` the cells no
    // current circle reaches), then their candidates 32 at a time
    auto scan_cells = [&](int xa, int xb, int ya, int yb, bool prune) {
        const int w = xb - xa + 1, ncell = w * (yb - ya + 1);
        for (int cb = 0; cb < ncell && status == R_OK; cb += 32) {
            const int ci = cb + lane;
            int start = 0, cnt = 0;
            if (ci < ncell) {
                const int rx = xa + ci % w, ry = ya + ci / w;
                const int cx = wrapi(b.ocx + rx, S.xsize), cy = wrapi(b.ocy + ry, S.ysize);
                const int blk = S.block_base + (cy >> BLOCK_SHIFT) * S.bxsize + (cx >> BLOCK_SHIFT);
                if (__ldg(&A.bcount[blk]) != 0 && (!prune || b.cell_reached(rx, ry, fx, fy))) {
                    const int c = S.cell_base + cy * S.xsize + cx;
                    start = __ldg(&A.cstart[c]);
                    cnt = __ldg(&A.cstart[c + 1]) - start;
                    b.ctr.add_cells();
                }
            }
            int incl = cnt;
            for (int o = 1; o < 32; o <<= 1) {
                int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31), excl = incl - cnt;
            for (int j0 = 0; j0 < total && status == R_OK; j0 += 32) {
                const int j = j0 + lane;
                int o = 0;   // the last lane whose cell range starts at or before j
                for (int step = 16; step > 0; step >>= 1) {
                    int e = __shfl_sync(0xffffffffu, excl, o + step);
                    if (e <= j) o += step;
                }
                const int sl = __shfl_sync(0xffffffffu, start, o) + j - __shfl_sync(0xffffffffu, excl, o);
                settle(sl, j < total);
            }
        }
    };

    for (int phase = 0; status == R_OK && phase < max_phase; ++phase) {
        int nx0 = x0, nx1 = x1, ny0 = y0, ny1 = y1;
        if (phase == 1) {
            b.refresh_r2max();   // after the own cell's insertions (same value on every lane)
            nx0 = S.xsize >= 3 ? -1 : 0;
            nx1 = S.xsize >= 2 ? 1 : 0;
            ny0 = S.ysize >= 3 ? -1 : 0;
            ny1 = S.ysize >= 2 ? 1 : 0;
        } else if (phase > 1) {
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
            if (phase < 2 || sw * sh <= 512) {
                scan_cells(sxa[q], sxb[q], sya[q], syb[q], phase >= 2);
                continue;
            }
            // a large strip: 8 x 8 tiles first, one per lane; a tile is scanned cell by cell
            // only when one of the occupancy blocks it touches holds points and its rectangle
            // meets a current circle (empty space costs one test per tile, not per cell)
            const int tw = (sw + 7) >> 3, th = (sh + 7) >> 3, ntile = tw * th;
            for (int tb = 0; tb < ntile && status == R_OK; tb += 32) {
                const int ti = tb + lane;
                int ta = 0, tbx = -1, tc = 0, td = -1;
                bool live = false;
                if (ti < ntile) {
                    // nearest tiles first: the left strip from its right edge, the bottom strip
                    // from its top edge (the others start next to the old rectangle already)
                    const int ix = q == 0 ? tw - 1 - ti % tw : ti % tw, iy = q == 2 ? th - 1 - ti / tw : ti / tw;
                    ta = sxa[q] + ix * 8;
                    tbx = min(ta + 7, sxb[q]);
                    tc = sya[q] + iy * 8;
                    td = min(tc + 7, syb[q]);
                    // occupancy of the (up to 3 x 3) blocks the tile touches
                    for (int xs = ta; xs <= tbx && !live;) {
                        const int ax = wrapi(b.ocx + xs, S.xsize), bx = ax >> BLOCK_SHIFT;
                        const int xe = xs + min((bx + 1) << BLOCK_SHIFT, S.xsize) - ax;   // next block's first x
                        for (int ys = tc; ys <= td && !live;) {
                            const int ay = wrapi(b.ocy + ys, S.ysize), by = ay >> BLOCK_SHIFT;
                            live = __ldg(&A.bcount[S.block_base + by * S.bxsize + bx]) != 0;
                            ys += min((by + 1) << BLOCK_SHIFT, S.ysize) - ay;
                        }
                        xs = xe;
                    }
                    live = live && b.rect_reached(ta, tbx, tc, td, fx, fy);
                }
                unsigned todo = __ballot_sync(0xffffffffu, live);
                while (todo && status == R_OK) {
                    const int src = __ffs(todo) - 1;
                    todo &= todo - 1;
                    scan_cells(__shfl_sync(0xffffffffu, ta, src), __shfl_sync(0xffffffffu, tbx, src),
                               __shfl_sync(0xffffffffu, tc, src), __shfl_sync(0xffffffffu, td, src), true);
                }
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

// kernel shapes the autotuner chooses from: (ring capacity on chip, threads per block)
// index 0 is the default
static const int kShapeCap[KERNEL_SHAPES] = { 14, 12, 16, 14, 12 };
static const int kShapeBlock[KERNEL_SHAPES] = { 64, 64, 64, 32, 32 };

int kernel_shape_cap(int shape) { return (shape >= 0 && shape < KERNEL_SHAPES) ? kShapeCap[shape] : -1; }
int kernel_shape_block(int shape) { return (shape >= 0 && shape < KERNEL_SHAPES) ? kShapeBlock[shape] : -1; }

cudaError_t launch_build(const RingArgs &a, int mode, int sms, int shape, cudaStream_t s)
{
    if (a.n_items <= 0) return cudaSuccess;
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

__global__ void k_call_end(DevCtl *ctl, DevStatus *st, int rounds)
{
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

cudaError_t launch_call_end(DevCtl *ctl, DevStatus *st, int rounds, cudaStream_t s)
{
    k_call_end<<<1, 1, 0, s>>>(ctl, st, rounds);
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

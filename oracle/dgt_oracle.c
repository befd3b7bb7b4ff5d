/*
 * dgt_oracle.c -- CPU ORACLE (test infrastructure only).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this file's
 * library (oracle/liboracle.so).  It is the checker, never the product path.
 *
 * Part A restates the reference's CPU path for the hot path in plain C, same arithmetic in
 * the same order, so its raw output (rings including their start index) can be compared
 * bit-for-bit with the reference itself (oracle/_ref):
 *   - bucket grid:   src/utilities/cellListGPU.cpp:97-117 (setGridSize) and :289-330
 *                    (compute(points): index-order fill, Nmax growth)
 *   - box geometry:  src/utilities/periodicBoundaries.h:131-152 (putInBoxReal),
 *                    :154-179 (minDist, square box branch)
 *   - circumcentre:  inc/functions.h:33-42 (Circumcenter with the origin as third point)
 *   - seed pass:     src/model/DelaunayGPU.cu:318-608 (virtual_voronoi_calc_function)
 *   - refine pass:   src/model/DelaunayGPU.cu:680-943 (get_oneRing_function, host branch)
 *   - triangles:     src/model/DelaunayGPU.cpp:673-705 (getCircumcirclesCPU)
 *   - circle test:   src/model/DelaunayGPU.cu:192-284 (test_circumcircle_kernel_function)
 *   - orchestration: src/model/DelaunayGPU.cpp:118-157 (global), :567-602 + :87-115 (repair)
 * Deviations, each needed to keep the restatement memory-safe: bins are clamped to the grid
 * like the GPU fill (cellListGPU.cu:41-42); a ring that would outgrow the row stride stops
 * with an error code instead of writing past the row (the host branch has no guard,
 * DelaunayGPU.cu:911-918).
 *
 * Part B is an independent exact-arithmetic verifier of a periodic Delaunay triangulation:
 * expansion arithmetic after Shewchuk, "Adaptive Precision Floating-Point Arithmetic and
 * Fast Robust Geometric Predicates" (1997): two-sum, two-product with Veltkamp splitting,
 * zero-eliminating expansion growth and scaling.  Geometry is the minimum-image offset of
 * each point relative to the owning point, rounded once to double (dgt_offset below, the
 * same formula the CUDA kernels use); predicates on those offsets are exact.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double x, y; } d2;

/* ------------------------------------------------------------------------------------ */
/* Part A: restatement of the reference CPU path                                          */
/* ------------------------------------------------------------------------------------ */

#define REF_EPS 1e-18 /* THRESHOLD and EPSILON, inc/std_include.h:16-17 */

typedef struct {
    double Lx, Ly, hx, hy, ix, iy; /* box edge, half edge, inverse edge (square box) */
    int xsize, ysize, nmax, cells;
    double bs;                     /* bucket edge, Lx / xsize for both axes */
    unsigned int *csize;
    int *cidx;
} refctx;

static void ref_box_init(refctx *c, double Lx, double Ly)
{
    c->Lx = Lx; c->Ly = Ly;
    c->ix = 1. / Lx; c->iy = 1. / Ly;
    c->hx = Lx * 0.5; c->hy = Ly * 0.5;
}

/* periodicBoundaries::minDist, square branch */
static inline d2 ref_min_dist(const refctx *c, d2 a, d2 b)
{
    d2 r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    while (r.x < -c->hx) r.x += c->Lx;
    while (r.y < -c->hy) r.y += c->Ly;
    while (r.x > c->hx) r.x -= c->Lx;
    while (r.y > c->hy) r.y -= c->Ly;
    return r;
}

/* periodicBoundaries::putInBoxReal: to unit coordinates, wrap, back */
static inline void ref_put_in_box(const refctx *c, d2 *p)
{
    double vx = c->ix * p->x, vy = c->iy * p->y;
    while (vx < 0) vx += 1.0;
    while (vy < 0) vy += 1.0;
    while (vx >= 1.0) vx -= 1.0;
    while (vy >= 1.0) vy -= 1.0;
    p->x = c->Lx * vx;
    p->y = c->Ly * vy;
}

/* Circumcenter(x1, x2) of the circle through x1, x2 and the origin */
static inline d2 ref_cc(d2 a, d2 b)
{
    double an = a.x * a.x + a.y * a.y;
    double bn = b.x * b.x + b.y * b.y;
    double den = 0.5 / (a.x * b.y - a.y * b.x);
    d2 r;
    r.x = den * (an * b.y - a.y * bn);
    r.y = den * (a.x * bn - an * b.x);
    return r;
}

/* checkCW(pa, pb, pc): 0 when the signed area is positive, else 1 */
static inline int ref_cw(double ax, double ay, double bx, double by, double cx, double cy)
{
    return ((ax - bx) * (ay - cy) - (ay - by) * (ax - cx)) > 0 ? 0 : 1;
}

static inline int ref_pmod(int i, int n)
{
    int m = i % n;
    if (i < 0) m += n;
    return m;
}

/* square spiral (dd, cc) successor used by every cell scan of the reference */
static inline void ref_spiral_next(int *dd, int *cc)
{
    int d = *dd, e = *cc;
    if (abs(d) <= abs(e) && (d != e || d >= 0)) {
        if (e >= 0) d += 1; else d -= 1;
    } else {
        if (d >= 0) e -= 1; else e += 1;
    }
    *dd = d; *cc = e;
}

/* grid geometry + index-order fill; returns 0 or -1 on allocation failure */
static int ref_grid(refctx *c, const d2 *pts, int n, double a)
{
    c->xsize = (int)floor(c->Lx / a);
    if (c->xsize % 2 == 1) c->xsize += 1;
    c->ysize = (int)floor(c->Ly / a);
    if (c->ysize % 2 == 1) c->ysize += 1;
    c->bs = c->Lx / c->xsize;
    c->cells = c->xsize * c->ysize;
    c->nmax = 0;
    if (ceil(n / c->cells) + 1 > c->nmax) c->nmax = (int)ceil(n / c->cells) + 3;
    c->csize = NULL; c->cidx = NULL;
    for (;;) {
        free(c->csize); free(c->cidx);
        c->csize = (unsigned int *)calloc((size_t)c->cells, sizeof(unsigned int));
        c->cidx = (int *)calloc((size_t)c->cells * c->nmax, sizeof(int));
        if (!c->csize || !c->cidx) return -1;
        int again = 0;
        for (int i = 0; i < n; ++i) {
            if (again) continue;
            int ib = (int)floor(pts[i].x / c->bs);
            int jb = (int)floor(pts[i].y / c->bs);
            if (ib < 0) ib = 0;
            if (ib > c->xsize - 1) ib = c->xsize - 1;
            if (jb < 0) jb = 0;
            if (jb > c->ysize - 1) jb = c->ysize - 1;
            int bin = ib + c->xsize * jb;
            int off = (int)c->csize[bin];
            if (off < c->nmax) c->cidx[(size_t)bin * c->nmax + off] = i;
            else { if (off + 1 > c->nmax) c->nmax = off + 1; again = 1; }
            c->csize[bin]++;
        }
        if (!again) return 0;
    }
}

static void ref_grid_free(refctx *c)
{
    free(c->csize); free(c->cidx);
    c->csize = NULL; c->cidx = NULL;
}

/*
 * One insertion step shared by both passes: candidate at offset `disp` (index `cand`) has
 * been found to cut Voronoi vertex `jj`.  `w0` is where the vertex scan starts (0 in the
 * seed pass, jj in the refine pass) and `ccw_on_last` says whether the last vertex being cut
 * opens the removal run (always in the seed pass, only for jj==0 in the refine pass).
 * Returns 1 if the ring changed, 0 if nothing was cut, -1 if the row stride would overflow.
 * Same vertex bookkeeping as DelaunayGPU.cu:489-585 / :795-926.
 */
static int ref_cut_and_insert(d2 *P, d2 *Q, int *I, unsigned *psz, int stride, int cand, d2 disp,
                              double xx, double yy, int side_origin, int w0, int ccw_on_last)
{
    unsigned ps = *psz;
    int removeCW, removeCCW = 0, firstRemove = 1, j = -1, w, pp, m;
    unsigned removed = 0;
    int cy = ref_cw(0.5 * disp.x, 0.5 * disp.y, xx, yy, Q[ps - 1].x, Q[ps - 1].y);
    removeCW = cy;
    if (cy != side_origin) {
        j = (int)ps - 1;
        removed++;
        if (ccw_on_last) removeCCW = 1;
    }
    for (w = w0; w < (int)ps - 1; w++) {
        cy = ref_cw(0.5 * disp.x, 0.5 * disp.y, xx, yy, Q[w].x, Q[w].y);
        if (cy != side_origin) {
            if (!removeCCW) {
                if (j < 0) j = w;
                else if (j > w) j = w;
                removed++;
                removeCCW = 1;
            } else {
                if (!firstRemove) {
                    for (pp = w; pp < (int)ps - 1; pp++) Q[pp] = Q[pp + 1];
                    for (pp = w; pp < (int)ps - 1; pp++) P[pp] = P[pp + 1];
                    for (pp = w; pp < (int)ps - 1; pp++) I[pp] = I[pp + 1];
                    ps--;
                    if (j > w) j--;
                    w--;
                } else {
                    firstRemove = 0;
                }
                removed++;
            }
        } else {
            removeCCW = 0;
        }
    }
    if (removeCW != side_origin && removeCCW && !firstRemove) {
        ps--;
        if (j > w) j--;
    }
    if (removed == 0) { *psz = ps; return 0; }
    if (removed > 1) m = (int)((unsigned)(j + 2) % ps);
    else m = (int)((unsigned)(j + 1) % ps);
    d2 q1 = ref_cc(P[j], disp);
    d2 q2 = ref_cc(disp, P[m]);
    if (removed == 1) {
        ps++;
        if ((int)ps > stride) { *psz = ps - 1; return -1; }
        for (pp = (int)ps - 2; pp > j; pp--) {
            Q[pp + 1] = Q[pp];
            P[pp + 1] = P[pp];
            I[pp + 1] = I[pp];
        }
    }
    m = (int)((unsigned)(j + 1) % ps);
    Q[m] = q2;
    Q[j] = q1;
    P[m] = disp;
    I[m] = cand;
    *psz = ps;
    return 1;
}

/* bisector point of the segment origin->disp, with the THRESHOLD special cases */
static inline void ref_bisector(d2 disp, double *xx, double *yy)
{
    if (fabs(disp.y) > REF_EPS) {
        *yy = (disp.y * disp.y + disp.x * disp.x) / (2 * disp.y);
        *xx = 0;
    } else if (fabs(disp.y) < REF_EPS) {
        *yy = disp.y / 2 + 1;
        *xx = disp.x / 2;
    }
    if (fabs(disp.x) < REF_EPS) {
        *yy = disp.y / 2;
        *xx = disp.x / 2 + 1;
    }
}

/* both passes for point k; refine==0: seed pass, refine==1: refinement pass.
   Returns 0, or -1 if the ring outgrew the stride. */
static int ref_point_pass(const refctx *c, const d2 *pts, int k, d2 *Pall, d2 *Qall, int *Iall,
                          int *nn, int stride, int refine)
{
    d2 *P = Pall + (size_t)k * stride;
    d2 *Q = Qall + (size_t)k * stride;
    int *I = Iall + (size_t)k * stride;
    unsigned ps;
    double xx = 0, yy = 0;
    if (!refine) {
        double Lmax = (c->xsize * c->bs) * 0.5;
        double LL = Lmax / 1.414213562373095 - REF_EPS;
        ps = 4;
        P[0].x = LL;  P[0].y = LL;
        P[1].x = -LL; P[1].y = LL;
        P[2].x = -LL; P[2].y = -LL;
        P[3].x = LL;  P[3].y = -LL;
        for (int m = 0; m < 4; m++) {
            I[m] = -1;
            Q[m] = ref_cc(P[m], P[(m + 1) % 4]);
        }
    } else {
        ps = (unsigned)nn[k];
    }
    d2 v = pts[k];
    for (int jj = 0; jj < (int)ps; jj++) {
        d2 cq = Q[jj];
        double rad = sqrt(cq.x * cq.x + cq.y * cq.y);
        d2 home = v;
        if (refine) { home.x = v.x + cq.x; home.y = v.y + cq.y; }
        ref_put_in_box(c, &home);
        int hx = (int)floor(home.x / c->bs) % c->xsize;
        int hy = (int)floor(home.y / c->bs) % c->ysize;
        int R = (int)ceil(rad / c->bs);
        if (R > c->xsize / 2) R = c->xsize / 2;
        int W = 2 * R + 1;
        int dd = 0, cc = 0, hit = 0;
        for (int s = 0; s < W * W && !hit; ++s) {
            int cx = ref_pmod(hx + dd, c->xsize);
            int cy = ref_pmod(hy + cc, c->ysize);
            ref_spiral_next(&dd, &cc);
            int bin = cx + c->xsize * cy;
            unsigned cnt = c->csize[bin];
            for (unsigned a = 0; a < cnt; ++a) {
                int cand = c->cidx[(size_t)bin * c->nmax + a];
                if (cand == k || cand == I[0]) continue;
                int skip = 0;
                for (int t = jj; t < (int)ps; ++t)
                    if (cand == I[t]) skip = 1;
                if (skip) continue;
                double rr = rad * rad;
                d2 disp = ref_min_dist(c, pts[cand], v);
                d2 t1 = ref_min_dist(c, disp, cq);
                if (t1.x * t1.x + t1.y * t1.y > rr) continue;
                ref_bisector(disp, &xx, &yy);
                int side0 = ref_cw(0.5 * disp.x, 0.5 * disp.y, xx, yy, 0., 0.);
                if (side0 == ref_cw(0.5 * disp.x, 0.5 * disp.y, xx, yy, Q[jj].x, Q[jj].y)) continue;
                int r = ref_cut_and_insert(P, Q, I, &ps, stride, cand, disp, xx, yy, side0,
                                           refine ? jj : 0, refine ? (jj == 0) : 1);
                if (r < 0) { nn[k] = (int)ps; return -1; }
                if (r == 0) continue;
                hit = 1;
                break;
            }
        }
        if (hit && refine) jj--;
    }
    nn[k] = (int)ps;
    return 0;
}

/* runs one pass over all points (or those with fix[i] >= 0); returns #points that overflowed */
static int ref_pass_all(const refctx *c, const d2 *pts, int n, d2 *P, d2 *Q, int *I, int *nn, int stride,
                        int refine, const int *fix, int threads)
{
    int bad = 0;
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) reduction(+ : bad) schedule(dynamic, 256)
#endif
    for (int i = 0; i < n; ++i) {
        if (fix && fix[i] < 0) continue;
        if (ref_point_pass(c, pts, i, P, Q, I, nn, stride, refine) < 0) bad++;
    }
    (void)threads;
    return bad;
}

/* Global triangulation, reference CPU semantics.  tri: n*stride, nn: n.
   Returns the largest ring size, or -(#overflowing points) if the stride was too small,
   or -1000000000 on allocation failure. */
int orc_ref_global(const double *pts_, int n, double Lx, double Ly, double cell_size, int stride,
                   int threads, int *tri, int *nn)
{
    const d2 *pts = (const d2 *)pts_;
    refctx c;
    ref_box_init(&c, Lx, Ly);
    if (ref_grid(&c, pts, n, cell_size) != 0) return -1000000000;
    d2 *P = (d2 *)malloc(sizeof(d2) * (size_t)stride * n);
    d2 *Q = (d2 *)malloc(sizeof(d2) * (size_t)stride * n);
    if (!P || !Q) { free(P); free(Q); ref_grid_free(&c); return -1000000000; }
    int bad = ref_pass_all(&c, pts, n, P, Q, tri, nn, stride, 0, NULL, threads);
    if (!bad) bad = ref_pass_all(&c, pts, n, P, Q, tri, nn, stride, 1, NULL, threads);
    free(P); free(Q);
    ref_grid_free(&c);
    if (bad) return -bad;
    int mx = 0;
    for (int i = 0; i < n; ++i) if (nn[i] > mx) mx = nn[i];
    return mx;
}

/* circle test for one triangle (x = owner): flags intruder and the triangle's vertices */
static void ref_test_triangle(const refctx *c, const d2 *pts, const int *tr, int *repair)
{
    d2 v = pts[tr[0]];
    d2 a = ref_min_dist(c, pts[tr[1]], v);
    d2 b = ref_min_dist(c, pts[tr[2]], v);
    d2 q = ref_cc(a, b);
    double rad = sqrt(q.x * q.x + q.y * q.y);
    d2 qb = { v.x + q.x, v.y + q.y };
    ref_put_in_box(c, &qb);
    int hx = (int)floor(qb.x / c->bs) % c->xsize;
    int hy = (int)floor(qb.y / c->bs) % c->ysize;
    int xy = c->xsize > c->ysize ? c->xsize : c->ysize;
    int R = (int)ceil(rad / c->bs);
    if (R > xy / 2) R = xy / 2;
    double r2 = rad * rad;
    int W = 2 * R + 1, dd = 0, cc = 0, bad = 0;
    for (int s = 0; s < W * W; ++s) {
        int cx = ref_pmod(hx + dd, c->xsize);
        int cy = ref_pmod(hy + cc, c->ysize);
        ref_spiral_next(&dd, &cc);
        int bin = cx + c->xsize * cy;
        for (unsigned p = 0; p < c->csize[bin]; ++p) {
            int id = c->cidx[(size_t)bin * c->nmax + p];
            if (id == tr[0] || id == tr[1] || id == tr[2]) continue;
            d2 t = ref_min_dist(c, pts[id], v);
            t.x = t.x - q.x;
            t.y = t.y - q.y;
            if (t.x * t.x + t.y * t.y < r2) {
                repair[id] = id;
                bad = 1;
            }
            if (bad) break;
        }
        if (bad) break;
    }
    if (bad) {
        repair[tr[0]] = tr[0];
        repair[tr[1]] = tr[1];
        repair[tr[2]] = tr[2];
    }
}

/* Test-and-repair, reference CPU semantics, in place on (tri, nn) with stride.
   repair_out: n ints of flags (-1 or own index).  Returns #triangles enumerated, -1 if more
   than 2n, -2 if a ring overflowed during repair, -3 on allocation failure. */
int orc_ref_test_and_repair(const double *pts_, int n, double Lx, double Ly, double cell_size, int stride,
                            int threads, int *tri, int *nn, int *repair_out)
{
    const d2 *pts = (const d2 *)pts_;
    int *tris = (int *)malloc(sizeof(int) * 3 * (size_t)2 * n);
    if (!tris) return -3;
    int nt = 0;
    for (int i = 0; i < n; ++i) {
        int m = nn[i];
        int y = tri[(size_t)i * stride + m - 1];
        for (int k = 0; k < m; ++k) {
            int z = tri[(size_t)i * stride + k];
            if (i < y && i < z) {
                if (nt >= 2 * n) { free(tris); return -1; }
                tris[3 * nt] = i; tris[3 * nt + 1] = y; tris[3 * nt + 2] = z;
                nt++;
            }
            y = z;
        }
    }
    refctx c;
    ref_box_init(&c, Lx, Ly);
    if (ref_grid(&c, pts, n, cell_size) != 0) { free(tris); return -3; }
    for (int i = 0; i < n; ++i) repair_out[i] = -1;
    /* only the enumerated triangles are tested (the class path throws unless there are
       exactly 2n of them, DelaunayGPU.cpp:701-705) */
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 1024)
#endif
    for (int t = 0; t < nt; ++t) ref_test_triangle(&c, pts, tris + 3 * t, repair_out);
    free(tris);
    d2 *P = (d2 *)malloc(sizeof(d2) * (size_t)stride * n);
    d2 *Q = (d2 *)malloc(sizeof(d2) * (size_t)stride * n);
    if (!P || !Q) { free(P); free(Q); ref_grid_free(&c); return -3; }
    int bad = ref_pass_all(&c, pts, n, P, Q, tri, nn, stride, 0, repair_out, threads);
    if (!bad) bad = ref_pass_all(&c, pts, n, P, Q, tri, nn, stride, 1, repair_out, threads);
    free(P); free(Q);
    ref_grid_free(&c);
    return bad ? -2 : nt;
}

/* ------------------------------------------------------------------------------------ */
/* Part B: exact predicates and the Delaunay verifier                                    */
/* ------------------------------------------------------------------------------------ */

/* Minimum-image offset c - p rounded once: when the raw difference says the image across
   the boundary is nearer, the box edge is first taken off the coordinate that lies in the
   far half (an exact subtraction for coordinates in [L/2, 2L], Sterbenz), so the final
   subtraction is the only rounding. */
static inline double dgt_offset1(double c, double p, double L)
{
    double d = c - p;
    if (d > 0.5 * L) d = (c - L) - p;
    else if (d < -0.5 * L) d = c - (p - L);
    return d;
}

void orc_offset(const double *c, const double *p, double Lx, double Ly, double *out)
{
    out[0] = dgt_offset1(c[0], p[0], Lx);
    out[1] = dgt_offset1(c[1], p[1], Ly);
}

/* General periodic box (periodicBoundaries::setGeneral, src/utilities/periodicBoundaries.h:
   86-101): a point is M u for fractional coordinates u, M = {{x11, x12}, {x21, x22}} (box[0..3]
   = x11, x12, x21, x22).  The offset c - p goes to the image whose fractional offset lies in
   [-1/2, 1/2] per component, as periodicBoundaries::minDist does for a general box
   (:165-178): the integer lattice shift s = rint(M^-1 (c - p)) is chosen in fractional
   coordinates and l = M s is taken off c when positive, added to p otherwise, per axis.
   Every operation is written out (fma where the product is fused) so that the library's
   kernels, which perform the same steps, produce the same doubles. */
typedef struct {
    double m11, m12, m21, m22;
    double i11, i12, i21, i22;
} gbox;

static void gbox_init(gbox *g, const double *box)
{
    const double det = box[0] * box[3] - box[1] * box[2];
    g->m11 = box[0];
    g->m12 = box[1];
    g->m21 = box[2];
    g->m22 = box[3];
    g->i11 = box[3] / det;
    g->i12 = -box[1] / det;
    g->i21 = -box[2] / det;
    g->i22 = box[0] / det;
}

static inline double gen_off1(double c, double p, double l)
{
    return l >= 0.0 ? (c - l) - p : c - (p + l);
}

static inline d2 gen_offset(const gbox *g, d2 c, d2 p)
{
    const double dx = c.x - p.x, dy = c.y - p.y;
    const double su = rint(fma(g->i11, dx, g->i12 * dy));
    const double sv = rint(fma(g->i21, dx, g->i22 * dy));
    const double lx = fma(g->m11, su, g->m12 * sv);
    const double ly = fma(g->m21, su, g->m22 * sv);
    d2 r;
    r.x = gen_off1(c.x, p.x, lx);
    r.y = gen_off1(c.y, p.y, ly);
    return r;
}

void orc_offset_general(const double *c, const double *p, const double *box, double *out)
{
    gbox g;
    gbox_init(&g, box);
    d2 cc = { c[0], c[1] }, pp = { p[0], p[1] };
    d2 r = gen_offset(&g, cc, pp);
    out[0] = r.x;
    out[1] = r.y;
}

/* Lagrange-Gauss reduction of the basis (columns (box[0], box[2]) and (box[1], box[3])), the
   steps the library applies before using a general box */
void orc_reduce_basis(double *box)
{
    double ax = box[0], ay = box[2], bx = box[1], by = box[3];
    for (int it = 0; it < 64; ++it) {
        if (ax * ax + ay * ay > bx * bx + by * by) {
            double t = ax; ax = bx; bx = t;
            t = ay; ay = by; by = t;
        }
        const double mu = nearbyint((ax * bx + ay * by) / (ax * ax + ay * ay));
        if (mu == 0.0) break;
        bx -= mu * ax;
        by -= mu * ay;
    }
    box[0] = ax;
    box[2] = ay;
    box[1] = bx;
    box[3] = by;
}

#define SPLITTER 134217729.0 /* 2^27 + 1 */

static inline void two_sum(double a, double b, double *x, double *y)
{
    double s = a + b;
    double bv = s - a;
    double av = s - bv;
    *x = s;
    *y = (a - av) + (b - bv);
}

static inline void split(double a, double *hi, double *lo)
{
    double c = SPLITTER * a;
    double big = c - a;
    *hi = c - big;
    *lo = a - *hi;
}

static inline void two_prod(double a, double b, double *x, double *y)
{
    double p = a * b;
    double ah, al, bh, bl;
    split(a, &ah, &al);
    split(b, &bh, &bl);
    double e1 = p - ah * bh;
    double e2 = e1 - al * bh;
    double e3 = e2 - ah * bl;
    *x = p;
    *y = al * bl - e3;
}

/* h = e + b, zero-eliminating; e has elen nonoverlapping components in increasing order */
static int grow_expansion(int elen, const double *e, double b, double *h)
{
    double q = b, hh;
    int hi = 0;
    for (int i = 0; i < elen; i++) {
        two_sum(q, e[i], &q, &hh);
        if (hh != 0.0) h[hi++] = hh;
    }
    if (q != 0.0 || hi == 0) h[hi++] = q;
    return hi;
}

/* h = e + f (repeated growth; fine for the short expansions used here) */
static int expansion_sum(int elen, const double *e, int flen, const double *f, double *h)
{
    double tmp[512];
    int hl = elen;
    for (int i = 0; i < elen; i++) h[i] = e[i];
    for (int i = 0; i < flen; i++) {
        hl = grow_expansion(hl, h, f[i], tmp);
        for (int k = 0; k < hl; k++) h[k] = tmp[k];
    }
    return hl;
}

/* h = e * b, zero-eliminating */
static int scale_expansion(int elen, const double *e, double b, double *h)
{
    double q, sum, hh, p1, p0;
    int hi = 0;
    two_prod(e[0], b, &q, &hh);
    if (hh != 0.0) h[hi++] = hh;
    for (int i = 1; i < elen; i++) {
        two_prod(e[i], b, &p1, &p0);
        two_sum(q, p0, &sum, &hh);
        if (hh != 0.0) h[hi++] = hh;
        two_sum(p1, sum, &q, &hh);
        if (hh != 0.0) h[hi++] = hh;
    }
    if (q != 0.0 || hi == 0) h[hi++] = q;
    return hi;
}

/* h = e * f */
static int expansion_prod(int elen, const double *e, int flen, const double *f, double *h)
{
    double part[512], acc[512];
    int al = 1;
    acc[0] = 0.0;
    for (int i = 0; i < flen; i++) {
        int pl = scale_expansion(elen, e, f[i], part);
        al = expansion_sum(al, acc, pl, part, h);
        for (int k = 0; k < al; k++) acc[k] = h[k];
    }
    for (int k = 0; k < al; k++) h[k] = acc[k];
    return al;
}

static inline int expansion_sign(int len, const double *e)
{
    for (int i = len - 1; i >= 0; i--) {
        if (e[i] > 0) return 1;
        if (e[i] < 0) return -1;
    }
    return 0;
}

/* exact u*v - w*z as an expansion (<= 4 terms) */
static int exact_cross(double u, double v, double w, double z, double *h)
{
    double a1, a0, b1, b0, t[4];
    two_prod(u, v, &a1, &a0);
    two_prod(w, z, &b1, &b0);
    double pos[2] = { a0, a1 }, neg[2] = { -b0, -b1 };
    int l = expansion_sum(2, pos, 2, neg, t);
    for (int i = 0; i < l; i++) h[i] = t[i];
    return l;
}

/* exact u*u + v*v */
static int exact_norm2(double u, double v, double *h)
{
    double a1, a0, b1, b0;
    two_prod(u, u, &a1, &a0);
    two_prod(v, v, &b1, &b0);
    double e[2] = { a0, a1 }, f[2] = { b0, b1 };
    return expansion_sum(2, e, 2, f, h);
}

/* sign of orient(0, a, b) = a.x*b.y - a.y*b.x, exact */
int orc_orient0(const double *a, const double *b)
{
    double h[8];
    int l = exact_cross(a[0], b[1], a[1], b[0], h);
    return expansion_sign(l, h);
}

/* sign of the in-circle test of d against the circle through (0, a, b):
   +1 when d lies strictly inside the circle of a CCW triangle (0, a, b), exact.
   value = |a|^2 (d x b) + |b|^2 (a x d) + |d|^2 (b x a) */
int orc_incircle0(const double *a, const double *b, const double *d)
{
    double na[8], nb[8], nd[8], c1[8], c2[8], c3[8];
    double t1[512], t2[512], t3[512], s12[512], s[512];
    int lna = exact_norm2(a[0], a[1], na);
    int lnb = exact_norm2(b[0], b[1], nb);
    int lnd = exact_norm2(d[0], d[1], nd);
    int l1 = exact_cross(d[0], b[1], d[1], b[0], c1);
    int l2 = exact_cross(a[0], d[1], a[1], d[0], c2);
    int l3 = exact_cross(b[0], a[1], b[1], a[0], c3);
    int lt1 = expansion_prod(lna, na, l1, c1, t1);
    int lt2 = expansion_prod(lnb, nb, l2, c2, t2);
    int lt3 = expansion_prod(lnd, nd, l3, c3, t3);
    int l12 = expansion_sum(lt1, t1, lt2, t2, s12);
    int ls = expansion_sum(l12, s12, lt3, t3, s);
    return expansion_sign(ls, s);
}

/* Verifier report (filled by orc_verify). */
typedef struct {
    long long sum_deg;        /* expected 6n on the torus */
    long long bad_index;      /* out-of-range / self / duplicate entries */
    long long asym;           /* j in ring(i) but adjacency in ring(j) does not match */
    long long nonpositive;    /* fan triangles with orient <= 0 */
    long long winding;        /* rings that do not wind exactly once */
    long long not_local_dt;   /* spokes failing the exact local Delaunay test */
    long long circle_intruders; /* triangles whose circumcircle holds another point (global scan) */
    long long triangles;      /* triangles owned by their min index */
    int min_deg, max_deg;
} orc_report;

/* the box a verification runs in: rectangular (general == 0, Lx x Ly) or general (g) */
typedef struct {
    int general;
    double Lx, Ly;
    gbox g;
} vbox;

static inline d2 off_of(const d2 *pts, int c, int p, const vbox *B)
{
    if (B->general) return gen_offset(&B->g, pts[c], pts[p]);
    d2 r;
    r.x = dgt_offset1(pts[c].x, pts[p].x, B->Lx);
    r.y = dgt_offset1(pts[c].y, pts[p].y, B->Ly);
    return r;
}

/* bucket coordinates (cell units of a gx x gy grid) of a point: rectangular pts / L * g; a
   general box's fractional coordinates wrapped into [0, 1) times g */
static inline void bucket_pos(const vbox *B, d2 p, int gx, int gy, double *fx, double *fy)
{
    if (!B->general) {
        *fx = p.x / B->Lx * gx;
        *fy = p.y / B->Ly * gy;
        return;
    }
    double u = fma(B->g.i11, p.x, B->g.i12 * p.y), v = fma(B->g.i21, p.x, B->g.i22 * p.y);
    u -= floor(u);
    v -= floor(v);
    *fx = u * gx;
    *fy = v * gy;
}

static int verify_impl(const d2 *pts, int n, const vbox *B, const int *tri, const int *nn, int stride,
                       int global_scan, int threads, orc_report *rep);

/* Exact check that (tri, nn) is the periodic Delaunay triangulation of pts.  A triangulation
   whose rings are mutually consistent, whose fan triangles are all positively oriented and
   wind once, and whose every edge is locally Delaunay is the Delaunay triangulation
   (Lawson); with `global_scan` the circumcircle of every triangle is additionally checked
   against every point of the cells it overlaps.  Returns 0 when everything holds. */
int orc_verify(const double *pts_, int n, double Lx, double Ly, const int *tri, const int *nn, int stride,
               int global_scan, int threads, orc_report *rep)
{
    vbox B;
    memset(&B, 0, sizeof(B));
    B.Lx = Lx;
    B.Ly = Ly;
    return verify_impl((const d2 *)pts_, n, &B, tri, nn, stride, global_scan, threads, rep);
}

/* the same for a general periodic box (box_in[0..3] = x11, x12, x21, x22; see gen_offset),
   in its reduced basis (the same lattice; a reduced basis is left as it is) */
int orc_verify_general(const double *pts_, int n, const double *box_in, const int *tri, const int *nn,
                       int stride, int global_scan, int threads, orc_report *rep)
{
    double box[4] = { box_in[0], box_in[1], box_in[2], box_in[3] };
    orc_reduce_basis(box);
    vbox B;
    memset(&B, 0, sizeof(B));
    B.general = 1;
    gbox_init(&B.g, box);
    /* strip widths between opposite box edges, in place of Lx and Ly */
    const double area = fabs(box[0] * box[3] - box[1] * box[2]);
    B.Lx = area / hypot(box[1], box[3]);
    B.Ly = area / hypot(box[0], box[2]);
    return verify_impl((const d2 *)pts_, n, &B, tri, nn, stride, global_scan, threads, rep);
}

static int verify_impl(const d2 *pts, int n, const vbox *B, const int *tri, const int *nn, int stride,
                       int global_scan, int threads, orc_report *rep)
{
    const double Lx = B->Lx, Ly = B->Ly;
    memset(rep, 0, sizeof(*rep));
    rep->min_deg = 1 << 30;
    long long sdeg = 0, bidx = 0, asym = 0, npos = 0, wind = 0, nld = 0, ntri = 0, intr = 0;
    int mind = 1 << 30, maxd = 0;
    for (int i = 0; i < n; ++i) {
        int m = nn[i];
        sdeg += m;
        if (m < mind) mind = m;
        if (m > maxd) maxd = m;
    }
    /* bucket grid for the global scan: cell edge ~ mean spacing */
    int gx = (int)floor(Lx / sqrt(Lx * Ly / (n > 0 ? n : 1)));
    int gy = (int)floor(Ly / sqrt(Lx * Ly / (n > 0 ? n : 1)));
    if (gx < 1) gx = 1;
    if (gy < 1) gy = 1;
    int *cstart = NULL, *cpts = NULL;
    if (global_scan) {
        cstart = (int *)calloc((size_t)gx * gy + 1, sizeof(int));
        cpts = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        int *fill = (int *)calloc((size_t)gx * gy, sizeof(int));
        for (int i = 0; i < n; ++i) {
            double fx, fy;
            bucket_pos(B, pts[i], gx, gy, &fx, &fy);
            int cx = (int)floor(fx), cy = (int)floor(fy);
            cx = cx < 0 ? 0 : (cx >= gx ? gx - 1 : cx);
            cy = cy < 0 ? 0 : (cy >= gy ? gy - 1 : cy);
            cstart[cy * gx + cx + 1]++;
        }
        for (int c = 0; c < gx * gy; ++c) cstart[c + 1] += cstart[c];
        for (int i = 0; i < n; ++i) {
            double fx, fy;
            bucket_pos(B, pts[i], gx, gy, &fx, &fy);
            int cx = (int)floor(fx), cy = (int)floor(fy);
            cx = cx < 0 ? 0 : (cx >= gx ? gx - 1 : cx);
            cy = cy < 0 ? 0 : (cy >= gy ? gy - 1 : cy);
            int c = cy * gx + cx;
            cpts[cstart[c] + fill[c]++] = i;
        }
        free(fill);
    }
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 256) \
    reduction(+ : bidx, asym, npos, wind, nld, ntri, intr)
#endif
    for (int i = 0; i < n; ++i) {
        int m = nn[i];
        const int *r = tri + (size_t)i * stride;
        int ok = (m >= 3 && m <= stride);
        for (int k = 0; ok && k < m; ++k) {
            if (r[k] < 0 || r[k] >= n || r[k] == i) ok = 0;
            for (int t = 0; ok && t < k; ++t)
                if (r[t] == r[k]) ok = 0;
        }
        if (!ok) { bidx++; continue; }
        /* adjacency consistency: ring(j) holds ..., r[k+1], i, r[k-1], ... */
        for (int k = 0; k < m; ++k) {
            int j = r[k], nx = r[(k + 1) % m], pv = r[(k + m - 1) % m];
            int mj = nn[j];
            const int *rj = tri + (size_t)j * stride;
            int pos = -1;
            if (mj >= 1 && mj <= stride)
                for (int t = 0; t < mj; ++t)
                    if (rj[t] == i) { pos = t; break; }
            if (pos < 0 || rj[(pos + mj - 1) % mj] != nx || rj[(pos + 1) % mj] != pv) asym++;
        }
        /* orientation, winding, local Delaunay */
        d2 off[512];
        int mm = m < 512 ? m : 512;
        for (int k = 0; k < mm; ++k) off[k] = off_of(pts, r[k], i, B);
        int cross = 0, allpos = 1;
        for (int k = 0; k < mm; ++k) {
            d2 a = off[k], b = off[(k + 1) % mm];
            if (orc_orient0(&a.x, &b.x) <= 0) { npos++; allpos = 0; }
            if (a.y < 0 && b.y >= 0) cross++;
        }
        if (!allpos || cross != 1) wind++;
        for (int k = 0; k < mm; ++k) {
            d2 a = off[(k + mm - 1) % mm], b = off[k], d = off[(k + 1) % mm];
            if (orc_incircle0(&a.x, &b.x, &d.x) > 0) nld++;
        }
        /* triangles owned by their min index: global empty-circle scan */
        for (int k = 0; k < mm; ++k) {
            int y = r[(k + mm - 1) % mm], z = r[k];
            if (!(i < y && i < z)) continue;
            ntri++;
            if (!global_scan) continue;
            d2 a = off[(k + mm - 1) % mm], b = off[k];
            double den = 2.0 * (a.x * b.y - a.y * b.x);
            double na = a.x * a.x + a.y * a.y, nb = b.x * b.x + b.y * b.y;
            double qx = (na * b.y - nb * a.y) / den, qy = (nb * a.x - na * b.x) / den;
            double rad = sqrt(qx * qx + qy * qy);
            if (!(rad == rad) || rad > 0.25 * (Lx < Ly ? Lx : Ly)) rad = 0.25 * (Lx < Ly ? Lx : Ly);
            double marg = rad * 1e-6 + 1e-9;
            int x0, x1, y0, y1;
            if (!B->general) {
                double ax = pts[i].x + qx - rad - marg, bx = pts[i].x + qx + rad + marg;
                double ay = pts[i].y + qy - rad - marg, by = pts[i].y + qy + rad + marg;
                x0 = (int)floor(ax / Lx * gx);
                x1 = (int)floor(bx / Lx * gx);
                y0 = (int)floor(ay / Ly * gy);
                y1 = (int)floor(by / Ly * gy);
            } else {
                /* the circle's bounding box in bucket units: its centre's wrapped position,
                   half extents (rad + marg) times the rows of diag(gx, gy) M^-1 */
                d2 cen = { pts[i].x + qx, pts[i].y + qy };
                double fx, fy;
                bucket_pos(B, cen, gx, gy, &fx, &fy);
                const double hu = (rad + marg) * gx * hypot(B->g.i11, B->g.i12) * (1 + 1e-9) + 1e-9;
                const double hv = (rad + marg) * gy * hypot(B->g.i21, B->g.i22) * (1 + 1e-9) + 1e-9;
                x0 = (int)floor(fx - hu);
                x1 = (int)floor(fx + hu);
                y0 = (int)floor(fy - hv);
                y1 = (int)floor(fy + hv);
            }
            if (x1 - x0 + 1 > gx) { x0 = 0; x1 = gx - 1; }
            if (y1 - y0 + 1 > gy) { y0 = 0; y1 = gy - 1; }
            int found = 0;
            for (int cy = y0; cy <= y1 && !found; ++cy)
                for (int cx = x0; cx <= x1 && !found; ++cx) {
                    int wx = ((cx % gx) + gx) % gx, wy = ((cy % gy) + gy) % gy;
                    int c = wy * gx + wx;
                    for (int t = cstart[c]; t < cstart[c + 1]; ++t) {
                        int e = cpts[t];
                        if (e == i || e == y || e == z) continue;
                        d2 de = off_of(pts, e, i, B);
                        if (orc_incircle0(&a.x, &b.x, &de.x) > 0) { found = 1; break; }
                    }
                }
            if (found) intr++;
        }
    }
    free(cstart);
    free(cpts);
    rep->sum_deg = sdeg;
    rep->bad_index = bidx;
    rep->asym = asym;
    rep->nonpositive = npos;
    rep->winding = wind;
    rep->not_local_dt = nld;
    rep->circle_intruders = intr;
    rep->triangles = ntri;
    rep->min_deg = n > 0 ? mind : 0;
    rep->max_deg = maxd;
    int good = (sdeg == 6LL * n) && !bidx && !asym && !npos && !wind && !nld && !intr && ntri == 2LL * n;
    return good ? 0 : 1;
}

/* rotate every ring so that its smallest index comes first (the start a ring is emitted at
   is arbitrary; this is the canonical form rings are compared in) */
void orc_canonical_rotate(int *tri, const int *nn, int n, int stride)
{
    int tmp[1024];
    for (int i = 0; i < n; ++i) {
        int m = nn[i];
        if (m <= 1 || m > 1024 || m > stride) continue;
        int *r = tri + (size_t)i * stride;
        int best = 0;
        for (int k = 1; k < m; ++k)
            if (r[k] < r[best]) best = k;
        if (best == 0) continue;
        for (int k = 0; k < m; ++k) tmp[k] = r[(best + k) % m];
        memcpy(r, tmp, sizeof(int) * (size_t)m);
    }
}

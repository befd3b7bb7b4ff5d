// Geometric predicates of the one-ring construction.
//
// Geometry.  Every decision about point p is made on the minimum-image offsets of the other
// points relative to p, each rounded once to double (wrap_off).  All three decisions the
// reference makes with constructed circumcentres (distance test DelaunayGPU.cu:767-769,
// bisector side tests :789-790/:801/:814, triangle test :263-268) are, in exact arithmetic,
// the sign of one in-circle determinant with p at the origin:
//     inc0(a, b, d) = |a|^2 (d x b) + |b|^2 (a x d) + |d|^2 (b x a),
// positive iff d lies strictly inside the circle through (0, a, b) for CCW (0, a, b).
//
// Evaluation is staged:
//  1. float32 filter.  Each ring edge (a, b) stores its circumcentre c = cc(0, a, b) computed
//     in float32 from float32-rounded offsets plus a rigorous bound E >= |c~ - c| (c the exact
//     centre of the double offsets).  For a candidate d the test is s = 2 d.c - |d|^2
//     (s > 0 iff d strictly inside); |s~ - s| <= |d| Eb + 8u|d|^2 covers the rounding of d to
//     float32, the error in c~ and the arithmetic (derivation in make_circ).  Undecided when
//     |s~| is inside that bound.
//  2. float64 recheck of inc0 on the double offsets with the permanent bound 10u|P|.
//  3. exact sign by expansion arithmetic (Shewchuk 1997: two-sum, fma two-product,
//     zero-eliminating growth / scaling), only for what 2 leaves undecided.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace dgt {

template <typename T> struct Prec;
template <> struct Prec<float> {
    typedef float2 T2;
    typedef float4 T4;
    static __device__ __forceinline__ float u() { return 5.9604644775390625e-08f; }   // 2^-24
    static __device__ __forceinline__ float tiny() { return 1e-30f; }
    static __device__ __forceinline__ float inf() { return __int_as_float(0x7f800000); }
    static __device__ __forceinline__ float from64(double x) { return __double2float_rn(x); }
    static __device__ __forceinline__ T2 mk2(float x, float y) { return make_float2(x, y); }
    static __device__ __forceinline__ T4 mk4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
};
template <> struct Prec<double> {
    typedef double2 T2;
    typedef double4 T4;
    static __device__ __forceinline__ double u() { return 1.1102230246251565e-16; }   // 2^-53
    static __device__ __forceinline__ double tiny() { return 1e-280; }
    static __device__ __forceinline__ double inf() { return __longlong_as_double(0x7ff0000000000000LL); }
    static __device__ __forceinline__ double from64(double x) { return x; }
    static __device__ __forceinline__ T2 mk2(double x, double y) { return make_double2(x, y); }
    static __device__ __forceinline__ T4 mk4(double x, double y, double z, double w) { return make_double4(x, y, z, w); }
};

// Minimum-image offset c - p rounded once.  When the raw difference says the image across
// the boundary is nearer, the box edge is first removed from the coordinate lying in the far
// half of the box (exact for coordinates in [L/2, 2L], Sterbenz), so the last subtraction is
// the only rounding.  Identical formula in the oracle (oracle/dgt_oracle.c dgt_offset1).
__device__ __forceinline__ double wrap_off(double c, double p, double L, double hL)
{
    double d = __dsub_rn(c, p);
    if (d > hL) d = __dsub_rn(__dsub_rn(c, L), p);
    else if (d < -hL) d = __dsub_rn(c, __dsub_rn(p, L));
    return d;
}

// Circle of a ring edge: {2cx, 2cy, Eb, rc} where c is the centre of the circle through
// (0, a, b), Eb the per-|d| coefficient of the test bound and rc >= |c| + |c~ - c| a safe
// radius around c~ for scan-region certification (every point strictly inside the exact
// circle lies within rc of c~).  A degenerate or ill-conditioned edge (gamma <= 0 or
// relative error of gamma above 1/8) gets Eb = rc = inf: every test against it is undecided
// and goes to the float64 recheck.
//
// Bound derivation (u = unit roundoff of T; a~, b~ are the T-rounded double offsets):
//   |n~a - na| <= 4.01u na; |N~ - N| <= 7.2u Nhat (N = na*by - nb*ay etc., Nhat its
//   permanent); |g~ - g| <= 4.1u ghat, rho = 4.1u ghat / g~.
//   2c~ = N~ * rcp(g~) (1+delta), |delta| <= 4u with the hardware reciprocal:
//   |2c~ - 2c| (1 - rho) <= 7.2u (Nxhat + Nyhat)/g~ + |2c~| (rho + 4u)
//   => E = |c~ - c| <= [3.6u (Nxhat+Nyhat)/g~ + |c~|(rho+4u)] / (1-rho), inflated by 1.1.
//   Test s~ = fma(dx, 2cx~, fma(dy, 2cy~, -nd~)):
//   |s~ - s| <= |d|(2E + 2u|c| + 4u|c~|)(1+2u) + 6.1u nd  <= |d| Eb + 8u nd + tiny,
//   Eb = 2.1E + 8u|c~|.
// Reciprocal and upper-bounded square root.  float: the hardware approximations (relative
// error below 2^-22, covered by the 4u terms of the bounds below); double: IEEE operations.
__device__ __forceinline__ float rcp_approx(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double rcp_approx(double x) { return 1.0 / x; }
// sqrt(x) * (1 + tiny) >= sqrt(x); NaN for x == 0 in float (callers treat NaN as undecided)
__device__ __forceinline__ float sqrt_up(float x) { return x * rsqrtf(x) * 1.00000191f; }
__device__ __forceinline__ double sqrt_up(double x) { return sqrt(x); }

template <typename T>
__device__ __forceinline__ typename Prec<T>::T4 make_circ(T ax, T ay, T bx, T by)
{
    typedef Prec<T> P;
    const T u = P::u();
    T na = ax * ax + ay * ay;
    T nb = bx * bx + by * by;
    T g = ax * by - ay * bx;
    T gh = fabs(ax * by) + fabs(ay * bx);
    if (!(g > (T)0) || !((T)4.1 * u * gh <= (T)0.125 * g)) return P::mk4((T)0, (T)0, P::inf(), P::inf());
    T ig = rcp_approx(g);
    T rho = (T)4.1 * u * gh * ig * ((T)1 + (T)4 * u);
    T nx = na * by - nb * ay;
    T nxh = na * fabs(by) + nb * fabs(ay);
    T ny = nb * ax - na * bx;
    T nyh = nb * fabs(ax) + na * fabs(bx);
    T cx2 = nx * ig, cy2 = ny * ig;   // relative error <= 4u beyond that of nx, ny
    T t = cx2 * cx2 + cy2 * cy2;
    T cn = (t > (T)0) ? (T)0.5 * sqrt_up(t) * ((T)1 + (T)4 * u) : (T)0;
    // 1 / (1 - rho) <= 1 + 1.2 rho for rho <= 1/8
    T E = ((T)3.6 * u * (nxh + nyh) * ig * ((T)1 + (T)4 * u) + cn * (rho + (T)4 * u)) * ((T)1 + (T)1.2 * rho);
    E = E * (T)1.1 + P::tiny();
    T eb = (T)2.1 * E + (T)8 * u * cn + P::tiny();
    T rc = cn * ((T)1 + (T)16 * u) + (T)2 * E;   // |c| + |c~ - c| <= |c~| + 2E
    if (!(eb < P::inf()) || !(rc < P::inf())) return P::mk4((T)0, (T)0, P::inf(), P::inf());
    return P::mk4(cx2, cy2, eb, rc);
}

// float64 in-circle on double offsets with the permanent error bound.
// Returns +1 inside, -1 outside, 0 undecided.
__device__ __forceinline__ int incircle64(double ax, double ay, double bx, double by, double dx, double dy)
{
    double na = ax * ax + ay * ay, nb = bx * bx + by * by, nd = dx * dx + dy * dy;
    double c1 = dx * by - dy * bx;   // d x b
    double c2 = ax * dy - ay * dx;   // a x d
    double c3 = bx * ay - by * ax;   // b x a
    double v = na * c1 + nb * c2 + nd * c3;
    double P = na * (fabs(dx * by) + fabs(dy * bx)) + nb * (fabs(ax * dy) + fabs(ay * dx)) +
               nd * (fabs(bx * ay) + fabs(by * ax));
    double bound = 1.1102230246251565e-15 * P + 1e-290;   // 10u P
    if (v > bound) return 1;
    if (v < -bound) return -1;
    return 0;
}

// float32 in-circle (test kernel) on float32-rounded double offsets: bound 16u|P| covers
// the input rounding (4.01u P) and the arithmetic (7u P) with margin.
__device__ __forceinline__ int incircle32(float ax, float ay, float bx, float by, float dx, float dy)
{
    float na = ax * ax + ay * ay, nb = bx * bx + by * by, nd = dx * dx + dy * dy;
    float c1 = dx * by - dy * bx;
    float c2 = ax * dy - ay * dx;
    float c3 = bx * ay - by * ax;
    float v = na * c1 + nb * c2 + nd * c3;
    float P = na * (fabsf(dx * by) + fabsf(dy * bx)) + nb * (fabsf(ax * dy) + fabsf(ay * dx)) +
              nd * (fabsf(bx * ay) + fabsf(by * ax));
    float bound = 9.5367431640625e-07f * P + 1e-30f;   // 16u P
    if (v > bound) return 1;
    if (v < -bound) return -1;
    return 0;
}

// orientation of (0, a, b): +1 CCW, -1 CW, 0 undecided
__device__ __forceinline__ int orient32(float ax, float ay, float bx, float by)
{
    float g = ax * by - ay * bx;
    float b = 3.5762786865234375e-07f * (fabsf(ax * by) + fabsf(ay * bx)) + 1e-30f;   // 6u
    if (g > b) return 1;
    if (g < -b) return -1;
    return 0;
}
__device__ __forceinline__ int orient64(double ax, double ay, double bx, double by)
{
    double g = ax * by - ay * bx;
    double b = 4.4408920985006262e-16 * (fabs(ax * by) + fabs(ay * bx)) + 1e-290;   // 4u
    if (g > b) return 1;
    if (g < -b) return -1;
    return 0;
}

// ---------------------------------------------------------------------------------------
// exact expansion arithmetic (slow path only)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void two_sum(double a, double b, double &x, double &y)
{
    x = __dadd_rn(a, b);
    double bv = __dsub_rn(x, a);
    double av = __dsub_rn(x, bv);
    y = __dadd_rn(__dsub_rn(a, av), __dsub_rn(b, bv));
}
__device__ __forceinline__ void two_prod(double a, double b, double &x, double &y)
{
    x = __dmul_rn(a, b);
    y = __fma_rn(a, b, -x);
}
// h = e + b (zero-eliminating); returns length
__device__ inline int ex_grow(int elen, const double *e, double b, double *h)
{
    double q = b, hh;
    int hi = 0;
    for (int i = 0; i < elen; i++) {
        two_sum(q, e[i], q, hh);
        if (hh != 0.0) h[hi++] = hh;
    }
    if (q != 0.0 || hi == 0) h[hi++] = q;
    return hi;
}
// h = e + f, h must not alias; tmp of size >= elen + flen
__device__ inline int ex_sum(int elen, const double *e, int flen, const double *f, double *h, double *tmp)
{
    int hl = elen;
    for (int i = 0; i < elen; i++) h[i] = e[i];
    for (int i = 0; i < flen; i++) {
        int nl = ex_grow(hl, h, f[i], tmp);
        for (int k = 0; k < nl; k++) h[k] = tmp[k];
        hl = nl;
    }
    return hl;
}
__device__ inline int ex_scale(int elen, const double *e, double b, double *h)
{
    double q, sum, hh, p1, p0;
    int hi = 0;
    two_prod(e[0], b, q, hh);
    if (hh != 0.0) h[hi++] = hh;
    for (int i = 1; i < elen; i++) {
        two_prod(e[i], b, p1, p0);
        two_sum(q, p0, sum, hh);
        if (hh != 0.0) h[hi++] = hh;
        two_sum(p1, sum, q, hh);
        if (hh != 0.0) h[hi++] = hh;
    }
    if (q != 0.0 || hi == 0) h[hi++] = q;
    return hi;
}
// exact u*v - w*z (<= 4 terms)
__device__ inline int ex_cross(double u, double v, double w, double z, double *h)
{
    double a1, a0, b1, b0, t[8], tmp[8];
    two_prod(u, v, a1, a0);
    two_prod(w, z, b1, b0);
    double pos[2] = { a0, a1 }, neg[2] = { -b0, -b1 };
    int l = ex_sum(2, pos, 2, neg, t, tmp);
    for (int i = 0; i < l; i++) h[i] = t[i];
    return l;
}
__device__ inline int ex_norm2(double u, double v, double *h)
{
    double a1, a0, b1, b0, tmp[8];
    two_prod(u, u, a1, a0);
    two_prod(v, v, b1, b0);
    double e[2] = { a0, a1 }, f[2] = { b0, b1 };
    return ex_sum(2, e, 2, f, h, tmp);
}
// product of a <=4-term and a <=4-term expansion (<= 32 terms)
__device__ inline int ex_prod44(int el, const double *e, int fl, const double *f, double *h)
{
    double part[8], acc[32], tmp[40];
    int al = 1;
    acc[0] = 0.0;
    for (int i = 0; i < fl; i++) {
        int pl = ex_scale(el, e, f[i], part);
        al = ex_sum(al, acc, pl, part, h, tmp);
        for (int k = 0; k < al; k++) acc[k] = h[k];
    }
    for (int k = 0; k < al; k++) h[k] = acc[k];
    return al;
}
__device__ inline int ex_sign(int l, const double *e)
{
    for (int i = l - 1; i >= 0; i--) {
        if (e[i] > 0) return 1;
        if (e[i] < 0) return -1;
    }
    return 0;
}
// exact sign of inc0(a, b, d)
__device__ inline int incircle_exact(double ax, double ay, double bx, double by, double dx, double dy)
{
    double na[4], nb[4], nd[4], c1[4], c2[4], c3[4];
    double t1[32], t2[32], t3[32], s12[64], s[96], tmp[96];
    int lna = ex_norm2(ax, ay, na), lnb = ex_norm2(bx, by, nb), lnd = ex_norm2(dx, dy, nd);
    int l1 = ex_cross(dx, by, dy, bx, c1);
    int l2 = ex_cross(ax, dy, ay, dx, c2);
    int l3 = ex_cross(bx, ay, by, ax, c3);
    int lt1 = ex_prod44(lna, na, l1, c1, t1);
    int lt2 = ex_prod44(lnb, nb, l2, c2, t2);
    int lt3 = ex_prod44(lnd, nd, l3, c3, t3);
    int l12 = ex_sum(lt1, t1, lt2, t2, s12, tmp);
    int ls = ex_sum(l12, s12, lt3, t3, s, tmp);
    return ex_sign(ls, s);
}
__device__ inline int orient_exact(double ax, double ay, double bx, double by)
{
    double h[4];
    int l = ex_cross(ax, by, ay, bx, h);
    return ex_sign(l, h);
}

}  // namespace dgt

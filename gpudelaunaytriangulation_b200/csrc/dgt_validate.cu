// Device-side validation of a triangulation held in the caller's arrays (no reference
// counterpart: the reference checks its output on the host against CGAL).
//
// One thread per point, index order, exact predicates (float64 filter, expansion residue):
//   - the row: length in [3, stride], indices in range, not the point itself, no repeats;
//   - the fan: every triangle (p, P_k, P_k+1) strictly counter-clockwise, winding once
//     (a fan with a non-positive triangle also counts as not winding once);
//   - symmetry: every neighbour j lists p, with p's neighbours P_k+1 before and P_k-1 after
//     it (the same two triangles seen from j);
//   - local Delaunay: P_k+1 not strictly inside the circle through (p, P_k-1, P_k).
// All row reads are bounds-checked, so a corrupt row is counted, never followed.  With every
// count zero and the ring lengths summing to 6n (Euler: a triangulation of the torus has
// 3n edges) the rings form a consistent triangulation of the torus whose edges are all
// locally Delaunay, i.e. the Delaunay triangulation (in general position).
#include "dgt.h"
#include "dgt_internal.cuh"
#include "dgt_predicates.cuh"

namespace dgt {

namespace {

__device__ __noinline__ int incircle_exact_v(double2 a, double2 b, double2 d)
{
    return incircle_exact(a.x, a.y, b.x, b.y, d.x, d.y);
}

// exact sign of "d strictly inside the circle through (0, a, b)"
__device__ int incircle_v(double2 a, double2 b, double2 d)
{
    const int r = incircle64(a.x, a.y, b.x, b.y, d.x, d.y);
    return r != 0 ? r : incircle_exact_v(a, b, d);
}

__device__ int orient_v(double2 a, double2 b)
{
    const int r = orient64(a.x, a.y, b.x, b.y);
    return r != 0 ? r : orient_exact(a.x, a.y, b.x, b.y);
}

struct ValidateArgs {
    const SetDesc *sets;
    const int *set_of;
    const double2 *pos;
    const int *tri;
    const int *nn;
    int stride;
    int n;
    unsigned long long *out;   // sum, bad_rows, asymmetric, not_ccw, winding, not_delaunay, points
};

constexpr int V_COUNTS = 7;

template <bool GEN>
__global__ void __launch_bounds__(256) k_validate(ValidateArgs A)
{
    unsigned long long c[V_COUNTS] = { 0, 0, 0, 0, 0, 0, 0 };
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        c[6]++;
        const int m = A.nn[i];
        const int *row = A.tri + (size_t)i * A.stride;
        bool bad = m < 3 || m > A.stride;
        c[0] += (unsigned long long)(long long)m;
        if (!bad) {
            for (int k = 0; k < m && !bad; ++k) {
                const int r = row[k];
                bad = r < 0 || r >= A.n || r == i;
                for (int t = 0; t < k && !bad; ++t) bad = row[t] == r;
            }
        }
        if (bad) {
            c[1]++;
            continue;
        }
        const SetDesc S = A.sets[A.set_of ? A.set_of[i] : 0];
        const double2 p = A.pos[i];
        auto off = [&](int j) {
            const double2 q = A.pos[j];
            return GEN ? gen_off(q, p, S) : make_double2(wrap_off(q.x, p.x, S.Lx, S.hLx), wrap_off(q.y, p.y, S.Ly, S.hLy));
        };
        double2 prev = off(row[m - 1]), cur = off(row[0]);
        int cross = 0;
        bool allpos = true;
        for (int k = 0; k < m; ++k) {
            const int jn = row[k + 1 == m ? 0 : k + 1];
            const double2 nxt = off(jn);
            const int o = orient_v(cur, nxt);
            if (o <= 0) {
                c[3]++;
                allpos = false;
            }
            if (cur.y < 0.0 && nxt.y >= 0.0) cross++;
            if (incircle_v(prev, cur, nxt) > 0) c[5]++;
            // symmetry of the spoke (p, P_k): ring(P_k) holds p between P_k+1 and P_k-1
            const int j = row[k], pk = row[k == 0 ? m - 1 : k - 1];
            const int mj = A.nn[j];
            bool sym = false;
            if (mj >= 1 && mj <= A.stride) {
                const int *rj = A.tri + (size_t)j * A.stride;
                for (int t = 0; t < mj; ++t) {
                    if (rj[t] != i) continue;
                    sym = rj[t == 0 ? mj - 1 : t - 1] == jn && rj[t + 1 == mj ? 0 : t + 1] == pk;
                    break;
                }
            }
            if (!sym) c[2]++;
            prev = cur;
            cur = nxt;
        }
        if (!allpos || cross != 1) c[4]++;
    }
    for (int q = 0; q < V_COUNTS; ++q) {
        for (int o = 16; o > 0; o >>= 1) c[q] += __shfl_down_sync(0xffffffffu, c[q], o);
        if ((threadIdx.x & 31) == 0 && c[q]) atomicAdd(&A.out[q], c[q]);
    }
}

}  // namespace

cudaError_t launch_validate(const SetDesc *sets, const int *set_of, const double2 *pos, const int *tri,
                            const int *nn, int stride, int n, unsigned long long *out, int sms, int general,
                            cudaStream_t s)
{
    ValidateArgs a{ sets, set_of, pos, tri, nn, stride, n, out };
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long) * V_COUNTS, s);
    if (e != cudaSuccess || n <= 0) return e;
    int blocks = (n + 255) / 256;
    const int cap = (sms > 0 ? sms : 148) * 8;
    if (blocks > cap) blocks = cap;
    if (general) k_validate<true><<<blocks, 256, 0, s>>>(a);
    else k_validate<false><<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace dgt

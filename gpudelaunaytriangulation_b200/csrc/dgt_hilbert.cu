// Hilbert-curve order of the points, set by set: the spatial pre-pass the reference offers
// for renumbering its inputs (hilbertSortArray, triangulation.cpp:63-88, which sorts by
// xy2d of src/utilities/hilbert_curve.cpp:229 on the host), here on the device and over each
// set's own box.
//
// Set s is covered by a 2^k x 2^k grid, the smallest with 4^k >= its points (1 <= k <= 15),
// laid over its box (over its fractional frame for a general box).  A point's key is the
// position of its grid square along the Hilbert curve of that grid: the standard conversion
// of square coordinates to a curve index, level by level from the coarsest -- the quadrant
// (rx, ry) at level s adds s^2 * ((3 rx) xor ry), then the coordinates are reflected and
// swapped into that quadrant's own frame.  The points are counting-sorted by (set, key):
// count and atomic rank per key, exclusive scan, scatter; the points sharing a key are then
// ordered by index, so the result does not depend on atomic arrival order.
#include "dgt_internal.cuh"

namespace dgt {

// Curve index of grid square (x, y) of a 2^k x 2^k grid (k <= 15: the index fits 30 bits)
__device__ __forceinline__ unsigned hilbert_index(int k, unsigned x, unsigned y)
{
    unsigned d = 0;
    for (int lv = k - 1; lv >= 0; --lv) {
        const unsigned s = 1u << lv;
        const unsigned rx = (x >> lv) & 1u, ry = (y >> lv) & 1u;
        d += s * s * ((3u * rx) ^ ry);
        // the quadrant's own frame: only the bits below this level matter from here on
        x &= s - 1u;
        y &= s - 1u;
        if (ry == 0u) {
            if (rx == 1u) {
                x = s - 1u - x;
                y = s - 1u - y;
            }
            const unsigned t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

// grid square along one axis: floor(u) within [0, 2^k) (NaN and negatives to 0)
__device__ __forceinline__ unsigned hilbert_square(double u, int k)
{
    const int g = 1 << k;
    if (!(u >= 0.0)) return 0u;
    return u < (double)g ? (unsigned)u : (unsigned)(g - 1);
}

__global__ void __launch_bounds__(256) k_hilbert_key(const double2 *pos, int n, const SetDesc *sets,
                                                     const int *set_of, const HilbertSet *hsets, int *hcount,
                                                     int *hbucket, int *hrank)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = set_of ? set_of[i] : 0;
        const SetDesc &S = sets[s];
        const HilbertSet h = hsets[s];
        const double2 p = pos[i];
        double u, v;
        if (S.general) {
            // fractional coordinates in the box's own frame, wrapped into [0, 1)
            u = __fma_rn(S.i11, p.x, __dmul_rn(S.i12, p.y));
            v = __fma_rn(S.i21, p.x, __dmul_rn(S.i22, p.y));
            u = (u - floor(u)) * h.sx;
            v = (v - floor(v)) * h.sy;
        } else {
            u = p.x * h.sx;
            v = p.y * h.sy;
        }
        const int b = h.base + (int)hilbert_index(h.k, hilbert_square(u, h.k), hilbert_square(v, h.k));
        hbucket[i] = b;
        hrank[i] = atomicAdd(&hcount[b], 1);
    }
}

__global__ void __launch_bounds__(256) k_hilbert_scatter(int n, const int *hstart, const int *hbucket,
                                                         const int *hrank, int *order)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        order[hstart[hbucket[i]] + hrank[i]] = i;
}

// the points of each curve square by index (insertion sort: about one point per square on
// average; dense clusters put a few hundred in one)
__global__ void __launch_bounds__(256) k_hilbert_sort(int nb, const int *hstart, int *order)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const int lo = hstart[b], hi = hstart[b + 1];
        for (int k = lo + 1; k < hi; ++k) {
            const int id = order[k];
            int j = k - 1;
            while (j >= lo && order[j] > id) {
                order[j + 1] = order[j];
                --j;
            }
            order[j + 1] = id;
        }
    }
}

static int grid_for(long long items)
{
    const long long g = (items + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 65535 ? 65535 : g));
}

__global__ void __launch_bounds__(256) k_gather_points(const double2 *src, const int *order, int n, double2 *dst)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dst[k] = src[order[k]];
}

cudaError_t launch_gather_points(const double2 *src, const int *order, int n, double2 *dst, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_gather_points<<<grid_for(n), 256, 0, s>>>(src, order, n, dst);
    return cudaGetLastError();
}

cudaError_t launch_hilbert_order(const HilbertArgs &a, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(a.hcount, 0, sizeof(int) * ((size_t)a.buckets + 1), s);
    if (e != cudaSuccess) return e;
    k_hilbert_key<<<grid_for(a.n), 256, 0, s>>>(a.pos, a.n, a.sets, a.set_of, a.hsets, a.hcount, a.hbucket,
                                                 a.hrank);
    e = launch_scan(a.hcount, a.buckets + 1, a.bsum, a.hstart, s);
    if (e != cudaSuccess) return e;
    k_hilbert_scatter<<<grid_for(a.n), 256, 0, s>>>(a.n, a.hstart, a.hbucket, a.hrank, a.order);
    k_hilbert_sort<<<grid_for(a.buckets), 256, 0, s>>>(a.buckets, a.hstart, a.order);
    return cudaGetLastError();
}

}  // namespace dgt

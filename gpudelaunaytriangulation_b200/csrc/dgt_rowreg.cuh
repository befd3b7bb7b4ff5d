// Ring rows held in registers: up to RR entries, every index a compile-time constant after
// unrolling (no local-memory arrays), rows loaded with 16-byte vector loads where aligned.
// Used by the edge flips, the repair bookkeeping of the ring kernels and the local test.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dgt {

// Rings up to RR entries fit the register path (longer rings take generic paths).
constexpr int RR = 16;

struct Ring16 {
    int r[RR];
};

// the first min(stride, RR) entries of a row (entries past the ring length are ignored by
// the searches); 16-byte vector loads when the row is aligned and the stride a multiple of 4
__device__ __forceinline__ void row_load(const int *row, int stride, Ring16 &R)
{
    const int lim = stride < RR ? stride : RR;
    if ((stride & 3) == 0 && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
        const int4 *v = reinterpret_cast<const int4 *>(row);
#pragma unroll
        for (int q = 0; q < RR / 4; ++q) {
            int4 x = make_int4(-1, -1, -1, -1);
            if (4 * q < lim) x = v[q];
            R.r[4 * q] = x.x;
            R.r[4 * q + 1] = x.y;
            R.r[4 * q + 2] = x.z;
            R.r[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int t = 0; t < RR; ++t) R.r[t] = t < lim ? row[t] : -1;
    }
}

// position of x in the ring of length m (<= RR), with its CCW predecessor and successor
__device__ __forceinline__ int ring_find(const Ring16 &R, int m, int x, int &pred, int &succ)
{
    int k = -1, last = R.r[0];
#pragma unroll
    for (int t = 1; t < RR; ++t)
        if (t == m - 1) last = R.r[t];
    pred = succ = -1;
#pragma unroll
    for (int t = 0; t < RR; ++t) {
        if (t < m && R.r[t] == x) {
            k = t;
            pred = t == 0 ? last : R.r[t > 0 ? t - 1 : 0];
            succ = t + 1 < m ? R.r[t + 1 < RR ? t + 1 : 0] : R.r[0];
        }
    }
    return k;
}

// remove position k (ring length m -> m - 1)
__device__ __forceinline__ void ring_drop(Ring16 &R, int k)
{
#pragma unroll
    for (int t = 0; t < RR - 1; ++t)
        if (t >= k) R.r[t] = R.r[t + 1];
}

// insert x right after position k (ring length m < RR -> m + 1)
__device__ __forceinline__ void ring_put_after(Ring16 &R, int k, int x)
{
#pragma unroll
    for (int t = RR - 1; t > 0; --t)
        if (t > k + 1) R.r[t] = R.r[t - 1];
#pragma unroll
    for (int t = 0; t < RR; ++t)
        if (t == k + 1) R.r[t] = x;
}

// write a ring of length w rotated to start at its smallest index
__device__ __forceinline__ void ring_store(int *row, const Ring16 &R, int w)
{
    int best = 0, bv = R.r[0];
#pragma unroll
    for (int t = 1; t < RR; ++t)
        if (t < w && R.r[t] < bv) {
            bv = R.r[t];
            best = t;
        }
#pragma unroll
    for (int t = 0; t < RR; ++t)
        if (t < w) {
            int d = t - best;
            if (d < 0) d += w;
            row[d] = R.r[t];
        }
}

}  // namespace dgt

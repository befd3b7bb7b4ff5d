// Edge flips: the first stage of test-and-repair.
//
// After a displacement most of a triangulation is still a triangulation (every fan winds
// once with strictly CCW triangles) and only some edges fail the in-circle test.  For such
// an edge (i, j) with i < j, ring(i) = ..., a, j, b, ... (triangles (i, a, j) and (i, j, b)),
// the edge is illegal iff b lies strictly inside the circle through (i, a, j); the two
// triangles then form a strictly convex quadrilateral (b is in the cap cut off by the chord
// ij, so segment ab crosses segment ij) and the flip replaces (i, j) by (a, b):
//     ring(i): a, j, b -> a, b        ring(j): b, i, a -> b, a
//     ring(a): j, i    -> j, b, i     ring(b): i, j    -> i, a, j
// This is Lawson's flip (the reference rebuilds every flagged point instead; its final
// triangulation is the same Delaunay triangulation).
//
// A round is two launches over the candidate list: k_flip_claim re-derives each candidate's
// quadrilateral from the current rings, drops it when it is legal (exact in-circle), gone, or
// touches a point already queued for rebuilding, and claims its four vertices with a 64-bit
// atomicMax of (round stamp, mixed list slot); k_flip_apply lets every candidate that holds
// all four claims flip (winners' quadrilaterals are vertex-disjoint, so no ring is edited
// twice in a round) and queues the losers and those outer edges of each flip that a float32
// in-circle cannot show legal.  Stamps
// only grow (a per-context device counter advanced at the end of each call), so claims are
// never cleared.  Anything the flips cannot settle -- a quadrilateral that is inconsistent
// between the rings, a ring that would outgrow the stride or shrink below three, offsets
// far from the owning point, a full list, or candidates left after the last round -- goes to
// the rebuild rounds (exact one-ring construction with consistency propagation), which
// finish the repair.
#include "dgt_internal.cuh"
#include "dgt_predicates.cuh"
#include "dgt_rowreg.cuh"

namespace dgt {

namespace {

// the exact residue, out of line (its expansion arrays stay off the callers' frames)
__device__ __noinline__ int incircle_exact_call(double2 a, double2 b, double2 d)
{
    return incircle_exact(a.x, a.y, b.x, b.y, d.x, d.y);
}

// double offset of q relative to p (minimum image, rounded once; GEN: general box)
template <bool GEN>
__device__ __forceinline__ double2 off64(double2 q, double2 p, const SetDesc &S)
{
    return GEN ? gen_off(q, p, S) : make_double2(wrap_off(q.x, p.x, S.Lx, S.hLx), wrap_off(q.y, p.y, S.Ly, S.hLy));
}

// float32 offset of q relative to p (the double offset rounded to float)
template <bool GEN>
__device__ __forceinline__ float2 off32(double2 q, double2 p, const SetDesc &S)
{
    const double2 d = off64<GEN>(q, p, S);
    return make_float2(__double2float_rn(d.x), __double2float_rn(d.y));
}

// an offset within a quarter of the box's half extent per axis (cell units for a general box)
template <bool GEN>
__device__ __forceinline__ bool near_owner(double2 o, const SetDesc &S)
{
    if (GEN)
        return fabs(S.g11 * o.x + S.g12 * o.y) < 0.25 * S.hxs && fabs(S.g21 * o.x + S.g22 * o.y) < 0.25 * S.hys;
    return fabs(o.x) < 0.25 * S.hLx && fabs(o.y) < 0.25 * S.hLy;
}

// exact sign of "d strictly inside the circle through (0, a, b)" (CCW (0, a, b))
__device__ int incircle_staged(double2 a, double2 b, double2 d)
{
    int r = incircle32(__double2float_rn(a.x), __double2float_rn(a.y), __double2float_rn(b.x),
                       __double2float_rn(b.y), __double2float_rn(d.x), __double2float_rn(d.y));
    if (r != 0) return r;
    r = incircle64(a.x, a.y, b.x, b.y, d.x, d.y);
    if (r != 0) return r;
    return incircle_exact_call(a, b, d);
}

__device__ int orient_staged(double2 a, double2 b)
{
    int r = orient64(a.x, a.y, b.x, b.y);
    if (r != 0) return r;
    return orient_exact(a.x, a.y, b.x, b.y);
}

// queue point v for the rebuild rounds (once per call)
__device__ __forceinline__ void to_rebuild(const FlipArgs &A, int ebase, int v)
{
    if (v >= 0 && v < A.n && atomicMax(&A.mark[v], ebase) < ebase) {
        A.rebuild_list[atomicAdd(A.rebuild_count, 1)] = v;
        atomicAdd(&A.st->flagged, 1ull);
    }
}

// append k edges per lane to the next list, one atomic per warp (every lane calls this);
// what does not fit goes to the rebuild rounds
__device__ __forceinline__ void warp_push_edges(const FlipArgs &A, int ebase, const int2 *items, int k)
{
    const int lane = threadIdx.x & 31;
    int incl = k;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(A.next_count, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    const int off = base + incl - k;
    for (int t = 0; t < k; ++t) {
        if (off + t < A.cap) {
            A.next[off + t] = items[t];
        } else {
            to_rebuild(A, ebase, items[t].x);
            to_rebuild(A, ebase, items[t].y);
        }
    }
}

// Claim key of list slot `slot` in the round with stamp `stamp`.  The low word is a bijection
// of the slot (xor-shift / odd-multiply steps are each invertible), so keys stay unique --
// two candidates can never both believe they hold a vertex -- while neighbouring slots (the
// list is appended in cell order) get unrelated priorities: with slot-ordered priorities a
// run of conflicting candidates would let only its last one win per round.
__device__ __forceinline__ unsigned long long claim_key(unsigned stamp, int slot)
{
    unsigned x = (unsigned)slot;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return ((unsigned long long)stamp << 32) | x;
}

template <bool GEN>
__global__ void __launch_bounds__(256, 2) k_flip_claim(FlipArgs A, int round)
{
    const int ebase = *A.epoch_ptr + 1;
    const unsigned stamp = *A.stamp_ptr + 1 + round;
    const int n = min(*A.cur_count, A.cap);
    // the next round's list is appended by this round's apply kernel: cleared here (the last
    // reader of that buffer, the previous round's apply, has finished) instead of by a memset
    if (blockIdx.x == 0 && threadIdx.x == 0) *A.next_count = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int2 ed = A.cur[e];
        const int i = ed.x, j = ed.y;
        int2 q = make_int2(-1, -1);
        if (i >= 0 && i < A.n && j >= 0 && j < A.n && i != j) {
            // loads of the edge's end points, all independent
            const int mi = A.nn[i], mj = A.nn[j];
            const bool free_ij = A.mark[i] < ebase && A.mark[j] < ebase;
            Ring16 ri, rj;
            row_load(A.tri + (size_t)i * A.stride, A.stride, ri);
            row_load(A.tri + (size_t)j * A.stride, A.stride, rj);
            const double2 p = __ldg(&A.pos[i]);
            const double2 qj = __ldg(&A.pos[j]);
            const bool rows_ok = mi >= 3 && mi <= min(A.stride, RR) && mj >= 3 && mj <= min(A.stride, RR);
            int a = -1, b = -1;
            const int k = rows_ok ? ring_find(ri, mi, j, a, b) : -1;
            if (!rows_ok && free_ij && (mi > RR || mj > RR)) {
                to_rebuild(A, ebase, i);   // a ring too long for the register path
                to_rebuild(A, ebase, j);
            } else if (k >= 0 && free_ij && a != b) {
                // loads of the opposite vertices, all independent
                const int ma = A.nn[a], mb = A.nn[b];
                const bool free_ab = A.mark[a] < ebase && A.mark[b] < ebase;
                const double2 qa = __ldg(&A.pos[a]), qb = __ldg(&A.pos[b]);
                Ring16 ra, rb;
                row_load(A.tri + (size_t)a * A.stride, A.stride, ra);
                row_load(A.tri + (size_t)b * A.stride, A.stride, rb);
                const SetDesc S = A.sets[A.set_of ? A.set_of[i] : 0];
                const double2 oa = off64<GEN>(qa, p, S), oj = off64<GEN>(qj, p, S), ob = off64<GEN>(qb, p, S);
                if (free_ab && incircle_staged(oa, oj, ob) > 0) {
                    // an illegal edge: flip it if the quadrilateral is consistent in all four
                    // rings, near the owning point and within the register rings, else rebuild
                    bool ok = near_owner<GEN>(oa, S) && near_owner<GEN>(oj, S) && near_owner<GEN>(ob, S);
                    ok = ok && orient_staged(oa, ob) > 0 && mi > 3 && mj > 3;
                    ok = ok && ma >= 3 && mb >= 3 && ma < min(A.stride, RR) && mb < min(A.stride, RR);
                    int pr, sc;
                    ok = ok && ring_find(rj, mj, i, pr, sc) >= 0 && pr == b && sc == a;
                    ok = ok && ring_find(ra, ma, i, pr, sc) >= 0 && pr == j;
                    ok = ok && ring_find(rb, mb, j, pr, sc) >= 0 && pr == i;
                    if (ok) {
                        q = make_int2(a, b);
                        const unsigned long long key = claim_key(stamp, e);
                        atomicMax(&A.claim[i], key);
                        atomicMax(&A.claim[j], key);
                        atomicMax(&A.claim[a], key);
                        atomicMax(&A.claim[b], key);
                    } else {
                        to_rebuild(A, ebase, i);
                        to_rebuild(A, ebase, j);
                        to_rebuild(A, ebase, a);
                        to_rebuild(A, ebase, b);
                    }
                }
            }
        }
        A.quad[e] = q;   // (-1, -1): nothing to flip
    }
}

template <bool GEN>
__global__ void __launch_bounds__(256, 2) k_flip_apply(FlipArgs A, int round)
{
    const int ebase = *A.epoch_ptr + 1;
    const unsigned stamp = *A.stamp_ptr + 1 + round;
    const int n = min(*A.cur_count, A.cap);
    unsigned long long flips = 0;
    // warp-uniform trip count: every lane reaches the warp-aggregated append
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int e = base + (int)threadIdx.x;
        int2 out[4];
        int k = 0;
        const int2 q = e < n ? A.quad[e] : make_int2(-1, -1);
        if (q.x >= 0) {
            const int2 ed = A.cur[e];
            const int i = ed.x, j = ed.y, a = q.x, b = q.y;
            const unsigned long long key = claim_key(stamp, e);
            if (A.claim[i] != key || A.claim[j] != key || A.claim[a] != key || A.claim[b] != key) {
                out[k++] = ed;   // lost a vertex to another flip: next round
            } else {
                // the four rings in registers (lengths checked by the claim: i, j > 3, a, b < RR)
                int *wi = A.tri + (size_t)i * A.stride, *wj = A.tri + (size_t)j * A.stride;
                int *wa = A.tri + (size_t)a * A.stride, *wb = A.tri + (size_t)b * A.stride;
                const int mi = A.nn[i], mj = A.nn[j], ma = A.nn[a], mb = A.nn[b];
                Ring16 Ri, Rj, Ra, Rb;
                row_load(wi, A.stride, Ri);
                row_load(wj, A.stride, Rj);
                row_load(wa, A.stride, Ra);
                row_load(wb, A.stride, Rb);
                int pr, sc;
                ring_drop(Ri, ring_find(Ri, mi, j, pr, sc));
                ring_drop(Rj, ring_find(Rj, mj, i, pr, sc));
                ring_put_after(Ra, ring_find(Ra, ma, j, pr, sc), b);
                ring_put_after(Rb, ring_find(Rb, mb, i, pr, sc), a);
                ring_store(wi, Ri, mi - 1);
                ring_store(wj, Rj, mj - 1);
                ring_store(wa, Ra, ma + 1);
                ring_store(wb, Rb, mb + 1);
                A.nn[i] = mi - 1;
                A.nn[j] = mj - 1;
                A.nn[a] = ma + 1;
                A.nn[b] = mb + 1;
                flips++;
                // The outer edges (i,a), (i,b) seen from i and (j,a), (j,b) seen from j, with
                // the vertices across them read off the new rings: queued unless the float32
                // in-circle says legal outside its error bound (a margin far above the rounding
                // of offsets to another owner, so the claim's exact test would agree).
                int x, y, z, w, dummy;
                ring_find(Ri, mi - 1, a, x, dummy);   // ring(i): x, a, b, y
                ring_find(Ri, mi - 1, b, dummy, y);
                ring_find(Rj, mj - 1, a, dummy, z);   // ring(j): w, b, a, z
                ring_find(Rj, mj - 1, b, w, dummy);
                const SetDesc S = A.sets[A.set_of ? A.set_of[i] : 0];
                const double2 pi = __ldg(&A.pos[i]), pj = __ldg(&A.pos[j]), pa = __ldg(&A.pos[a]),
                              pb = __ldg(&A.pos[b]), px = __ldg(&A.pos[x]), py = __ldg(&A.pos[y]),
                              pz = __ldg(&A.pos[z]), pw = __ldg(&A.pos[w]);
                const float2 ia = off32<GEN>(pa, pi, S), ib = off32<GEN>(pb, pi, S), ix = off32<GEN>(px, pi, S),
                             iy = off32<GEN>(py, pi, S);
                const float2 ja = off32<GEN>(pa, pj, S), jb = off32<GEN>(pb, pj, S), jz = off32<GEN>(pz, pj, S),
                             jw = off32<GEN>(pw, pj, S);
                if (incircle32(ix.x, ix.y, ia.x, ia.y, ib.x, ib.y) >= 0) out[k++] = make_int2(min(i, a), max(i, a));
                if (incircle32(ia.x, ia.y, ib.x, ib.y, iy.x, iy.y) >= 0) out[k++] = make_int2(min(i, b), max(i, b));
                if (incircle32(jb.x, jb.y, ja.x, ja.y, jz.x, jz.y) >= 0) out[k++] = make_int2(min(j, a), max(j, a));
                if (incircle32(jw.x, jw.y, jb.x, jb.y, ja.x, ja.y) >= 0) out[k++] = make_int2(min(j, b), max(j, b));
            }
        }
        warp_push_edges(A, ebase, out, k);
    }
    for (int o = 16; o > 0; o >>= 1) flips += __shfl_down_sync(0xffffffffu, flips, o);
    if ((threadIdx.x & 31) == 0 && flips) atomicAdd(&A.st->flips, flips);
}

// candidates left after the last round: their end points go to the rebuild rounds
__global__ void __launch_bounds__(256) k_flip_spill(FlipArgs A, int rounds)
{
    const int ebase = *A.epoch_ptr + 1;
    const int n = min(*A.cur_count, A.cap);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int2 ed = A.cur[e];
        to_rebuild(A, ebase, ed.x);
        to_rebuild(A, ebase, ed.y);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicMax(&A.st->flip_rounds, rounds);
        if (n > 0) atomicAdd(&A.st->flip_spilled, (unsigned long long)n);
    }
}

__global__ void k_flip_stamp(DevCtl *ctl, int rounds)
{
    ctl->flip_stamp += (unsigned)rounds + 1u;
}

int flip_grid(int sms) { return (sms > 0 ? sms : 148) * 8; }

}  // namespace

cudaError_t launch_flip_round(const FlipArgs &a, int round, int sms, cudaStream_t s)
{
    if (a.general) k_flip_claim<true><<<flip_grid(sms), 256, 0, s>>>(a, round);
    else k_flip_claim<false><<<flip_grid(sms), 256, 0, s>>>(a, round);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.general) k_flip_apply<true><<<flip_grid(sms), 256, 0, s>>>(a, round);
    else k_flip_apply<false><<<flip_grid(sms), 256, 0, s>>>(a, round);
    return cudaGetLastError();
}

cudaError_t launch_flip_spill(const FlipArgs &a, int rounds, DevCtl *ctl, int sms, cudaStream_t s)
{
    k_flip_spill<<<flip_grid(sms), 256, 0, s>>>(a, rounds);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_flip_stamp<<<1, 1, 0, s>>>(ctl, rounds);
    return cudaGetLastError();
}

}  // namespace dgt

// Global triangulation without any device allocation (dgt_global_triangulation_noalloc).
//
// Some callers cannot call cudaMalloc: code running where the allocator is owned by
// someone else (a host application with its own pool that forbids side allocations,
// plugins loaded into a process whose memory budget is fixed up front, or paths that must
// not touch the allocator at all).  This entry point keeps every piece of scratch it needs
// (cell grid, cell-order copies, status block, rows of the exact / large-ring path) in one
// file-scope device array of fixed size, so a call allocates nothing: the caller passes the
// points, the output rows and the output lengths, nothing else is needed.
//
// Limits: at most DGT_NOALLOC_MAX_POINTS points and DGT_NOALLOC_MAX_CELLS grid cells; larger
// inputs are rejected with DGT_ERR_INVALID_ARGUMENT before any work is queued.  The array
// (NA_BYTES = 4,720,384 bytes, about 4.72 MB) exists on every GPU that loads this library,
// until the process exits.
//
// Sharing: all calls use the same array and it keeps the last call's contents; the parts
// that must start at zero (cell counts, status block) are cleared by every call.  Calls
// whose kernels overlap on a GPU (different streams or host threads without ordering)
// race on the array; callers must order them.
//
// Set-up: every call, with the caller's device current, looks up the array's device address
// (cudaGetSymbolAddress; in host code the array's name is only a host-side stand-in, never a
// device address).  Nothing is cached: after a cudaDeviceReset, or in another context on the
// same device, the library's module is loaded again at another address, and a cached pointer
// would send the kernels to stale memory.  The lookup is a host-side call, small next to the
// synchronisation that ends every call.
//
// Synchronisation: a call copies its status to pageable host memory and synchronises
// `stream`, so it must not be called while `stream` (or any stream in global capture mode) is
// capturing a CUDA graph.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "dgt.h"
#include "dgt_internal.cuh"

using namespace dgt;

namespace {

constexpr int NA_MAX_POINTS = DGT_NOALLOC_MAX_POINTS;
constexpr int NA_MAX_CELLS = DGT_NOALLOC_MAX_CELLS;
constexpr size_t NA_ALIGN = 256;

constexpr size_t up(size_t x) { return (x + NA_ALIGN - 1) / NA_ALIGN * NA_ALIGN; }

// byte offsets of each region inside the array
constexpr size_t OFF_SETS = 0;
constexpr size_t OFF_STATUS = OFF_SETS + up(sizeof(SetDesc));
constexpr size_t OFF_CCOUNT = OFF_STATUS + up(sizeof(DevStatus));
constexpr size_t OFF_CSTART = OFF_CCOUNT + up(sizeof(int) * (NA_MAX_CELLS + 1));
constexpr size_t OFF_BSUM = OFF_CSTART + up(sizeof(int) * (NA_MAX_CELLS + 1));
constexpr size_t OFF_CELLOF = OFF_BSUM + up(sizeof(int) * ((NA_MAX_CELLS + 1) / 4096 + 2));
constexpr size_t OFF_RANK = OFF_CELLOF + up(sizeof(int) * NA_MAX_POINTS);
constexpr size_t OFF_SIDX = OFF_RANK + up(sizeof(int) * NA_MAX_POINTS);
constexpr size_t OFF_SLOTOF = OFF_SIDX + up(sizeof(int) * NA_MAX_POINTS);
constexpr size_t OFF_DEFERLIST = OFF_SLOTOF + up(sizeof(int) * NA_MAX_POINTS);
constexpr size_t OFF_SPOS = OFF_DEFERLIST + up(sizeof(int) * NA_MAX_POINTS);
// occupancy blocks: bx*by <= cells/64 + (xsize+ysize)/8 + 1 <= cells/4 + 16
constexpr size_t NA_MAX_BLOCKS = NA_MAX_CELLS / 4 + 16;
constexpr size_t OFF_BCOUNT = OFF_SPOS + up(sizeof(double2) * NA_MAX_POINTS);
constexpr size_t NA_BYTES = OFF_BCOUNT + up(sizeof(int) * NA_MAX_BLOCKS);

}  // namespace

// the scratch array itself (device code could name it directly; host code needs its address)
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

namespace {

// the array's device address in the current context (looked up on every call, see above)
int scratch_base(unsigned char **out)
{
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) return DGT_ERR_CUDA;
    *out = static_cast<unsigned char *>(ptr);
    return DGT_OK;
}

double pow2_at_least(double x)
{
    double v = 1.0;
    while (v < x) v *= 2.0;
    return v;
}

}  // namespace

// writes the set descriptor and clears what must start at zero (cell counts, status)
__global__ void k_noalloc_setup(SetDesc S, SetDesc *sets, DevStatus *st, int *ccount, int ncount, int *bcount,
                                int nblocks)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *sets = S;
        *st = DevStatus();
    }
    for (int k = i; k < ncount; k += gridDim.x * blockDim.x) ccount[k] = 0;
    for (int k = i; k < nblocks; k += gridDim.x * blockDim.x) bcount[k] = 0;
}

extern "C" int dgt_global_triangulation_noalloc(const double *d_points, int n, double Lx, double Ly,
                                                double cell_size, int *d_tri, int *d_neighnum, int stride,
                                                int *out_required_stride, void *stream)
{
    if (out_required_stride) *out_required_stride = 0;
    if (n < 0 || !(Lx > 0) || !(Ly > 0) || !std::isfinite(Lx) || !std::isfinite(Ly) || !std::isfinite(cell_size))
        return DGT_ERR_INVALID_ARGUMENT;
    if (n == 0) return DGT_OK;
    if (n > NA_MAX_POINTS || !d_points || !d_tri || !d_neighnum || stride < 3 || stride > (1 << 16))
        return DGT_ERR_INVALID_ARGUMENT;
    // cell grid: the requested edge (mean spacing when cell_size <= 0), but no finer than ~4
    // cells per point, because the array holds a fixed number of cells (a context allows ~16);
    // the output does not depend on the cell size
    double spacing = std::sqrt(Lx * Ly / n);
    double a = cell_size > 0 ? cell_size : spacing;
    double amin = std::sqrt(Lx * Ly / (4.0 * n + 16.0));
    if (a < amin) a = amin;
    // judged in double before the conversion to int: a box of extreme aspect ratio can ask
    // for more cells along one axis than an int holds
    const double fxs = std::floor(Lx / a), fys = std::floor(Ly / a);
    if (!(fxs <= (double)NA_MAX_CELLS) || !(fys <= (double)NA_MAX_CELLS)) return DGT_ERR_INVALID_ARGUMENT;
    int xs = std::max(1, (int)fxs), ys = std::max(1, (int)fys);
    if ((long long)xs * ys > NA_MAX_CELLS) return DGT_ERR_INVALID_ARGUMENT;
    SetDesc S{};   // value-initialised: every field not set below (general box, ...) is zero
    S.Lx = Lx;
    S.Ly = Ly;
    S.hLx = 0.5 * Lx;
    S.hLy = 0.5 * Ly;
    S.xsize = xs;
    S.ysize = ys;
    S.cw = Lx / xs;
    S.ch = Ly / ys;
    S.icw = (double)xs / Lx;
    S.ich = (double)ys / Ly;
    S.cell_base = 0;
    S.point_base = 0;
    S.n = n;
    S.V = (float)pow2_at_least(std::max(Lx, Ly));
    const int blocks = set_block_grid(S, 0);
    const int cells = xs * ys;
    if ((size_t)blocks > NA_MAX_BLOCKS) return DGT_ERR_INVALID_ARGUMENT;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DGT_ERR_CUDA;
    unsigned char *base = nullptr;
    int rc = scratch_base(&base);
    if (rc != DGT_OK) return rc;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    cudaStream_t s = (cudaStream_t)stream;

    SetDesc *d_sets = reinterpret_cast<SetDesc *>(base + OFF_SETS);
    DevStatus *d_st = reinterpret_cast<DevStatus *>(base + OFF_STATUS);
    k_noalloc_setup<<<std::min((cells + 1 + 255) / 256, 1024), 256, 0, s>>>(S, d_sets, d_st,
                                                                          reinterpret_cast<int *>(base + OFF_CCOUNT),
                                                                          cells + 1,
                                                                          reinterpret_cast<int *>(base + OFF_BCOUNT),
                                                                          blocks);
    if (cudaGetLastError() != cudaSuccess) return DGT_ERR_CUDA;

    BinArgs b;
    b.pos = reinterpret_cast<const double2 *>(d_points);
    b.n = n;
    b.sets = d_sets;
    b.set_of = nullptr;
    b.total_cells = cells;
    b.ccount = reinterpret_cast<int *>(base + OFF_CCOUNT);
    b.cstart = reinterpret_cast<int *>(base + OFF_CSTART);
    b.cell_of = reinterpret_cast<int *>(base + OFF_CELLOF);
    b.rank = reinterpret_cast<int *>(base + OFF_RANK);
    b.sidx = reinterpret_cast<int *>(base + OFF_SIDX);
    b.slot_of = reinterpret_cast<int *>(base + OFF_SLOTOF);
    b.spos = reinterpret_cast<double2 *>(base + OFF_SPOS);
    b.block_sums = reinterpret_cast<int *>(base + OFF_BSUM);
    b.bcount = reinterpret_cast<int *>(base + OFF_BCOUNT);
    b.deterministic = 1;
    b.cond = nullptr;
    b.num_sets = 1;
    b.total_blocks = blocks;
    if (launch_bin_st(b, d_st, s) != cudaSuccess) return DGT_ERR_CUDA;

    RingArgs r;
    std::memset(&r, 0, sizeof(r));
    r.sets = d_sets;
    r.set_of = nullptr;
    r.pos = b.pos;
    r.spos = b.spos;
    r.sidx = b.sidx;
    r.slot_of = b.slot_of;
    r.cstart = b.cstart;
    r.bcount = b.bcount;
    r.tri = d_tri;
    r.nn = d_neighnum;
    r.stride = stride;
    r.npoints = n;
    r.n_items = n;
    r.defer_list = reinterpret_cast<int *>(base + OFF_DEFERLIST);
    r.defer_count = &d_st->defer_count;
    r.work_budget = DEFAULT_WORK_BUDGET;
    r.st = d_st;
    if (launch_build(r, MODE_F32, sms, 0, s) != cudaSuccess) return DGT_ERR_CUDA;
    if (launch_deferred(r, sms, s) != cudaSuccess) return DGT_ERR_CUDA;

    // status into host stack memory (pageable: no pinned buffer is allocated)
    DevStatus h;
    if (cudaMemcpyAsync(&h, d_st, sizeof(DevStatus), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DGT_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DGT_ERR_CUDA;
    if (h.err_flags & EF_BAD_INPUT) return DGT_ERR_BAD_POINTS;
    if (h.need_stride > 0) {
        if (out_required_stride) *out_required_stride = h.need_stride;
        return DGT_ERR_NEED_RESIZE;
    }
    if (h.err_flags & ~EF_MINIMAGE) return DGT_ERR_DEGENERATE;
    return DGT_OK;
}

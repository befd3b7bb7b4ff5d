/*
 * ref_harness.cu -- TEST INFRASTRUCTURE ONLY (oracle side, never the product).
 *
 * Links the reference's own sources (compiled in place by oracle/build_ref.sh into
 * oracle/_ref/libdgtref.so) and exposes two flavours of its CPU/OpenMP path behind a
 * plain C ABI so Python tests and bench.py's reference arm can drive it:
 *
 *  ref_fn_*  : calls the reference's kernel *callers* with GPUcompute=false
 *              (src/model/DelaunayGPU.cu:1116-1189 gpu_voronoi_calc,
 *               :1258-1317 gpu_get_neighbors, :1036-1114 gpu_voronoi_calc_no_sort,
 *               :1191-1256 gpu_get_neighbors_no_sort, :1346-1409 gpu_test_circumcircles).
 *              These run the reference's __host__ __device__ per-point functions in
 *              OpenMP loops over host pointers and need no CUDA device.  The bucket grid
 *              they read is filled here the way cellListGPU::setGridSize + compute(points)
 *              do it (src/utilities/cellListGPU.cpp:97-117, 289-330): even cell counts,
 *              points inserted in index order.  The triangle list is built the way
 *              DelaunayGPU::getCircumcirclesCPU does (src/model/DelaunayGPU.cpp:673-705).
 *
 *  ref_cls_* : drives the reference's public class DelaunayGPU unchanged
 *              (src/model/DelaunayGPU.h:22-58) with setGPUcompute(false) and
 *              setOMPthreads(k).  GPUArray allocates device memory, so these entry
 *              points need a CUDA device even though all arithmetic runs on the host.
 *
 *  ref_gpu_* : the same class with setGPUcompute(true) and setSafetyMode(true): the
 *              reference's own CUDA kernels (DelaunayGPU.cu:649-675 seed pass, :981-1006
 *              refine pass, :1008-1028 triangle list, :290-313 circle test, :611-640 and
 *              :945-975 repair passes; cellListGPU.cu:20-58 binning) compiled for sm_100a,
 *              timed with CUDA events on the legacy default stream the reference launches
 *              on.  Two guards keep its device writes in bounds (the reference has none for
 *              either):
 *                - the seed pass grows a polygon without checking the row capacity
 *                  (DelaunayGPU.cu:568-582); ref_fn_seed_max runs the same seed pass on the
 *                  host so a caller can check, before any GPU run, that the polygons of its
 *                  input stay far below MaxSize;
 *                - the triangle-list kernel appends into an array of exactly 2N entries
 *                  (DelaunayGPU.cpp:628, DelaunayGPU.cu:1021-1025); ref_gpu_triangles_ok
 *                  counts, on the host, the triangles of the class's current triangulation
 *                  the way DelaunayGPU::getCircumcirclesCPU does (DelaunayGPU.cpp:673-705),
 *                  and ref_gpu_repair refuses to run unless they are exactly 2N.
 */
#include <vector>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <omp.h>

#include "std_include.h"
#include "indexer.h"
#include "periodicBoundaries.h"
#include "DelaunayGPU.cuh"
#include "DelaunayGPU.h"
#include "hilbert_curve.hpp"

namespace {

struct BucketGrid {
    int xsize = 0, ysize = 0, nmax = 0, cells = 0;
    double boxsize = 0.0;
    std::vector<unsigned int> sizes;
    std::vector<int> idx;
};

// grid geometry as cellListGPU::setGridSize computes it, then an index-order fill with the
// same Nmax growth rule as cellListGPU::compute(points).  Bins are clamped like the GPU fill
// (cellListGPU.cu:41-42) so a coordinate that rounds to the box edge cannot index past the grid.
void fill_grid(BucketGrid &g, const double2 *pts, int n, double Lx, double Ly, double a)
{
    g.xsize = (int)floor(Lx / a);
    if (g.xsize % 2 == 1) g.xsize += 1;
    g.ysize = (int)floor(Ly / a);
    if (g.ysize % 2 == 1) g.ysize += 1;
    g.boxsize = Lx / g.xsize;
    g.cells = g.xsize * g.ysize;
    g.nmax = 0;
    if (std::ceil(n / g.cells) + 1 > g.nmax) g.nmax = (int)std::ceil(n / g.cells) + 3;
    bool again = true;
    while (again) {
        again = false;
        g.sizes.assign(g.cells, 0u);
        g.idx.assign((size_t)g.cells * g.nmax, 0);
        for (int i = 0; i < n; ++i) {
            if (again) continue;
            int ib = (int)floor(pts[i].x / g.boxsize);
            int jb = (int)floor(pts[i].y / g.boxsize);
            ib = std::max(0, std::min(g.xsize - 1, ib));
            jb = std::max(0, std::min(g.ysize - 1, jb));
            int bin = ib + g.xsize * jb;
            int off = (int)g.sizes[bin];
            if (off < g.nmax) g.idx[(size_t)bin * g.nmax + off] = i;
            else { g.nmax = std::max(g.nmax, off + 1); again = true; }
            g.sizes[bin]++;
        }
    }
}

}  // namespace

extern "C" {

/* Global triangulation through the reference's callers.  pts: n x (x,y) doubles.
   tri: n*stride ints (stride >= ring sizes; the host path has no overflow guard,
   DelaunayGPU.cu:911-918, so callers pass a generous stride).  Returns the largest
   ring size written. */
int ref_fn_global(const double *pts, int n, double Lx, double Ly, double cell_size,
                  int stride, int threads, int *tri, int *nn)
{
    const double2 *p = reinterpret_cast<const double2 *>(pts);
    BucketGrid g;
    fill_grid(g, p, n, Lx, Ly, cell_size);
    periodicBoundaries box(Lx, Ly);
    Index2D ci(g.xsize, g.ysize), cli(g.nmax, g.cells), ring(stride, n);
    std::vector<double2> P((size_t)stride * n), Q((size_t)stride * n);
    int maxRing = stride;
    gpu_voronoi_calc(const_cast<double2 *>(p), g.sizes.data(), g.idx.data(), tri, P.data(), Q.data(), nn,
                     n, g.xsize, g.ysize, g.boxsize, box, ci, cli, ring, false, (unsigned)threads);
    gpu_get_neighbors(const_cast<double2 *>(p), g.sizes.data(), g.idx.data(), tri, P.data(), Q.data(), nn,
                      n, g.xsize, g.ysize, g.boxsize, box, ci, cli, ring, &maxRing, stride, false,
                      (unsigned)threads);
    int mx = 0;
    for (int i = 0; i < n; ++i) mx = std::max(mx, nn[i]);
    return mx;
}

/* Test-and-repair through the reference's callers on an existing (tri, nn) of row stride
   `stride`: triangle list (DelaunayGPU.cpp:673-705 order), bucket fill, circumcircle test
   (DelaunayGPU.cu:192-284) with repair[] reset to -1, then the two passes restricted to
   repair[i] >= 0.  repair_out (n ints) receives the flags.  Returns the number of
   triangles enumerated (2n on a valid torus triangulation), or -1 if the triangle list
   would not fit 2n entries. */
int ref_fn_test_and_repair(const double *pts, int n, double Lx, double Ly, double cell_size,
                           int stride, int threads, int *tri, int *nn, int *repair_out)
{
    const double2 *p = reinterpret_cast<const double2 *>(pts);
    std::vector<int3> ccs((size_t)2 * n);
    int cidx = 0;
    for (int i = 0; i < n; ++i) {
        int m = nn[i];
        int3 c;
        c.x = i;
        c.y = tri[(size_t)i * stride + m - 1];
        for (int k = 0; k < m; ++k) {
            c.z = tri[(size_t)i * stride + k];
            if (c.x < c.y && c.x < c.z) {
                if (cidx >= 2 * n) return -1;
                ccs[cidx++] = c;
            }
            c.y = c.z;
        }
    }
    BucketGrid g;
    fill_grid(g, p, n, Lx, Ly, cell_size);
    periodicBoundaries box(Lx, Ly);
    Index2D ci(g.xsize, g.ysize), cli(g.nmax, g.cells), ring(stride, n);
    for (int i = 0; i < n; ++i) repair_out[i] = -1;
    /* only the enumerated triangles are tested: the class path throws unless there are
       exactly 2n (DelaunayGPU.cpp:701-705), and a zero-filled slot would describe a
       degenerate triangle whose circle is NaN */
    gpu_test_circumcircles(repair_out, ccs.data(), cidx, const_cast<double2 *>(p), g.sizes.data(),
                           g.idx.data(), n, g.xsize, g.ysize, g.boxsize, box, ci, cli, false,
                           (unsigned)threads);
    std::vector<double2> P((size_t)stride * n), Q((size_t)stride * n);
    int maxRing = stride;
    gpu_voronoi_calc_no_sort(const_cast<double2 *>(p), g.sizes.data(), g.idx.data(), tri, P.data(), Q.data(),
                             nn, n, g.xsize, g.ysize, g.boxsize, box, ci, cli, repair_out, ring, false,
                             (unsigned)threads);
    gpu_get_neighbors_no_sort(const_cast<double2 *>(p), g.sizes.data(), g.idx.data(), tri, P.data(), Q.data(),
                              nn, n, g.xsize, g.ysize, g.boxsize, box, ci, cli, repair_out, ring,
                              &maxRing, stride, false, (unsigned)threads);
    return cidx;
}

/* ---- the reference's public class, unchanged (needs a CUDA device for GPUArray) ---- */
struct RefCls {
    DelaunayGPU *del = nullptr;
    GPUArray<double2> pts;
    GPUArray<int> tri, nn;
    int n = 0;
};

void *ref_cls_create(int n, int max_neighs, double cell_size, double Lx, double Ly, int threads)
{
    try {
        RefCls *r = new RefCls();
        r->n = n;
        PeriodicBoxPtr box = make_shared<periodicBoundaries>(Lx, Ly);
        r->del = new DelaunayGPU(n, max_neighs, cell_size, box);
        r->del->setGPUcompute(false);
        r->del->setOMPthreads((unsigned)threads);
        r->del->setSafetyMode(true);
        r->pts.resize(n);
        r->tri.resize((unsigned)(max_neighs * n));
        r->nn.resize(n);
        return r;
    } catch (...) {
        return nullptr;
    }
}

static void cls_upload(RefCls *r, const double *pts)
{
    ArrayHandle<double2> h(r->pts, access_location::host, access_mode::overwrite);
    std::memcpy(h.data, pts, sizeof(double2) * (size_t)r->n);
}

static int cls_download(RefCls *r, int *tri, int *nn, int stride)
{
    int rowlen = (int)(r->tri.getNumElements() / r->n);
    ArrayHandle<int> ht(r->tri, access_location::host, access_mode::read);
    ArrayHandle<int> hn(r->nn, access_location::host, access_mode::read);
    int mx = 0;
    for (int i = 0; i < r->n; ++i) {
        nn[i] = hn.data[i];
        mx = std::max(mx, nn[i]);
        for (int k = 0; k < std::min(rowlen, stride); ++k)
            tri[(size_t)i * stride + k] = ht.data[(size_t)i * rowlen + k];
    }
    return mx;
}

/* globalDelaunayTriangulation on host buffers; returns the largest ring, -1 on error. */
int ref_cls_global(void *h, const double *pts, int *tri, int *nn, int stride)
{
    try {
        RefCls *r = static_cast<RefCls *>(h);
        cls_upload(r, pts);
        r->del->globalDelaunayTriangulation(r->pts, r->tri, r->nn);
        return tri ? cls_download(r, tri, nn, stride) : 0;
    } catch (...) {
        return -1;
    }
}

/* testAndRepairDelaunayTriangulation on the class's current triangulation with new
   positions; returns the largest ring, -1 on error. */
int ref_cls_test_and_repair(void *h, const double *pts, int *tri, int *nn, int stride)
{
    try {
        RefCls *r = static_cast<RefCls *>(h);
        cls_upload(r, pts);
        r->del->testAndRepairDelaunayTriangulation(r->pts, r->tri, r->nn);
        return tri ? cls_download(r, tri, nn, stride) : 0;
    } catch (...) {
        return -1;
    }
}

void ref_cls_destroy(void *h)
{
    RefCls *r = static_cast<RefCls *>(h);
    if (!r) return;
    delete r->del;
    delete r;
}

int ref_omp_max_threads(void) { return omp_get_max_threads(); }

/* The reference's seed pass alone (gpu_voronoi_calc on the host, DelaunayGPU.cu:1116-1189),
   over all points: returns the largest candidate polygon it builds (its rows have no
   capacity check), or -1 when that reaches `stride` (the scratch rows here are `stride`
   wide, so a larger polygon could not be measured; one spare row at the end keeps an
   overflow of the last point inside the allocation). */
int ref_fn_seed_max(const double *pts, int n, double Lx, double Ly, double cell_size, int stride, int threads)
{
    const double2 *p = reinterpret_cast<const double2 *>(pts);
    BucketGrid g;
    fill_grid(g, p, n, Lx, Ly, cell_size);
    periodicBoundaries box(Lx, Ly);
    Index2D ci(g.xsize, g.ysize), cli(g.nmax, g.cells), ring(stride, n);
    std::vector<double2> P((size_t)stride * (n + 1)), Q((size_t)stride * (n + 1));
    std::vector<int> tri((size_t)stride * (n + 1)), nn(n);
    gpu_voronoi_calc(const_cast<double2 *>(p), g.sizes.data(), g.idx.data(), tri.data(), P.data(), Q.data(),
                     nn.data(), n, g.xsize, g.ysize, g.boxsize, box, ci, cli, ring, false, (unsigned)threads);
    int mx = 0;
    for (int i = 0; i < n; ++i) mx = std::max(mx, nn[i]);
    return mx >= stride ? -1 : mx;
}

/* ---- the reference's public class on its GPU path (its own CUDA kernels) ---- */
struct RefGpu {
    DelaunayGPU *del = nullptr;
    GPUArray<double2> p0, p1;
    GPUArray<int> tri, nn;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int n = 0;
};

/* p0: the points of the global triangulation, p1: the moved points of the repair (both
   n x (x,y) doubles, copied to the device here, outside any timing). */
void *ref_gpu_create(int n, int max_neighs, double cell_size, double Lx, double Ly, const double *p0,
                     const double *p1)
{
    try {
        RefGpu *r = new RefGpu();
        r->n = n;
        PeriodicBoxPtr box = make_shared<periodicBoundaries>(Lx, Ly);
        r->del = new DelaunayGPU(n, max_neighs, cell_size, box);
        r->del->setGPUcompute(true);
        r->del->setSafetyMode(true);
        r->p0.resize(n);
        r->p1.resize(n);
        r->tri.resize((unsigned)(max_neighs * n));
        r->nn.resize(n);
        {
            ArrayHandle<double2> h0(r->p0, access_location::host, access_mode::overwrite);
            ArrayHandle<double2> h1(r->p1, access_location::host, access_mode::overwrite);
            std::memcpy(h0.data, p0, sizeof(double2) * (size_t)n);
            std::memcpy(h1.data, p1, sizeof(double2) * (size_t)n);
        }
        {   // resident on the device before the first timed call
            ArrayHandle<double2> d0(r->p0, access_location::device, access_mode::read);
            ArrayHandle<double2> d1(r->p1, access_location::device, access_mode::read);
        }
        if (cudaEventCreate(&r->e0) != cudaSuccess || cudaEventCreate(&r->e1) != cudaSuccess) return nullptr;
        if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
        return r;
    } catch (...) {
        return nullptr;
    }
}

static int gpu_timed(RefGpu *r, bool build, float *ms)
{
    cudaEventRecord(r->e0, 0);
    if (build) r->del->globalDelaunayTriangulation(r->p0, r->tri, r->nn);
    else r->del->testAndRepairDelaunayTriangulation(r->p1, r->tri, r->nn);
    cudaEventRecord(r->e1, 0);
    if (cudaEventSynchronize(r->e1) != cudaSuccess) return -1;
    if (cudaGetLastError() != cudaSuccess) return -1;
    if (ms) cudaEventElapsedTime(ms, r->e0, r->e1);
    return 0;
}

/* globalDelaunayTriangulation(p0) on the GPU; *ms = device time.  0, or -1 on error. */
int ref_gpu_build(void *h, float *ms)
{
    try {
        return gpu_timed(static_cast<RefGpu *>(h), true, ms);
    } catch (...) {
        return -1;
    }
}

/* 1 when the class's current triangulation has exactly 2N triangles by smallest-index
   ownership, ring sizes summing to 6N and every entry a valid index: the input the
   triangle-list kernel can take without writing past its 2N-entry array. */
int ref_gpu_triangles_ok(void *h)
{
    try {
        RefGpu *r = static_cast<RefGpu *>(h);
        const int n = r->n;
        const long long rowlen = (long long)(r->tri.getNumElements() / n);
        ArrayHandle<int> ht(r->tri, access_location::host, access_mode::read);
        ArrayHandle<int> hn(r->nn, access_location::host, access_mode::read);
        long long tris = 0, deg = 0;
        for (int i = 0; i < n; ++i) {
            const int m = hn.data[i];
            if (m < 3 || m > rowlen) return 0;
            deg += m;
            const int *row = ht.data + (size_t)i * rowlen;
            for (int k = 0; k < m; ++k)
                if (row[k] < 0 || row[k] >= n) return 0;
            int y = row[m - 1];
            for (int k = 0; k < m; ++k) {
                const int z = row[k];
                if (i < y && i < z) tris++;
                y = z;
            }
        }
        return (tris == 2LL * n && deg == 6LL * n) ? 1 : 0;
    } catch (...) {
        return 0;
    }
}

/* testAndRepairDelaunayTriangulation(p1) on the GPU, on the class's current triangulation;
   refused (-2) unless ref_gpu_triangles_ok holds for it.  *ms = device time. */
int ref_gpu_repair(void *h, float *ms)
{
    try {
        if (ref_gpu_triangles_ok(h) != 1) return -2;
        return gpu_timed(static_cast<RefGpu *>(h), false, ms);
    } catch (...) {
        return -1;
    }
}

/* the class's current rings into tri (n x stride) and nn; returns its row length MaxSize */
int ref_gpu_fetch(void *h, int *tri, int *nn, int stride)
{
    try {
        RefGpu *r = static_cast<RefGpu *>(h);
        const int rowlen = (int)(r->tri.getNumElements() / r->n);
        ArrayHandle<int> ht(r->tri, access_location::host, access_mode::read);
        ArrayHandle<int> hn(r->nn, access_location::host, access_mode::read);
        for (int i = 0; i < r->n; ++i) {
            nn[i] = hn.data[i];
            for (int k = 0; k < std::min(rowlen, stride); ++k)
                tri[(size_t)i * stride + k] = ht.data[(size_t)i * rowlen + k];
        }
        return rowlen;
    } catch (...) {
        return -1;
    }
}

void ref_gpu_destroy(void *h)
{
    RefGpu *r = static_cast<RefGpu *>(h);
    if (!r) return;
    if (r->e0) cudaEventDestroy(r->e0);
    if (r->e1) cudaEventDestroy(r->e1);
    delete r->del;
    delete r;
}

/* The reference's Hilbert index of square (x, y) of a 2^m x 2^m grid
   (src/utilities/hilbert_curve.cpp:229; the key of its hilbertSortArray pre-pass). */
int ref_xy2d(int m, int x, int y) { return xy2d(m, x, y); }

}  // extern "C"

// dgt_delaunay.hpp -- header-only C++ adapter with the reference's DelaunayGPU interface
// (src/model/DelaunayGPU.h:18-130) over the C ABI of include/dgt.h.
//
// Existing host code keeps its calls:
//     dgt::DelaunayGPU delGPU(N, maxNeighs, cellSize, domain);      // DelaunayGPU.h:25
//     delGPU.setSafetyMode(true);                                   // :46
//     delGPU.globalDelaunayTriangulation(points, tri, neighNum);    // :30
//     delGPU.testAndRepairDelaunayTriangulation(points, tri, neighNum);  // :33
//     int m = delGPU.MaxSize;                                       // :55 (public member)
//     delGPU.Box->putInBoxReal(p);                                  // :53 (public member)
// The blank constructor plus initialize(N, maxNeighs, cellSize, box) (:23, :36) work too.
// `Box` holds the box object the class was given: with dgt::DelaunayGPUT<PeriodicBoxPtr> it is
// the caller's own PeriodicBoxPtr; the default dgt::DelaunayGPU keeps a dgt::BoxDims copy of
// the box (getBoxDims, isBoxSquare, putInBoxReal of a rectangular or general box).
// The array arguments can be any container for which dgt::array_traits is specialised
// (device pointer, element count, resize).  DeviceArray below is a minimal owning one;
// include/dgt_gpuarray.hpp specialises it for the reference's GPUArray<T>.
// Like the reference, the triangulation array may be resized by the callee to MaxSize*N
// (DelaunayGPU.cpp:126-132, :152-155) and errors throw std::runtime_error
// (inc/std_include.h:61-72 throws on CUDA errors).
#ifndef DGT_DELAUNAY_HPP
#define DGT_DELAUNAY_HPP

#include <cuda_runtime_api.h>

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "dgt.h"

namespace dgt {

template <class Array> struct array_traits;   // specialise: device_ptr, size, resize

// minimal owning device array (element type T, contents undefined after resize)
template <class T> class DeviceArray {
  public:
    DeviceArray() = default;
    explicit DeviceArray(size_t n) { resize(n); }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    ~DeviceArray() { release(); }
    void resize(size_t n)
    {
        if (n == n_) return;
        release();
        if (n) {
            if (cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)) != cudaSuccess)
                throw std::runtime_error("DeviceArray: cudaMalloc failed");
            cudaMemset(p_, 0, n * sizeof(T));
        }
        n_ = n;
    }
    size_t getNumElements() const { return n_; }
    T *data() { return p_; }
    const T *data() const { return p_; }
    void upload(const T *h, size_t n)
    {
        resize(n);
        if (n && cudaMemcpy(p_, h, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("DeviceArray: upload failed");
    }
    void download(T *h) const
    {
        if (n_ && cudaMemcpy(h, p_, n_ * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("DeviceArray: download failed");
    }

  private:
    void release()
    {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T *p_ = nullptr;
    size_t n_ = 0;
};

template <class T> struct array_traits<DeviceArray<T>> {
    static T *device_ptr(DeviceArray<T> &a) { return a.data(); }
    static size_t size(const DeviceArray<T> &a) { return a.getNumElements(); }
    static void resize(DeviceArray<T> &a, size_t n) { a.resize(n); }
};

// A periodic box by its matrix (xx, xy, yx, yy): lattice vectors (xx, yx) and (xy, yy), the
// argument order of periodicBoundaries(a, b, c, d) (periodicBoundaries.h:30-31).
struct BoxDims {
    double xx = 0, xy = 0, yx = 0, yy = 0;
    BoxDims() = default;
    BoxDims(double a, double b, double c, double d) : xx(a), xy(b), yx(c), yy(d) {}
    void getBoxDims(double &a, double &b, double &c, double &d) const
    {
        a = xx;
        b = xy;
        c = yx;
        d = yy;
    }
    bool isBoxSquare() const { return xy == 0.0 && yx == 0.0; }
    // the point moved into the primary cell [0, 1)^2 in fractional coordinates
    // (periodicBoundaries::putInBoxReal, periodicBoundaries.h:131-152)
    void putInBoxReal(double2 &p) const
    {
        if (isBoxSquare()) {
            p.x = wrap(p.x, xx);
            p.y = wrap(p.y, yy);
            return;
        }
        const double det = xx * yy - xy * yx;
        const double u = wrap((yy * p.x - xy * p.y) / det, 1.0), v = wrap((-yx * p.x + xx * p.y) / det, 1.0);
        p.x = xx * u + xy * v;
        p.y = yx * u + yy * v;
    }

  private:
    static double wrap(double x, double L)
    {
        x -= L * std::floor(x / L);
        if (x >= L) x -= L;
        if (x < 0) x += L;
        return x;
    }
};

// The class's phase profiler (the reference's `prof`, DelaunayGPU.h:51, a multiProfiler):
// here the library's own per-phase device times of the last call, recorded when enabled.
class PhaseProfiler {
  public:
    explicit PhaseProfiler(dgt_context **ctx) : ctx_(ctx) {}
    void enable(bool on) { if (*ctx_) dgt_set_timing(*ctx_, on ? 1 : 0); }
    // the reference brackets its sections by name; the library times its own phases
    void start(const std::string &) {}
    void end(const std::string &) {}
    void print() const
    {
        double ms[DGT_NUM_PHASES];
        if (!*ctx_ || dgt_get_phase_times(*ctx_, ms) != DGT_OK) return;
        static const char *names[DGT_NUM_PHASES] = { "cell grid", "one-ring build", "deferred points",
                                                     "local test", "repair rounds" };
        for (int i = 0; i < DGT_NUM_PHASES; ++i)
            if (ms[i] >= 0) std::printf("%s: %.4f ms\n", names[i], ms[i]);
    }

  private:
    dgt_context **ctx_;
};

template <class BoxPtr> class DelaunayGPUT {
  public:
    //! blank constructor (DelaunayGPU.h:23); initialize() before use
    DelaunayGPUT() = default;
    //! DelaunayGPU(int N, int maximumNeighborsGuess, double cellSize, PeriodicBoxPtr bx) (:25)
    template <class AnyBoxPtr>
    DelaunayGPUT(int N, int maximumNeighborsGuess, double cellSize, const AnyBoxPtr &bx)
    {
        initialize(N, maximumNeighborsGuess, cellSize, bx);
    }
    //! a rectangular box by its sides
    DelaunayGPUT(int N, int maximumNeighborsGuess, double cellSize, double Lx, double Ly)
    {
        initialize(N, maximumNeighborsGuess, cellSize, std::make_shared<BoxDims>(Lx, 0.0, 0.0, Ly));
    }
    DelaunayGPUT(const DelaunayGPUT &) = delete;
    DelaunayGPUT &operator=(const DelaunayGPUT &) = delete;
    ~DelaunayGPUT() { dgt_destroy(ctx_); }

    //! initialize(N, maximumNeighborsGuess, cellSize, bx) (DelaunayGPU.h:36): a fresh context
    //! (any earlier one is released); `bx` is any pointer to an object with getBoxDims
    template <class AnyBoxPtr>
    void initialize(int N, int maximumNeighborsGuess, double cellSize, const AnyBoxPtr &bx)
    {
        double xx, xy, yx, yy;
        (*bx).getBoxDims(xx, xy, yx, yy);
        dgt_context *c = nullptr;
        if (xy == 0.0 && yx == 0.0) {
            check(dgt_create(N, maximumNeighborsGuess, cellSize, xx, yy, &c), "dgt_create");
        } else {
            // a general box (periodicBoundaries::setGeneral): created on the bounding
            // rectangle, then given the box matrix
            check(dgt_create(N, maximumNeighborsGuess, cellSize, std::fabs(xx) + std::fabs(xy),
                             std::fabs(yx) + std::fabs(yy), &c), "dgt_create");
            const int rc = dgt_set_box_general(c, xx, xy, yx, yy);
            if (rc != DGT_OK) {
                dgt_destroy(c);
                check(rc, "setBox");
            }
        }
        dgt_destroy(ctx_);
        ctx_ = c;
        n_ = N;
        if (!safety_) dgt_set_safety_mode(ctx_, 0);
        Box = keep_box(bx, xx, xy, yx, yy);
        sync();
    }

    template <class PointArray, class IntArray>
    void globalDelaunayTriangulation(PointArray &points, IntArray &tri, IntArray &neighNum)
    {
        if (n_ == 0) return;
        fit(tri, neighNum);
        for (;;) {
            int stride = (int)(array_traits<IntArray>::size(tri) / n_);
            int r = dgt_global_triangulation(ctx(), pts(points), array_traits<IntArray>::device_ptr(tri),
                                             array_traits<IntArray>::device_ptr(neighNum), stride, stream_);
            sync();
            if (r == DGT_ERR_NEED_RESIZE && safety_) {
                array_traits<IntArray>::resize(tri, (size_t)MaxSize * n_);
                continue;
            }
            check(r, "globalDelaunayTriangulation");
            return;
        }
    }

    template <class PointArray, class IntArray>
    void testAndRepairDelaunayTriangulation(PointArray &points, IntArray &tri, IntArray &neighNum)
    {
        if (n_ == 0) return;
        for (;;) {
            int stride = (int)(array_traits<IntArray>::size(tri) / n_);
            int *t = array_traits<IntArray>::device_ptr(tri);
            int *nn = array_traits<IntArray>::device_ptr(neighNum);
            int r = dgt_test_and_repair(ctx(), pts(points), t, nn, stride, stream_);
            sync();
            if (r == DGT_ERR_NEED_RESIZE && safety_) {
                // grow keeping every row in place (re-strided copy, not a linear one)
                int ns = MaxSize;
                int *tmp = nullptr;
                if (cudaMalloc(reinterpret_cast<void **>(&tmp), sizeof(int) * (size_t)n_ * stride) != cudaSuccess)
                    throw std::runtime_error("testAndRepair: cudaMalloc failed");
                cudaMemcpyAsync(tmp, t, sizeof(int) * (size_t)n_ * stride, cudaMemcpyDeviceToDevice,
                                (cudaStream_t)stream_);
                array_traits<IntArray>::resize(tri, (size_t)ns * n_);
                int rs = dgt_restride(tmp, stride, array_traits<IntArray>::device_ptr(tri), ns, nn, n_, stream_);
                cudaStreamSynchronize((cudaStream_t)stream_);
                cudaFree(tmp);
                check(rs, "dgt_restride");
                continue;
            }
            check(r, "testAndRepairDelaunayTriangulation");
            return;
        }
    }

    template <class PointArray> void updateList(PointArray &points)
    {
        check(dgt_update_list(ctx(), pts(points), stream_), "updateList");
    }
    void resize(int nmax)
    {
        check(dgt_resize(ctx(), nmax), "resize");
        sync();
    }
    void setCellListSize(double csize) { check(dgt_set_cell_size(ctx(), csize), "setCellListSize"); }
    void setBox(double Lx, double Ly)
    {
        check(dgt_set_box(ctx(), Lx, Ly), "setBox");
        Box = keep_box(std::make_shared<BoxDims>(Lx, 0.0, 0.0, Ly), Lx, 0.0, 0.0, Ly);
    }
    // setBox(bx) (DelaunayGPU.h:44) with any box type with getBoxDims, rectangular or general
    template <class AnyBoxPtr>
    void setBox(const AnyBoxPtr &bx)
    {
        double xx, xy, yx, yy;
        (*bx).getBoxDims(xx, xy, yx, yy);
        if (xy == 0.0 && yx == 0.0) check(dgt_set_box(ctx(), xx, yy), "setBox");
        else check(dgt_set_box_general(ctx(), xx, xy, yx, yy), "setBox");
        Box = keep_box(bx, xx, xy, yx, yy);
    }
    void setSafetyMode(bool on)
    {
        safety_ = on;
        if (ctx_) check(dgt_set_safety_mode(ctx_, on ? 1 : 0), "setSafetyMode");
    }
    // the reference can run on the host instead; this library is GPU-only
    void setGPUcompute(bool flag)
    {
        if (!flag) throw std::invalid_argument("DelaunayGPU: no CPU path");
    }
    void setOMPthreads(unsigned int) {}
    void setPrecision(int precision) { check(dgt_set_precision(ctx(), precision), "setPrecision"); }
    void setStream(cudaStream_t s) { stream_ = s; }
    // knobs without a reference counterpart (include/dgt.h); none changes the output
    void setFlipRepair(bool on) { check(dgt_set_flip_repair(ctx(), on ? 1 : 0), "setFlipRepair"); }
    void setWorkBudget(int budget) { check(dgt_set_work_budget(ctx(), budget), "setWorkBudget"); }
    void setGraphFlipRounds(int rounds) { check(dgt_set_graph_flip_rounds(ctx(), rounds), "setGraphFlipRounds"); }
    void setCheckMode(bool on) { check(dgt_set_check_mode(ctx(), on ? 1 : 0), "setCheckMode"); }
    void setDeferredOverlap(int chunks) { check(dgt_set_deferred_overlap(ctx(), chunks), "setDeferredOverlap"); }
    //! the reference driver's hilbertSortArray (triangulation.cpp:63-88) on the device: the
    //! points reordered in place along a Hilbert curve over the box (triangulate again after)
    template <class PointArray> void hilbertSortArray(PointArray &points)
    {
        check(dgt_hilbert_sort_points(ctx(), const_cast<double *>(pts(points)), nullptr, stream_),
              "hilbertSortArray");
    }
    //! the ring capacity as the library holds it (the same value as the MaxSize member)
    int getMaxSize() const
    {
        int v = 0;
        if (ctx_) dgt_get_max_size(ctx_, &v);
        return v;
    }
    dgt_stats stats()
    {
        dgt_stats s;
        check(dgt_get_stats(ctx(), &s), "dgt_get_stats");
        return s;
    }
    dgt_context *handle() { return ctx_; }

    //! public members of the reference class (DelaunayGPU.h:51-55)
    PhaseProfiler prof{ &ctx_ };
    BoxPtr Box{};
    int MaxSize = 0;   //!< ring capacity; kept equal to the library's after every call

  private:
    static void check(int r, const char *where)
    {
        if (r != DGT_OK) throw std::runtime_error(std::string(where) + ": " + dgt_error_string(r));
    }
    dgt_context *ctx()
    {
        if (!ctx_) throw std::logic_error("DelaunayGPU: initialize() was not called");
        return ctx_;
    }
    void sync() { MaxSize = getMaxSize(); }
    // Box keeps the caller's pointer when it converts to BoxPtr, else a BoxDims copy
    template <class AnyBoxPtr>
    static BoxPtr keep_box(const AnyBoxPtr &bx, double, double, double, double,
                           typename std::enable_if<std::is_convertible<AnyBoxPtr, BoxPtr>::value>::type * = nullptr)
    {
        return bx;
    }
    template <class AnyBoxPtr>
    static BoxPtr keep_box(const AnyBoxPtr &, double xx, double xy, double yx, double yy,
                           typename std::enable_if<!std::is_convertible<AnyBoxPtr, BoxPtr>::value>::type * = nullptr)
    {
        return make_dims(xx, xy, yx, yy, (BoxPtr *)nullptr);
    }
    static std::shared_ptr<BoxDims> make_dims(double xx, double xy, double yx, double yy, std::shared_ptr<BoxDims> *)
    {
        return std::make_shared<BoxDims>(xx, xy, yx, yy);
    }
    template <class Other> static Other make_dims(double, double, double, double, Other *) { return Other{}; }
    template <class PointArray> const double *pts(PointArray &points)
    {
        if (array_traits<PointArray>::size(points) != (size_t)n_)
            throw std::invalid_argument("DelaunayGPU: points array has the wrong size");
        return reinterpret_cast<const double *>(array_traits<PointArray>::device_ptr(points));
    }
    template <class IntArray> void fit(IntArray &tri, IntArray &nn)
    {
        if (array_traits<IntArray>::size(nn) != (size_t)n_) array_traits<IntArray>::resize(nn, n_);
        size_t t = array_traits<IntArray>::size(tri);
        if (t % n_ != 0 || t / n_ < (size_t)MaxSize) array_traits<IntArray>::resize(tri, (size_t)MaxSize * n_);
    }

    dgt_context *ctx_ = nullptr;
    int n_ = 0;
    bool safety_ = true;
    void *stream_ = nullptr;
};

//! the adapter with the box kept as a dgt::BoxDims copy
using DelaunayGPU = DelaunayGPUT<std::shared_ptr<BoxDims>>;

}  // namespace dgt

#endif  // DGT_DELAUNAY_HPP

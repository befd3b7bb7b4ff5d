// dgt_delaunay.hpp -- header-only C++ adapter with the reference's DelaunayGPU interface
// (src/model/DelaunayGPU.h:18-130) over the C ABI of include/dgt.h.
//
// Existing host code keeps its calls:
//     dgt::DelaunayGPU delGPU(N, maxNeighs, cellSize, Lx, Ly);   // DelaunayGPU.h:25
//     delGPU.setSafetyMode(true);                                   // :46
//     delGPU.globalDelaunayTriangulation(points, tri, neighNum);    // :30
//     delGPU.testAndRepairDelaunayTriangulation(points, tri, neighNum);  // :33
// The array arguments can be any container for which dgt::array_traits is specialised
// (device pointer, element count, resize).  DeviceArray below is a minimal owning one; a
// specialisation for the reference's GPUArray<T> is a few lines (see the integration notes).
// Like the reference, the triangulation array may be resized by the callee to MaxSize*N
// (DelaunayGPU.cpp:126-132, :152-155) and errors throw std::runtime_error
// (inc/std_include.h:61-72 throws on CUDA errors).
#ifndef DGT_DELAUNAY_HPP
#define DGT_DELAUNAY_HPP

#include <cuda_runtime_api.h>

#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>

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

class DelaunayGPU {
  public:
    // DelaunayGPU(int N, int maximumNeighborsGuess, double cellSize, PeriodicBoxPtr bx)
    DelaunayGPU(int N, int maximumNeighborsGuess, double cellSize, double Lx, double Ly) : n_(N)
    {
        check(dgt_create(N, maximumNeighborsGuess, cellSize, Lx, Ly, &ctx_), "dgt_create");
    }
    // any box type with getBoxDims(xx, xy, yx, yy) (periodicBoundaries.h:34-35), or a
    // pointer to one (PeriodicBoxPtr)
    template <class BoxPtr>
    DelaunayGPU(int N, int maximumNeighborsGuess, double cellSize, const BoxPtr &box) : n_(N)
    {
        double xx, xy, yx, yy;
        (*box).getBoxDims(xx, xy, yx, yy);
        if (xy == 0.0 && yx == 0.0) {
            check(dgt_create(N, maximumNeighborsGuess, cellSize, xx, yy, &ctx_), "dgt_create");
            return;
        }
        // a general box (periodicBoundaries::setGeneral): created on the bounding rectangle,
        // then given the box matrix
        check(dgt_create(N, maximumNeighborsGuess, cellSize, std::fabs(xx) + std::fabs(xy),
                         std::fabs(yx) + std::fabs(yy), &ctx_), "dgt_create");
        const int rc = dgt_set_box_general(ctx_, xx, xy, yx, yy);
        if (rc != DGT_OK) {
            dgt_destroy(ctx_);
            ctx_ = nullptr;
            check(rc, "setBox");
        }
    }
    DelaunayGPU(const DelaunayGPU &) = delete;
    DelaunayGPU &operator=(const DelaunayGPU &) = delete;
    ~DelaunayGPU() { dgt_destroy(ctx_); }

    template <class PointArray, class IntArray>
    void globalDelaunayTriangulation(PointArray &points, IntArray &tri, IntArray &neighNum)
    {
        if (n_ == 0) return;
        fit(tri, neighNum);
        for (;;) {
            int stride = (int)(array_traits<IntArray>::size(tri) / n_);
            int r = dgt_global_triangulation(ctx_, pts(points), array_traits<IntArray>::device_ptr(tri),
                                             array_traits<IntArray>::device_ptr(neighNum), stride, stream_);
            if (r == DGT_ERR_NEED_RESIZE && safety_) {
                array_traits<IntArray>::resize(tri, (size_t)MaxSize() * n_);
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
            int r = dgt_test_and_repair(ctx_, pts(points), t, nn, stride, stream_);
            if (r == DGT_ERR_NEED_RESIZE && safety_) {
                // grow keeping every row in place (re-strided copy, not a linear one)
                int ns = MaxSize();
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
        check(dgt_update_list(ctx_, pts(points), stream_), "updateList");
    }
    void resize(int nmax) { check(dgt_resize(ctx_, nmax), "resize"); }
    void setCellListSize(double csize) { check(dgt_set_cell_size(ctx_, csize), "setCellListSize"); }
    void setBox(double Lx, double Ly) { check(dgt_set_box(ctx_, Lx, Ly), "setBox"); }
    // setBox(bx) (DelaunayGPU.h:44) with any box type with getBoxDims, rectangular or general
    template <class BoxPtr>
    void setBox(const BoxPtr &box)
    {
        double xx, xy, yx, yy;
        (*box).getBoxDims(xx, xy, yx, yy);
        if (xy == 0.0 && yx == 0.0) check(dgt_set_box(ctx_, xx, yy), "setBox");
        else check(dgt_set_box_general(ctx_, xx, xy, yx, yy), "setBox");
    }
    void setSafetyMode(bool on)
    {
        safety_ = on;
        check(dgt_set_safety_mode(ctx_, on ? 1 : 0), "setSafetyMode");
    }
    // the reference can run on the host instead; this library is GPU-only
    void setGPUcompute(bool flag)
    {
        if (!flag) throw std::invalid_argument("DelaunayGPU: no CPU path");
    }
    void setOMPthreads(unsigned int) {}
    void setPrecision(int precision) { check(dgt_set_precision(ctx_, precision), "setPrecision"); }
    void setStream(cudaStream_t s) { stream_ = s; }
    // knobs without a reference counterpart (include/dgt.h); none changes the output
    void setFlipRepair(bool on) { check(dgt_set_flip_repair(ctx_, on ? 1 : 0), "setFlipRepair"); }
    void setWorkBudget(int budget) { check(dgt_set_work_budget(ctx_, budget), "setWorkBudget"); }
    void setGraphFlipRounds(int rounds) { check(dgt_set_graph_flip_rounds(ctx_, rounds), "setGraphFlipRounds"); }
    void setCheckMode(bool on) { check(dgt_set_check_mode(ctx_, on ? 1 : 0), "setCheckMode"); }
    int MaxSize() const
    {
        int v = 0;
        dgt_get_max_size(ctx_, &v);
        return v;
    }
    dgt_stats stats()
    {
        dgt_stats s;
        check(dgt_get_stats(ctx_, &s), "dgt_get_stats");
        return s;
    }
    dgt_context *handle() { return ctx_; }

  private:
    static void check(int r, const char *where)
    {
        if (r != DGT_OK) throw std::runtime_error(std::string(where) + ": " + dgt_error_string(r));
    }
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
        if (t % n_ != 0 || t / n_ < (size_t)MaxSize()) array_traits<IntArray>::resize(tri, (size_t)MaxSize() * n_);
    }

    dgt_context *ctx_ = nullptr;
    int n_ = 0;
    bool safety_ = true;
    void *stream_ = nullptr;
};

}  // namespace dgt

#endif  // DGT_DELAUNAY_HPP

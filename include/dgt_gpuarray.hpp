// dgt_gpuarray.hpp -- dgt::array_traits for the reference's GPUArray<T> container
// (inc/gpuarray.h:429-551), so host code that keeps its GPUArray buffers can hand them to the
// C++ adapter of include/dgt_delaunay.hpp unchanged:
//     #include "gpuarray.h"          // the reference's container (ENABLE_CUDA defined)
//     #include "dgt_gpuarray.hpp"
//     dgt::DelaunayGPUT<PeriodicBoxPtr> delGPU(N, maxNeighs, cellSize, domain);
//     delGPU.globalDelaunayTriangulation(gpuPts, gpuTriangulation, cellNeighborNumber);
// The device pointer comes from the container's own ArrayHandle with device read-write
// access: the handle brings the data to the device if the host copy is newer, marks the host
// copy stale, and leaves the pointer valid after the handle is released (the adapter's call
// runs right after, on the same device).  Resizing goes through GPUArray::resize, which
// keeps the leading elements (the adapter only resizes to grow the ring rows, then
// recomputes or re-strides them itself).
#ifndef DGT_GPUARRAY_HPP
#define DGT_GPUARRAY_HPP

#include "dgt_delaunay.hpp"

namespace dgt {

template <class T> struct array_traits<GPUArray<T>> {
    static T *device_ptr(GPUArray<T> &a)
    {
        ArrayHandle<T> h(a, access_location::device, access_mode::readwrite);
        return h.data;
    }
    static size_t size(const GPUArray<T> &a) { return a.getNumElements(); }
    static void resize(GPUArray<T> &a, size_t n) { a.resize((unsigned int)n); }
};

}  // namespace dgt

#endif  // DGT_GPUARRAY_HPP

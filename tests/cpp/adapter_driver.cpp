// Drives the C++ adapter (include/dgt_delaunay.hpp) the way the reference's driver drives its
// DelaunayGPU class (triangulation.cpp:224-246, :299, :327-345, :390): construct, safety mode
// on, global triangulation, new positions, test-and-repair.  Box given as a pointer to an
// object with getBoxDims, like PeriodicBoxPtr.
//   adapter_driver <in.bin> <out.bin>
// in.bin : int32 n, float64 L, n*2 float64 points, n*2 float64 moved points
// out.bin: int32 stride, n int32 ring lengths, n*stride int32 rows (after the build),
//          then the same after the repair
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "dgt_delaunay.hpp"

struct Box {
    double L;
    void getBoxDims(double &xx, double &xy, double &yx, double &yy) const
    {
        xx = L;
        xy = 0;
        yx = 0;
        yy = L;
    }
};

static void dump(FILE *f, dgt::DeviceArray<int> &tri, dgt::DeviceArray<int> &nn, int n)
{
    int stride = (int)(tri.getNumElements() / n);
    std::vector<int> t(tri.getNumElements()), k(n);
    tri.download(t.data());
    nn.download(k.data());
    fwrite(&stride, sizeof(int), 1, f);
    fwrite(k.data(), sizeof(int), n, f);
    fwrite(t.data(), sizeof(int), t.size(), f);
}

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 3;
    int n = 0;
    double L = 0;
    if (fread(&n, sizeof(int), 1, in) != 1 || fread(&L, sizeof(double), 1, in) != 1) return 4;
    std::vector<double> p0(2 * (size_t)n), p1(2 * (size_t)n);
    if (fread(p0.data(), sizeof(double), p0.size(), in) != p0.size()) return 5;
    if (fread(p1.data(), sizeof(double), p1.size(), in) != p1.size()) return 6;
    fclose(in);
    try {
        auto domain = std::make_shared<Box>(Box{ L });
        int maxNeighs = 4;   // deliberately small: safety mode must grow it
        dgt::DelaunayGPU delGPU(n, maxNeighs, 1.0, domain);
        delGPU.setSafetyMode(true);
        dgt::DeviceArray<double2> pts;
        pts.upload(reinterpret_cast<const double2 *>(p0.data()), n);
        dgt::DeviceArray<int> tri((size_t)maxNeighs * n), nn(n);
        delGPU.globalDelaunayTriangulation(pts, tri, nn);
        FILE *out = fopen(argv[2], "wb");
        if (!out) return 7;
        dump(out, tri, nn, n);
        pts.upload(reinterpret_cast<const double2 *>(p1.data()), n);
        delGPU.testAndRepairDelaunayTriangulation(pts, tri, nn);
        dump(out, tri, nn, n);
        fclose(out);
        printf("ok MaxSize=%d\n", delGPU.MaxSize);
    } catch (const std::exception &e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}

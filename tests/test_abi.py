"""CPU checks of the drop-in boundary: libdgt.so loads, exports every function include/dgt.h
declares, rejects bad arguments with status codes (no GPU needed for those), and the C++
adapter header compiles."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from gpudelaunaytriangulation_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dgt.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dgt_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_header():
    L = N.lib()
    names = declared_functions()
    assert names, "no declarations parsed"
    assert sorted(N.EXPORTED) == names
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", N.library_path()], capture_output=True, text=True).stdout
    for name in names:
        assert re.search(rf"\bT {name}$", out, re.M), name


def test_error_strings_and_version():
    L = N.lib()
    assert L.dgt_version() >= 1
    for code in range(8):
        assert L.dgt_error_string(code)
    assert b"unknown" in L.dgt_error_string(99)


def test_invalid_arguments_without_device():
    L = N.lib()
    h = ctypes.c_void_p()
    assert L.dgt_create(-1, 16, 1.0, 10.0, 10.0, ctypes.byref(h)) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_create(10, 16, 1.0, 0.0, 10.0, ctypes.byref(h)) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_create(10, 16, float("nan"), 10.0, 10.0, ctypes.byref(h)) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_create(10, 16, 1.0, 10.0, 10.0, None) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_create_batch(0, None, None, 1.0, 16, ctypes.byref(h)) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_global_triangulation(None, None, None, None, 16, None) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_test_and_repair(None, None, None, None, 16, None) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_set_precision(None, 0) == N.DGT_ERR_INVALID_ARGUMENT
    v = ctypes.c_int()
    assert L.dgt_get_max_size(None, ctypes.byref(v)) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_restride(None, 4, None, 8, None, 5, None) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_set_box_general(None, 1.0, 0.5, 0.0, 1.0) == N.DGT_ERR_INVALID_ARGUMENT
    assert L.dgt_set_graph_flip_rounds(None, 3) == N.DGT_ERR_INVALID_ARGUMENT
    box = (ctypes.c_double * 4)()
    assert L.dgt_get_box(None, box) == N.DGT_ERR_INVALID_ARGUMENT
    L.dgt_destroy(None)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_cpp_adapter_header_compiles(tmp_path):
    src = tmp_path / "use.cpp"
    # the box-object constructor and setBox instantiated with a general box type
    src.write_text('#include <memory>\n#include "dgt_delaunay.hpp"\n'
                   'struct Box { void getBoxDims(double &a, double &b, double &c, double &d) const '
                   '{ a = 10; b = 5; c = 0; d = 8; } };\n'
                   'void use() { auto bx = std::make_shared<Box>(); dgt::DelaunayGPU g(100, 16, 1.0, bx); '
                   'g.setBox(bx); int m = g.MaxSize; (void)m; dgt::DelaunayGPU b; b.initialize(100, 16, 1.0, bx); '
                   'dgt::DelaunayGPUT<std::shared_ptr<Box>> k(100, 16, 1.0, bx); double a, c, d, e; '
                   'k.Box->getBoxDims(a, c, d, e); }\nint main(){ return 0; }\n')
    cuda_inc = "/usr/local/cuda/include"
    r = subprocess.run(["g++", "-std=c++14", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_python_mirror_fails_loudly_without_device():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from gpudelaunaytriangulation_b200.delaunay import DelaunayGPU

    with pytest.raises(N.DgtError) as e:
        DelaunayGPU(10, 16, 1.0, (3.0, 3.0))
    assert e.value.code == N.DGT_ERR_CUDA


REFERENCE_USE = r"""
#include "std_include.h"
#include "gpuarray.h"
#include "periodicBoundaries.h"
#include "dgt_gpuarray.hpp"
// the reference's driver code (triangulation.cpp:224-246, :299, :361, :390) over the adapter
void use()
{
    PeriodicBoxPtr domain = make_shared<periodicBoundaries>(10.0, 10.0);
    GPUArray<double2> gpuPts(100u);
    GPUArray<int> gpuTriangulation(1600u), cellNeighborNumber(100u);
    dgt::DelaunayGPUT<PeriodicBoxPtr> delGPU(100, 16, 1.0, domain);
    delGPU.setSafetyMode(true);
    delGPU.setGPUcompute(true);
    delGPU.globalDelaunayTriangulation(gpuPts, gpuTriangulation, cellNeighborNumber);
    double2 pTarget;
    pTarget.x = 11.0;
    pTarget.y = -1.0;
    delGPU.Box->putInBoxReal(pTarget);
    delGPU.testAndRepairDelaunayTriangulation(gpuPts, gpuTriangulation, cellNeighborNumber);
    int maxSize = delGPU.MaxSize;
    (void)maxSize;
    delGPU.prof.print();
    delGPU.hilbertSortArray(gpuPts);   // the driver's hilbertSortArray pre-pass, on the device
    dgt::DelaunayGPU blank;
    blank.initialize(100, 16, 1.0, domain);
    blank.updateList(gpuPts);
}
int main() { return 0; }
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_cpp_adapter_compiles_against_reference_gpuarray(tmp_path):
    # the GPUArray<T> traits (include/dgt_gpuarray.hpp) instantiated with the reference's own
    # container and box headers, as a maintainer of the reference would build them
    from oracle import oracle as O

    ref = O.reference_dir()
    if not os.path.exists(os.path.join(ref, "inc", "gpuarray.h")):
        pytest.skip("the reference's sources are not present")
    src = tmp_path / "use_gpuarray.cpp"
    src.write_text(REFERENCE_USE)
    cuda_inc = "/usr/local/cuda/include"
    r = subprocess.run(["g++", "-std=c++14", "-fsyntax-only", "-DENABLE_CUDA",
                        "-I", os.path.join(ref, "inc"), "-I", os.path.join(ref, "src"),
                        "-I", os.path.join(ref, "src", "utilities"), "-I", os.path.join(ROOT, "include"),
                        "-I", cuda_inc, "-I", os.path.join(cuda_inc, "nvtx3"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_adapter_box_wraps_points_like_the_reference(tmp_path):
    # dgt::BoxDims::putInBoxReal (the adapter's copy of the box, host code) puts points into
    # the primary cell the way periodicBoundaries::putInBoxReal does, for rectangular and
    # general boxes; no device involved
    src = tmp_path / "box.cpp"
    src.write_text(r"""
#include <cstdio>
#include "dgt_delaunay.hpp"
int main()
{
    dgt::BoxDims r(10.0, 0.0, 0.0, 8.0), g(10.0, 5.0, 0.0, 8.0);
    const double in[6][2] = { {-1.0, 3.0}, {10.0, 8.0}, {25.5, -17.25}, {3.0, 4.0}, {-1e-12, 7.999999999}, {1e6, -1e6} };
    for (int k = 0; k < 6; ++k) {
        double2 p; p.x = in[k][0]; p.y = in[k][1];
        double2 q = p;
        r.putInBoxReal(p);
        g.putInBoxReal(q);
        // fractional coordinates of q in the general box
        const double det = 10.0 * 8.0 - 5.0 * 0.0;
        const double u = (8.0 * q.x - 5.0 * q.y) / det, v = (-0.0 * q.x + 10.0 * q.y) / det;
        std::printf("%.17g %.17g %.17g %.17g\n", p.x, p.y, u, v);
    }
    return 0;
}
""")
    exe = tmp_path / "box"
    r = subprocess.run(["g++", "-std=c++14", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [list(map(float, ln.split())) for ln in out if ln.strip()]
    for x, y, u, v in rows:
        assert 0.0 <= x < 10.0 and 0.0 <= y < 8.0
        assert -1e-12 <= u < 1.0 + 1e-12 and -1e-12 <= v < 1.0 + 1e-12
    assert rows[0][:2] == [9.0, 3.0] and rows[3][:2] == [3.0, 4.0]

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
                   'g.setBox(bx); }\nint main(){ return 0; }\n')
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

"""The header-only C++ adapter used like the reference's DelaunayGPU class by a compiled
host program (tests/cpp/adapter_driver.cpp): results must equal the oracle's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from gpudelaunaytriangulation_b200 import build as B
from gpudelaunaytriangulation_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def read_rings(f, n):
    stride = int(np.fromfile(f, np.int32, 1)[0])
    nn = np.fromfile(f, np.int32, n)
    tri = np.fromfile(f, np.int32, n * stride).reshape(n, stride)
    return tri, nn


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_cpp_adapter_driver(tmp_path):
    exe = tmp_path / "adapter_driver"
    cuda = "/usr/local/cuda"
    r = subprocess.run(["g++", "-std=c++14", "-O2", os.path.join(HERE, "cpp", "adapter_driver.cpp"),
                        "-I", os.path.join(ROOT, "include"), "-I", cuda + "/include",
                        "-L", B.LIBDIR, "-ldgt", "-L", cuda + "/lib64", "-lcudart",
                        "-Wl,-rpath," + B.LIBDIR, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n = 20000
    L = float(np.sqrt(n))
    p0 = W.uniform_points(n, L, 77)
    p1 = W.displace(p0, 0.05, L, L, 78)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([n], np.int32).tofile(f)
        np.array([L], np.float64).tofile(f)
        p0.tofile(f)
        p1.tofile(f)
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    with open(out, "rb") as f:
        t0, k0 = read_rings(f, n)
        t1, k1 = read_rings(f, n)
    for pts, t, k in ((p0, t0, k0), (p1, t1, k1)):
        ref = O.restated_global(pts, L, L, 1.0, 32)
        w = t.shape[1]
        assert np.array_equal(k, ref.nn)
        assert np.array_equal(O.canonical(t, k)[:, :w], O.canonical(ref.tri, ref.nn)[:, :w])

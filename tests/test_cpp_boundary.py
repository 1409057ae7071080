"""The C++ boundary: tests/cpp/boundary_demo.cpp is compiled against include/amethyst.hpp and
include/amethyst.h with the host compiler and linked to libamethyst_b200.so (on any machine);
on a B200 it runs the src/lib.cuh-named launchers, the slab/nogaps forms and a program plus its
graph, and every output is compared with the C oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "boundary_demo.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out_dir):
    from amethyst_b200 import build as B

    if not os.path.exists(B.LIB):
        B.build()
    exe = os.path.join(out_dir, "boundary_demo")
    libdir = os.path.dirname(B.LIB)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), SRC, "-o", exe, "-L", libdir, "-lamethyst_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{libdir}", f"-Wl,-rpath,{CUDA}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_cpp_boundary_compiles(tmp_path):
    exe = build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_boundary_matches_the_oracle(cuda, tmp_path):
    from oracle import oracle as O

    SLAB, PLAIN64, NOGAPS = 2, 1, 3
    exe = build(str(tmp_path))
    n = 300007
    a = O.uniform_values(31, 11, n)
    b = O.uniform_values(32, 11, n)
    d = str(tmp_path)
    for name, v in (("a", a), ("b", b)):
        O.encode(SLAB, 11, v).tofile(os.path.join(d, f"{name}.slab"))
        O.encode(PLAIN64, 11, v).tofile(os.path.join(d, f"{name}.plain64"))
        O.encode(NOGAPS, 11, v).tofile(os.path.join(d, f"{name}.nogaps"))
    rng = np.random.default_rng(3)
    mask = rng.integers(0, 2**32, size=(n + 31) // 32, dtype=np.uint64).astype(np.uint32)
    if n % 32:
        mask[-1] &= np.uint32((1 << (n % 32)) - 1)
    mask.tofile(os.path.join(d, "mask.bin"))
    r = subprocess.run([exe, d, str(n)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

    def got(name):
        return np.fromfile(os.path.join(d, name), dtype=np.uint8)

    sraw, praw, nraw = O.encode(SLAB, 11, a), O.encode(PLAIN64, 11, a), O.encode(NOGAPS, 11, a)
    assert np.array_equal(got("add_slab.out"), O.binary(0, sraw, SLAB, 11, O.encode(SLAB, 11, b), SLAB, 11, n, SLAB, 12))
    assert np.array_equal(got("add_nogaps.out"),
                          O.binary(0, nraw, NOGAPS, 11, O.encode(NOGAPS, 11, b), NOGAPS, 11, n, NOGAPS, 12))
    assert np.array_equal(got("mul_plain64.out"),
                          O.binary(2, praw, PLAIN64, 11, O.encode(PLAIN64, 11, b), PLAIN64, 11, n, PLAIN64, 22))
    want, cnt = O.compressstore(praw, n, PLAIN64, 11, mask, PLAIN64, 11)
    assert int(got("cs_plain64.count").view(np.uint64)[0]) == cnt
    assert np.array_equal(got("cs_plain64.out"), want)
    half = O.filter(praw, n, PLAIN64, 11, O.pred(9, bits=11))
    assert np.array_equal(got("filter_half_plain64.out").view(np.uint32), half)
    lt = O.filter(sraw, n, SLAB, 11, O.pred(1, 205))
    assert np.array_equal(got("filter_slab.out").view(np.uint32), lt)
    want, cnt = O.compressstore(sraw, n, SLAB, 11, mask, SLAB, 11)
    assert int(got("cs_slab.count").view(np.uint64)[0]) == cnt
    assert np.array_equal(got("cs_slab.out"), want)
    hop = got("hop.out").view(np.uint64)
    assert int(hop[0]) == O.reduce(0, nraw, n, NOGAPS, 11) and int(hop[1]) == O.reduce(2, sraw, n, SLAB, 11)
    # the program: (a + b) >= 1024 compressed to 12-bit slabs, sum and min of the survivors
    v = a + b
    keep = v[v >= 1024]
    res = got("program_res.out").view(np.uint64)
    assert res.tolist() == [keep.size, int(keep.sum()), int(keep.min())]
    assert np.array_equal(got("program_col.out"), O.encode(SLAB, 12, keep)[: O.storage_bytes(SLAB, 12, keep.size)])
    assert np.array_equal(got("graph_res.out").view(np.uint64), res)

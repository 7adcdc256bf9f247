"""The drop-in C++ header (include/fasttree/hlbvh.hpp) compiles in every reference
configuration (CPU) and its parity program passes on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_self_knn_b200.cpp")
OUT = os.path.join(ROOT, "tests", "cpp", "_build")
CUDA = "/usr/local/cuda"
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

CONFIGS = {
    "morton_f64": ["-DSFC_TYPE_MORTON", "-DCOORDS_TYPE_DOUBLE"],
    "morton_f32": ["-DSFC_TYPE_MORTON"],
    "ph_f64": ["-DSFC_TYPE_PEANO_HILBERT", "-DCOORDS_TYPE_DOUBLE"],
    "ph_u32": ["-DSFC_TYPE_PEANO_HILBERT", "-DFASTTREE_INTEGER_COORDS", "-DPOSITIONS_IN_32BIT"],
    "ph_u64_per": ["-DSFC_TYPE_PEANO_HILBERT", "-DFASTTREE_INTEGER_COORDS", "-DPOSITIONS_IN_64BIT", "-DPERIODIC_BC"],
    "ph_u64_per_orig": ["-DSFC_TYPE_PEANO_HILBERT", "-DFASTTREE_INTEGER_COORDS", "-DPOSITIONS_IN_64BIT",
                        "-DPERIODIC_BC", "-DRETURN_ORIG_INDICES"],
    # the header's default is the fast walk; this one runs the reference traversal itself
    "ph_u64_per_plain": ["-DSFC_TYPE_PEANO_HILBERT", "-DFASTTREE_INTEGER_COORDS", "-DPOSITIONS_IN_64BIT",
                         "-DPERIODIC_BC", "-DFASTTREE_B200_PLAIN_TRAVERSAL"],
    "morton_f64_plain": ["-DSFC_TYPE_MORTON", "-DCOORDS_TYPE_DOUBLE", "-DFASTTREE_B200_PLAIN_TRAVERSAL"],
}


def build(name, flags):
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, f"test_self_knn_{name}")
    lib_dir = os.path.join(ROOT, "fasttree_b200")
    cmd = [CXX, "-std=c++17", "-O2", *flags, "-I" + os.path.join(ROOT, "include"), "-I" + CUDA + "/include", SRC,
           "-o", exe, "-L" + lib_dir, "-l:libfasttree_b200.so", "-Wl,-rpath," + lib_dir, "-L" + CUDA + "/lib64",
           "-lcudart", "-Wl,-rpath," + CUDA + "/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


@pytest.mark.parametrize("name", list(CONFIGS))
def test_header_compiles(name):
    build(name, CONFIGS[name])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_cpp_parity_program(name):
    exe = build(name, CONFIGS[name])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "ALL TESTS PASSED" in r.stdout

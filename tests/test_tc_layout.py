"""Host checks of the tensor-core filtering's packed taps and tile
geometries (CPU, no GPU).

tests/cpp/tc_tap_layout.cpp rebuilds every stage's banded Toeplitz matrix
from the library's packing (brc::tc::pack_taps) for banks of 3 and 6
filters.  For split BF16 it adds the hi and lo parts; for TF32 it places
each stored value of a sample pair (P, P + 8) by the metadata nibble of the
TMEM lane that the kernel writes (brc::tc::metadata_word).  It then compares
the matrix with the filter taps: BF16 hi + lo to 2^-16, TF32 bit for bit
after rounding to TF32.  The kernels' results are checked on the GPU
against the FP64 oracle (test_gpu_tc.py).  This test also runs without a
GPU and catches a packing or metadata change that breaks the layout.

tests/cpp/tc_geometry.cu walks a grid of volume heights and depths.  It
checks that every tile height the cost model offers gives a launchable
geometry: N within the precision's limit (240 for TF32, whose metadata
takes a TMEM column), every GEMM's B rows inside the staged array, and
shared memory within a CTA's 227 KB."""
import os
import subprocess

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "tc_tap_layout.cpp")
GEOM = os.path.join(ROOT, "tests", "cpp", "tc_geometry.cu")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def test_packed_taps_rebuild_the_banded_matrices(tmp_path):
    exe = os.path.join(str(tmp_path), "tc_tap_layout")
    libdir = os.path.join(ROOT, "broccoli_b200")
    subprocess.check_call(["g++", "-O2", "-std=c++17", SRC, "-L", libdir, "-lbroccoli_b200",
                           f"-Wl,-rpath,{libdir}", "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_tile_geometries_fit_the_kernel(tmp_path):
    exe = os.path.join(str(tmp_path), "tc_geometry")
    libdir = os.path.join(ROOT, "broccoli_b200")
    subprocess.check_call([NVCC, "-std=c++17", "-O2", "--expt-relaxed-constexpr",
                           "-gencode", "arch=compute_100a,code=sm_100a", GEOM, "-L", libdir, "-lbroccoli_b200",
                           "-Xlinker", "-rpath", "-Xlinker", libdir, "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok ")

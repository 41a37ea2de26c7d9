"""The C++ drop-in (include/cucosma.hpp, cucosma_config_compat.h): a caller
written like the reference's (config.h macros, six-argument cosmaSgemm on
cudaMallocPitch'ed rows) compiles against the headers and links the library
(CPU test), and computes C = ALPHA*A*B + BETA*C on a B200 (GPU test)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cu")
LIBDIR = os.path.join(ROOT, "cucosma_b200")


def build(out_dir):
    exe = os.path.join(out_dir, "dropin_main")
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe, "-L" + LIBDIR, "-lcucosma", "-lcublas",
           "-Xlinker", "-rpath=" + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_dropin_compiles_and_links(tmp_path):
    assert os.path.exists(build(str(tmp_path)))


@pytest.mark.gpu
def test_dropin_runs(cuda, tmp_path):
    exe = build(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr

"""Build recipe for oracle/_ref/: the reference's own code compiled from its sources.

TEST INFRASTRUCTURE ONLY.  Everything here reads the cuCOSMA sources where they
lie (REF_ROOT, default /root/reference) and writes only into oracle/_ref/:

  libref_cpu.so        Matrix<T>::operator* and Matrix<T>::fillRandom
                       (Kernel/cuda/src/Matrix.h:75-87, :183-201)
  ref_schedgen         the ScheduleGenerator (ScheduleGenerator/ScheduleGeneratorv4.h:13)
  libref_gpu_<tag>.so  the reference kernel cosmaSgemm (Kernel/cuda/src/cuCOSMAV100.cuh)
                       for one compile-time configuration each, tiles chosen by
                       ref_schedgen exactly as run.sh would take them from a
                       TESTS_TO_RUN row (Kernel/cuda/run.sh:189-257)

The reference has no build system of its own in the tree (run.sh expects
Debug/Release Makefile directories that are not shipped), so the recipe calls
nvcc / g++ directly on the few files the path needs.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REF_ROOT = os.environ.get("CUCOSMA_REF_ROOT", "/root/reference")
KSRC = os.path.join(REF_ROOT, "Kernel", "cuda", "src")
SCHED = os.path.join(REF_ROOT, "ScheduleGenerator")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (tag, dtype, m, n, k, alpha, beta).  Tiles/split-K come from ref_schedgen.
GPU_CONFIGS = [
    ("f32_1024_a1b0", "float", 1024, 1024, 1024, "1", "0"),
    ("f32_1024_a1b05", "float", 1024, 1024, 1024, "1", "0.5"),
    ("f32_127_a1b05", "float", 127, 127, 127, "1", "0.5"),
    ("f32_300x200x100_a15b05", "float", 300, 200, 100, "1.5", "0.5"),
    ("f32_256x256x65536_a1b05", "float", 256, 256, 65536, "1", "0.5"),
    ("f32_8192_a1b05", "float", 8192, 8192, 8192, "1", "0.5"),
    ("f64_1024_a1b05", "double", 1024, 1024, 1024, "1", "0.5"),
    ("f64_300x200x100_a15b05", "double", 300, 200, 100, "1.5", "0.5"),
]


def have_reference() -> bool:
    return os.path.isfile(os.path.join(KSRC, "cuCOSMAV100.cuh"))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout[-4000:], r.stderr[-4000:]))
    return r.stdout


def _stale(target, *sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_schedgen():
    exe = os.path.join(OUT, "ref_schedgen")
    src = os.path.join(HERE, "ref", "ref_schedgen.cpp")
    if _stale(exe, src):
        _run(["g++", "-std=c++17", "-O2", "-include", "cstdint", "-I" + SCHED, src, "-o", exe])
    return exe


def schedule(m, n, k):
    """One ScheduleGenerator row (main.cpp:309-331 column order) as a dict."""
    out = _run([build_schedgen(), str(m), str(n), str(k)]).strip().split(",")
    if out[0] == "none":
        raise RuntimeError("ScheduleGenerator found no schedule for %dx%dx%d" % (m, n, k))
    keys = ["occupancy", "type", "v2", "v4", "m", "n", "k", "tbm", "tbn", "tbk", "load_k", "wm", "wn",
            "tm", "tn", "split_k", "alpha", "beta", "swizzle", "a_off", "b_off", "atomic"]
    return dict(zip(keys, out))


def build_cpu():
    so = os.path.join(OUT, "libref_cpu.so")
    src = os.path.join(HERE, "ref", "ref_cpu.cu")
    if _stale(so, src):
        _run([NVCC, "-O3", "-std=c++17", *ARCH, "-Xcompiler", "-fPIC,-fopenmp", "-shared",
              "-I" + KSRC, "-o", so, src, "-lgomp"])
    return so


def _gpu_one(cfg):
    tag, dtype, m, n, k, alpha, beta = cfg
    so = os.path.join(OUT, "libref_gpu_%s.so" % tag)
    src = os.path.join(HERE, "ref", "ref_gpu.cu")
    if not _stale(so, src, __file__):
        return so
    s = schedule(m, n, k)
    v2, v4 = ("float2", "float4") if dtype == "float" else ("double2", "double4")
    # FP64 at the FP32 tiles spills heavily at two CTAs per SM; one CTA per SM.
    occ = "2" if dtype == "float" else "1"
    defs = dict(CONFIG_H_="", TYPE=dtype, VECTORTYPE2=v2, VECTORTYPE4=v4, M=m, N=n, K=k,
                THREADBLOCK_TILE_M=s["tbm"], THREADBLOCK_TILE_N=s["tbn"], THREADBLOCK_TILE_K=s["tbk"],
                LOAD_K=s["load_k"], WARP_TILE_M=s["wm"], WARP_TILE_N=s["wn"], THREAD_TILE_M=s["tm"],
                THREAD_TILE_N=s["tn"], A_OFFSET=s["a_off"], B_OFFSET=s["b_off"], SWIZZLE=1,
                SPLIT_K=s["split_k"], ATOMIC_REDUCTION=s["atomic"], ADDITIONAL_OCCUPANCY_SM=occ,
                ALPHA=alpha, BETA=beta)
    flags = ["-D%s=%s" % (a, b) if b != "" else "-D%s" % a for a, b in defs.items()]
    if dtype == "double":
        flags.append("-DREF_FP64")
    _run([NVCC, "-O3", "-std=c++17", *ARCH, "-Xcompiler", "-fPIC", "-shared", "-w", "-I" + KSRC,
          *flags, "-o", so, src, "-lcublas"])
    return so


def build_gpu(jobs=None):
    jobs = jobs or min(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        return list(ex.map(_gpu_one, GPU_CONFIGS))


def build(verbose=True):
    if not have_reference():
        if verbose:
            print("oracle/_ref: reference sources not present; keeping prebuilt files")
        return False
    os.makedirs(OUT, exist_ok=True)
    build_schedgen()
    build_cpu()
    build_gpu()
    if verbose:
        print("oracle/_ref: built", sorted(os.listdir(OUT)))
    return True


if __name__ == "__main__":
    sys.exit(0 if build() else 1)

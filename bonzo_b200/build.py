"""Build libbnzgpu.so in-tree for sm_100a (B200).

Translation units:
  bnz_kernels_exact.cu  --fmad=false  (bit-for-bit parity kernels)
  bnz_kernels_fast.cu   --fmad=true   (DFMA-contracted production kernels)
  bnz_ctx.cu                          (C ABI host code)
  bnz_noalloc.cu                      (the step that allocates no device memory)
  bnz_adjoint.cu                      (adjoint rollouts: tape and reverse pass)
  bnz_io.cu                           (history reduction, asynchronous snapshots)
linked with -shared into bonzo_b200/libbnzgpu.so.  nvcc cross-compiles, so
this runs on machines without a GPU.
"""
import concurrent.futures
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbnzgpu.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]
UNITS = [
    ("bnz_kernels_exact.cu", ["--fmad=false"]),
    ("bnz_kernels_fast.cu", ["--fmad=true"]),
    ("bnz_ctx.cu", []),
    ("bnz_noalloc.cu", []),
    ("bnz_adjoint.cu", []),
    ("bnz_io.cu", []),
    ("bnz_peak.cu", ["--fmad=true"]),
]


def _newer(dst, srcs):
    if not os.path.exists(dst):
        return False
    t = os.path.getmtime(dst)
    return all(os.path.getmtime(s) <= t for s in srcs)


def build(verbose=True, force=False, extra=()):
    os.makedirs(OUT, exist_ok=True)
    # a unit depends on its own source, every header (.h / .cuh), the C ABI
    # header and this recipe (a flag change rebuilds)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    common = headers + [os.path.join(HERE, "..", "include", "bnz_gpu.h"), os.path.abspath(__file__)]
    objs, jobs = [], []
    for src, flags in UNITS:
        obj = os.path.join(OUT, src.replace(".cu", ".o"))
        objs.append(obj)
        if not force and _newer(obj, common + [os.path.join(CSRC, src)]):
            continue
        jobs.append((src, [NVCC] + ARCH + COMMON + list(flags) + list(extra) +
                     ["-c", os.path.join(CSRC, src), "-o", obj]))

    def run(job):
        src, cmd = job
        t0 = time.time()
        subprocess.run(cmd, check=True)
        if verbose:
            print("nvcc %s (%.1fs)" % (src, time.time() - t0))

    # the units compile independently: one nvcc process per unit
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(run, j) for j in jobs]:
            f.result()
    if force or not _newer(LIB, objs):
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"], check=True)
        if verbose:
            print("linked", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)

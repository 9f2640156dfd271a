"""Build recipe of the CUDA library (sm_100a).

Two variants are built from the same sources:
  lib/libfosite_gpu.so        the product (FMA contraction on)
  lib/libfosite_gpu_exact.so  --fmad=false: every operation rounded as in the
                              reference's CPU build; used to prove bit-level
                              agreement with the CPU oracle
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(verbose=False, variants=("fast", "exact")):
    os.makedirs(LIBDIR, exist_ok=True)
    src = os.path.join(CSRC, "fgpu_host.cu")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "fosite_gpu.h")]
    newest = max(os.path.getmtime(d) for d in deps)
    outs, procs = [], []
    for var in variants:
        name = "libfosite_gpu.so" if var == "fast" else "libfosite_gpu_exact.so"
        out = os.path.join(LIBDIR, name)
        outs.append(out)
        if os.path.exists(out) and os.path.getmtime(out) >= newest:
            continue
        cmd = [nvcc(), "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-lineinfo",
               "--expt-relaxed-constexpr", *ARCH, "-o", out + ".tmp", src]
        if var == "exact":
            cmd[1:1] = ["--fmad=false", "-DFGPU_EXACT"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd), out))   # the two variants compile concurrently
    failed = []
    for p, out in procs:
        if p.wait() != 0:
            failed.append(out)
        else:
            os.replace(out + ".tmp", out)
            # stamp the library with the sources' time, so that a source edited while
            # nvcc ran still counts as newer than the library
            os.utime(out, (newest, newest))
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    return outs


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)

"""Build recipe of the CUDA library (sm_100a).

Two variants are built from the same sources:
  lib/libfosite_gpu.so        the product (FMA contraction on)
  lib/libfosite_gpu_exact.so  --fmad=false: every operation rounded as in the
                              reference's CPU build; used to prove bit-level
                              agreement with the CPU oracle
Each variant links six translation units compiled in parallel: fgpu_host.cu (the C ABI, host
drivers, boundary / FARGO / viscosity / Runge-Kutta control kernels), the shared-memory stage
kernels of 2D and 3D meshes (fgpu_stage_2d.cu, fgpu_stage_3d.cu) and the TMA-staged stage
kernels (fgpu_tma_2d.cu: 2D 32 x 8 tiles and batches, fgpu_tma_2d4.cu: 2D 32 x 4 tiles,
fgpu_tma_3d.cu).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILDDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
UNITS = ["fgpu_host.cu", "fgpu_stage_2d.cu", "fgpu_stage_3d.cu", "fgpu_tma_2d.cu", "fgpu_tma_2d4.cu", "fgpu_tma_3d.cu"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _flags(var, verbose):
    f = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "--expt-relaxed-constexpr", *ARCH]
    if var == "exact":
        f = ["--fmad=false", "-DFGPU_EXACT"] + f
    if verbose:
        f = ["-Xptxas=-v"] + f
    return f


def _obj(unit, var):
    return os.path.join(BUILDDIR, "%s_%s.o" % (os.path.splitext(unit)[0], var))


def build(verbose=False, variants=("fast", "exact")):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILDDIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "fosite_gpu.h")]
    newest = max(os.path.getmtime(d) for d in deps)
    todo = []
    for var in variants:
        name = "libfosite_gpu.so" if var == "fast" else "libfosite_gpu_exact.so"
        out = os.path.join(LIBDIR, name)
        if os.path.exists(out) and os.path.getmtime(out) >= newest:
            continue
        todo.append((var, out))
    # every translation unit of every variant compiles concurrently
    procs = []
    for var, out in todo:
        for u in UNITS:
            cmd = [nvcc(), *_flags(var, verbose), "-c", "-o", _obj(u, var), os.path.join(CSRC, u)]
            print(" ".join(cmd), file=sys.stderr)
            procs.append((subprocess.Popen(cmd), _obj(u, var)))
    failed = [obj for p, obj in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    for var, out in todo:
        cmd = [nvcc(), "-shared", *ARCH, "-o", out + ".tmp", *[_obj(u, var) for u in UNITS]]
        print(" ".join(cmd), file=sys.stderr)
        if subprocess.call(cmd) != 0:
            raise RuntimeError("link failed for " + out)
        os.replace(out + ".tmp", out)
        # stamp the library with the sources' time, so that a source edited while nvcc ran
        # still counts as newer than the library
        os.utime(out, (newest, newest))
    return [os.path.join(LIBDIR, n) for n in ("libfosite_gpu.so", "libfosite_gpu_exact.so")]


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)

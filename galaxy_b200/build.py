"""Build the in-tree CUDA library galaxy_b200/libgalaxy_gpu.so for sm_100a.

    python -m galaxy_b200.build            # or galaxy_b200.build.build()

One nvcc invocation compiles every csrc/*.cu into a shared library with a
plain C ABI (include/galaxy_gpu.h); the CUDA runtime is linked statically
so the library needs nothing beyond the driver at run time.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgalaxy_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-cudart", "static",
    "-ldl",
]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        [os.path.join(ROOT, "include", "galaxy_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    cmd = [NVCC] + FLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-o", LIB] + sources()
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)

"""Build the in-tree CUDA library galaxy_b200/libgalaxy_gpu.so for sm_100a.

    python -m galaxy_b200.build            # or galaxy_b200.build.build()

nvcc compiles every csrc/*.cu (in parallel) and links them into a shared
library with a plain C ABI (include/galaxy_gpu.h); the CUDA runtime is
linked statically so the library needs nothing beyond the driver at run
time.
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


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed: " + cmd[-1])
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)


def build(force=False, verbose=False, extra=()):
    """Compile every csrc/*.cu to an object (in parallel, under _build/) and
    link them into the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(ROOT, "_build", "galaxy_b200")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in FLAGS if f not in ("-shared", "-ldl")]
    compile_flags.remove("-cudart")
    compile_flags.remove("static")
    inc = ["-I", os.path.join(ROOT, "include")]
    jobs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        jobs.append((obj, [NVCC] + compile_flags + list(extra) + inc + ["-c", "-o", obj, src]))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda j: _run(j[1], verbose), jobs))
    _run([NVCC] + FLAGS + ["-o", LIB] + [j[0] for j in jobs], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)

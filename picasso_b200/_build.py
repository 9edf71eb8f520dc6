"""Compile the CUDA sources of the package into libpicasso_b200.so (sm_100a).

Each ``csrc/*.cu`` is compiled to an object under ``_build/`` with nvcc and
the objects are linked into ``libpicasso_b200.so`` next to this file (the
CUDA runtime is linked statically, so the library only needs the driver).
Objects are rebuilt when their source or any ``csrc/*.cuh`` / public header
is newer.
"""

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "picasso_b200")
LIB = os.path.join(HERE, "libpicasso_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
              "-I" + os.path.join(ROOT, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps_mtime():
    deps = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max([os.path.getmtime(d) for d in deps] + [0.0])


def _compile(src, obj, extra):
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return r.stderr


def build(verbose=False, extra_flags=(), jobs=None):
    """Build (or refresh) libpicasso_b200.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    dep_t = _deps_mtime()
    todo, objs = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), dep_t):
            todo.append((s, o))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        futs = {ex.submit(_compile, s, o, list(extra_flags)): s for s, o in todo}
        for f in cf.as_completed(futs):
            msg = f.result()
            if verbose and msg:
                print(msg)
    lib_t = os.path.getmtime(LIB) if os.path.exists(LIB) else -1.0
    if todo or lib_t < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    import sys
    print(build(verbose="-v" in sys.argv))

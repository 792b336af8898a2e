"""Build the native parts in-tree (sm_100a only).

* batch-cc_b200/libbcc.so  -- the product: CUDA kernels + C ABI (include/bcc.h)
* batch-cc_b200/batch_cc   -- the drop-in CLI driver (scripts/batch_cc_mbm.cpp's
                              `batch_cc <robot> <num_envs> <num_edges>`)

Every nvcc invocation targets `-gencode arch=compute_100a,code=sm_100a`; nvcc
cross-compiles without a GPU.  Rebuilds only when a source is newer than the
output.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbcc.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _newer(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(ROOT, "include", "bcc.h")]


def build_lib(force=False):
    objs = []
    dep = deps()
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    jobs = []
    for src in sources():
        obj = os.path.join(HERE, "_build", os.path.basename(src) + ".o")
        if force or _newer(obj, dep):
            jobs.append([NVCC] + ARCH + NVFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    # one nvcc process per translation unit, run side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


CXX = os.environ.get("CXX", "g++")
CLI = os.path.join(HERE, "batch_cc")


def build_cli(force=False):
    """The drop-in command-line driver, linked against libbcc.so (rpath $ORIGIN)."""
    srcs = glob.glob(os.path.join(HERE, "cli", "*")) + glob.glob(os.path.join(ROOT, "include", "src", "**", "*.hh"),
                                                                  recursive=True) + [LIB]
    if force or _newer(CLI, srcs):
        _run([CXX, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "cli"),
              os.path.join(HERE, "cli", "batch_cc.cpp"), "-o", CLI, "-L", HERE, "-lbcc", "-Wl,-rpath,$ORIGIN"])
    return CLI


def build_all(force=False):
    build_lib(force)
    build_cli(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)

"""Build recipe of the engine: every CUDA source of csrc/ compiled for sm_100a into
lib/libgpudb.so (C ABI, include/gpudb_capi.h), and the `gpudb` command-line driver
(csrc/host/*.cpp) linked against it.

    python -m gpudbmetalbenchmark_b200.build [--verbose]

nvcc cross-compiles without a GPU. Objects are rebuilt when their source or any header
changed; the link step runs when an object changed.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "lib")
OBJ = os.path.join(OUT, "obj")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC] + ARCH
LIB = os.path.join(OUT, "libgpudb.so")
CLI = os.path.join(OUT, "gpudb")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "gpudb_capi.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj, False, ""
    cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj, True, r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), sources))
    objs = [r[0] for r in results]
    if verbose:
        for _, _, log in results:
            if log:
                sys.stderr.write(log)
    if _stale(LIB, objs):
        subprocess.run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"], check=True)
    host = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    if host and _stale(CLI, host + [LIB] + glob.glob(os.path.join(CSRC, "host", "*.hpp"))):
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-o", CLI] + host +
                       ["-L", OUT, "-lgpudb", "-Wl,-rpath,$ORIGIN", "-lpthread"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))

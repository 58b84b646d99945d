"""Build recipe for the oracle (test infrastructure only).

  oracle/_build/liboracle.so   the C restatement (oracle.c), always built.
  oracle/_ref/libgpudbref.so   the reference's own kernels (kernels/*.metal of
                               nd-tung/GPUDBMetalBenchmark) compiled in place for the CPU
                               through oracle/refshim; built only where the reference
                               source tree is present (GPUDB_REFERENCE_DIR, else a
                               checkout named `reference` beside this repository).
                               Elsewhere the prebuilt file is used.

Usage: python oracle/build.py
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.environ.get("GPUDB_REFERENCE_DIR",
                         os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def _run(cmd):
    subprocess.run(cmd, check=True)


def build_oracle():
    out = os.path.join(HERE, "_build")
    os.makedirs(out, exist_ok=True)
    lib = os.path.join(out, "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if _fresh(lib, [src, os.path.join(HERE, "oracle.h")]):
        return lib
    _run(["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-pthread", src, "-o", lib])
    return lib


def build_reference():
    """Compile the reference's kernels with the shim. Returns the .so path or None."""
    out = os.path.join(HERE, "_ref")
    lib = os.path.join(out, "libgpudbref.so")
    kdir = os.path.join(REF_DIR, "kernels")
    if not os.path.isdir(kdir):
        return lib if os.path.exists(lib) else None
    os.makedirs(out, exist_ok=True)
    deps = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "refshim", "metal_stdlib")]
    deps += [os.path.join(kdir, f) for f in ("common.h", "q1.metal", "q3.metal", "q4.metal", "q5.metal", "q6.metal", "q7.metal", "q8.metal",
                                              "q9.metal", "q10.metal", "q12.metal", "q13.metal", "microbenchmarks.metal")]
    if _fresh(lib, deps):
        return lib
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-Wno-attributes",
          "-I", os.path.join(HERE, "refshim"), "-I", kdir,
          os.path.join(HERE, "ref_harness.cpp"), "-o", lib])
    return lib


def _fresh(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


if __name__ == "__main__":
    print(build_oracle())
    print(build_reference())
    sys.exit(0)

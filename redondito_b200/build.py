"""Build the sm_100a transform-core library in-tree.

    python -m redondito_b200.build        # -> redondito_b200/_lib/libsph_b200.so

nvcc cross-compiles for sm_100a without a GPU.  The library is C ABI only
(include/sph_b200.h); torch is not linked.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libsph_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "sph_b200.h"))
    return hs


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


PEAK_SRC = os.path.join(HERE, "peak", "fp64_peak.cu")
PEAK_BIN = os.path.join(LIBDIR, "fp64_peak")


def build_peak(force=False):
    """The FP64 DMMA throughput probe used as the FP64 roofline denominator."""
    if not force and os.path.exists(PEAK_BIN) and os.path.getmtime(PEAK_BIN) >= os.path.getmtime(PEAK_SRC):
        return PEAK_BIN
    os.makedirs(LIBDIR, exist_ok=True)
    subprocess.run([NVCC, *ARCH, "-O3", "-ccbin", "/usr/bin/g++", "-o", PEAK_BIN, PEAK_SRC], check=True)
    return PEAK_BIN


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    failed = []
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or (verbose and out):
            sys.stdout.write(out.decode())
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=True, verbose=v or bool(extra), extra=extra))
    print(build_peak(force=True))

"""Builds the CUDA library libsvof_b200.so in place (sm_100a).

Every translation unit of the FP64 paths is compiled with -fmad=false: every
multiply and add rounds separately, like the reference's C code on x86-64,
so the device arithmetic follows the reference's rounding.  Host code is
compiled with -ffp-contract=off for the same reason (its tables feed the
kernels).  The 3D mixed path's FP32 kernels have no rounding to follow: the
files that hold them (SPLIT below) are compiled a second time with
SVOF3_PRECISION=32 and FMA contraction on, holding only the FP32
instantiations, while their FP64 pass (SVOF3_PRECISION=64) holds the FP64
instantiations and the shared code.  Objects are compiled in parallel into a
temporary directory and linked into one shared library.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsvof_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# files whose FP32 template instantiations are compiled separately with FMA on
SPLIT = ("k3_interface.cu", "k3_predict.cu")


def nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def units():
    """(source, extra flags, object name) of every translation unit"""
    out = []
    for src in sources():
        base = os.path.splitext(os.path.basename(src))[0]
        if os.path.basename(src) in SPLIT:
            out.append((src, ["-fmad=false", "-DSVOF3_PRECISION=64"], base + ".f64.o"))
            out.append((src, ["-fmad=true", "-DSVOF3_PRECISION=32"], base + ".f32.o"))
        else:
            out.append((src, ["-fmad=false"], base + ".o"))
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I" + os.path.join(ROOT, "include")]
    tmp = tempfile.mkdtemp(prefix="svof_build_")
    try:
        cmds = [common + flags + ["-c", src, "-o", os.path.join(tmp, obj)] for src, flags, obj in units()]

        def run(cmd):
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)

        with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
            list(ex.map(run, cmds))
        link = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp"] + [c[-1] for c in cmds]
        run(link)
        os.replace(LIB + ".tmp", LIB)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))

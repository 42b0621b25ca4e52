"""Build the sm_100a shared library synergia2_b200/libsb2.so in-tree.

    python -m synergia2_b200.build          # or: python synergia2_b200/build.py

The particle maps of the FP64 path (track.cu) are compiled with
--fmad=false: they keep the IEEE rounding of every multiply and add, as the
reference does, and match the oracle bit for bit.  The mixed path's
particle passes (track_fast.cu) and the solver (sc3d.cu, held to
tolerances) fuse multiply-adds.  The host runtime is built with
-ffp-contract=off.  The CUDA runtime is
linked statically so the library loads without a CUDA toolkit on the
loader path.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libsb2.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["track.cu", "track_fast.cu", "sc3d.cu", "sort.cu", "noalloc.cu", "diag.cu"]
# fused multiply-adds where the results are held to tolerances, not bits:
# the mixed path's particle passes and the solver (fields within 1e-10 of
# the oracle; the FFTs of the reference's own FFT libraries fuse as well)
FMAD = {"track_fast.cu": "--fmad=true", "sc3d.cu": "--fmad=true"}
CXX_SOURCES = ["host.cc"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "sb2.h"))
    objs = []
    nv = nvcc()
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nv)), "include")
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or newer([s] + headers, o):
            out = run([nv, *ARCH, "-lineinfo", "-O3", "-std=c++17", FMAD.get(src, "--fmad=false"), "-Xcompiler", "-fPIC",
                       "-Xptxas", "-v", "-I" + CSRC, "-c", "-o", o, s])
            if verbose:
                sys.stdout.write(out)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or newer([s] + headers, o):
            run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                 "-I" + cuda_inc, "-I" + CSRC, "-c", "-o", o, s])
        objs.append(o)
    if force or newer(objs, OUT):
        run([nv, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs])
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))

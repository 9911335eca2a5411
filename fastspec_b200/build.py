"""Build the sm_100a CUDA library fastspec_b200/libfastspec_b200.so with nvcc.

The FP64 translation unit is compiled with -fmad=false so its double-precision arithmetic
keeps the reference's unfused multiply/add order; the FP32 accumulation unit uses FMA.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfastspec_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++"] + ARCH

UNITS = [
    ("fsg_kernels64.cu", ["-fmad=false"]),
    ("fsg_mag.cu", ["-fmad=false"]),
    ("fsg_fast.cu", ["-fmad=true"]),
    ("fsg_api.cu", ["-fmad=false"]),
    ("fsg_noalloc.cu", ["-fmad=false"]),
    ("fsg_adjoint.cu", ["-fmad=false"]),
    ("fsg_magfast.cu", ["-fmad=true"]),
    ("fsg_adjoint_line.cu", ["-fmad=true"]),
    ("fsg_hestark.cpp", ["-Xcompiler", "-ffp-contract=off"]),
]


def sources():
    return [os.path.join(CSRC, f) for f, _ in UNITS if os.path.exists(os.path.join(CSRC, f))]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "fastspec_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, ptxas_v=False):
    if not force and not needs_build():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for f, flags in UNITS:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(objdir, os.path.splitext(f)[0] + ".o")
        cmd = [NVCC] + COMMON + flags + (["-Xptxas", "-v"] if ptxas_v else []) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0 or verbose or ptxas_v:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on " + f)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", "/usr/bin/g++", "-o", OUT] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_v="--ptxas" in sys.argv)
    print(OUT)

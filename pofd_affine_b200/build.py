"""Build libpofd_b200.so in-tree with nvcc for sm_100a.

    python -m pofd_affine_b200.build [--verbose-ptxas]

The library lands in pofd_affine_b200/_lib/ so that it travels with the
source tree; nothing is installed into site-packages.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUTDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUTDIR, "libpofd_b200.so")
SOURCES = ["setup.cc", "fits.cc", "engine1d.cu", "engine2d.cu", "ensemble.cu", "surrogate.cu", "capi.cu",
           "noalloc.cu", "shard.cu", "ingest.cu"]
# measurement and test helpers, kept out of the likelihood's ABI
SUPPORT_LIB = os.path.join(OUTDIR, "libpofd_b200_support.so")
SUPPORT_SOURCES = [os.path.join("support", "support.cu")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or \
        "/usr/local/cuda/bin/nvcc"
    return cand


def _stale():
    if not os.path.exists(LIB) or not os.path.exists(SUPPORT_LIB):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(SUPPORT_LIB))
    deps = [os.path.join(d, f) for d in (CSRC, os.path.join(CSRC, "support"))
            for f in os.listdir(d)]
    deps += [os.path.join(HERE, "..", "include", h)
             for h in ("pofd_b200.h", "pofd_b200_support.h")]
    return any(os.path.getmtime(d) > t for d in deps
               if os.path.isfile(d))


def build(force=False, verbose_ptxas=False):
    if not force and not _stale():
        return LIB
    os.makedirs(OUTDIR, exist_ok=True)
    objdir = os.path.join(OUTDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall"] + ARCH
    if verbose_ptxas:
        common += ["-Xptxas", "-v"]
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc] + common + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cc"):
            cmd = [nvcc, "-x", "c++"] + common + ["-c", os.path.join(CSRC, src),
                                                   "-o", obj]
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc] + ARCH + ["-shared", "-o", tmp] + objs +
                          ["-lcufft", "-lcudart", "-ldl"])
    os.replace(tmp, LIB)
    sobjs = []
    for src in SUPPORT_SOURCES:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        subprocess.check_call([nvcc] + common + ["-c", os.path.join(CSRC, src),
                                                 "-o", obj])
        sobjs.append(obj)
    tmp = SUPPORT_LIB + ".tmp"
    subprocess.check_call([nvcc] + ARCH + ["-shared", "-o", tmp] + sobjs +
                          ["-lcudart"])
    os.replace(tmp, SUPPORT_LIB)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv)
    print(LIB)

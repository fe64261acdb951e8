"""Build libmstm_b200.so (sm_100a) in-tree with nvcc.

    python -m mstm_b200.build        # or mstm_b200.build.build()
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmstm_b200.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["tcpass.cu", "opgen.cu", "translate.cu", "translate_tiled.cu", "translate_rows.cu", "sphere_kernels.cu", "bicg.cu", "mrhs.cu", "ranorient.cu", "fftpath.cu", "warmstart.cu", "densepair.cu", "postproc.cu", "capi.cu", "capi_pass.cu", "capi_solve.cu", "capi_origin.cu", "noalloc.cu", "tables.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(os.path.dirname(HERE), "include", "mstm_b200.h")
    return os.path.exists(hdr) and os.path.getmtime(hdr) > t


def _headers_mtime():
    t = 0.0
    for d in (CSRC, os.path.join(os.path.dirname(HERE), "include")):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".h")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def build(force=False, verbose=False, extra=()):
    """Compile every source to an object (in parallel, only the stale ones)
    and link the shared library."""
    if not force and not _stale():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-rdc=false",
              "--expt-relaxed-constexpr", "-I", CSRC, "-I", os.path.join(os.path.dirname(HERE), "include"), *extra]
    th = _headers_mtime()
    jobs = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJDIR, s + ".o")
        objs.append(obj)
        if force or extra or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), th):
            jobs.append(common + ["-c", src, "-o", obj + ".tmp"])

    def run(cmd):
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(cmd[-1], cmd[-1][:-4])

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(run, j) for j in jobs]:
            f.result()
    link = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcufft"]
    if verbose:
        print(" ".join(link))
    subprocess.check_call(link)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a.startswith("-X")])

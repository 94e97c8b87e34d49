"""Builds the native library bismit_b200/libbismit_b200.so for sm_100a.

Each source under bismit_b200/csrc/ is compiled by nvcc into build/ (in
parallel) and linked into one shared object with the CUDA runtime linked
statically, so the library only needs the NVIDIA driver at run time.

Usage: python -m bismit_b200.build [--force] [-v]
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
LIB = os.path.join(HERE, "libbismit_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
SOURCES = ["bm_api.cu", "bm_plain.cu", "bm_fused.cu", "bm_grow.cu", "bm_static.cu", "bm_batch.cu", "bm_server.cu", "bm_sampler.cu", "bm_encode.cu", "bm_layout.cpp"]


def _newer(src_paths, dst):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "bismit_b200.h"))
    return hs


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _newer([sp] + headers, obj):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", sp, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [NVCC, "-x", "cu"] + ARCH + FLAGS + ["-c", sp, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    if jobs:
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for cmd, p in ex.map(run, jobs):
                if p.returncode != 0:
                    raise RuntimeError("nvcc failed:\n%s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
                if verbose and (p.stdout or p.stderr):
                    print(p.stdout + p.stderr)
    if force or jobs or _newer(objs, LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

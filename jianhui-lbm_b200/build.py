"""Builds liblbm.so in-tree for sm_100a (B200).

    python jianhui-lbm_b200/build.py [--verbose] [--ptxas-info]

CUDA sources are compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``,
host sources by the system g++ (shared libstdc++), and everything is linked
against the static CUDA runtime into ``lbm_b200/liblbm.so``.  Objects are
cached under ``_build/`` and rebuilt when a source or header is newer.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "lbm_b200", "liblbm.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
GEN = os.path.join(BUILD, "gen")  # generated headers (mi_pattern.h)
INCLUDES = ["-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I", GEN]

# (source, extra nvcc flags).  The *_faithful.cu files must not contract a*b+c
# into FMA: they reproduce the reference's FP64 arithmetic bit for bit.
CUDA_SOURCES = [
    ("sp_kernels.cu", []),
    ("sp_faithful.cu", ["-fmad=false"]),
    ("reduce_noalloc.cu", ["-fmad=false"]),
    ("batch_kernels.cu", []),
    ("setup_kernels.cu", []),
    ("cg_faithful.cu", ["-fmad=false"]),
    ("cg_fast.cu", []),
    ("st7_kernels.cu", []),
    ("st7_faithful.cu", ["-fmad=false"]),
    ("box_sums.cu", []),
]
CXX_SOURCES = ["api.cpp", "geometry.cpp", "mrt.cpp", "io.cpp", "batch.cpp", "cg_api.cpp", "st7_api.cpp", "output.cpp", "transfer.cpp"]
# Command-line drivers linked against liblbm.so: (source, executable name).
EXECUTABLES = [("lbm_sp_main.cpp", "lbm_sp"), ("lbm_cg_main.cpp", "lbm_cg"), ("lbm_st7_main.cpp", "lbm_st7")]
BIN = os.path.join(HERE, "lbm_b200")


def _headers():
    hs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def _generate(headers, verbose, force):
    """Writes _build/gen/mi_pattern.h (the zero / power-of-two pattern of the
    Gauss-Jordan M^-1, gen_mi_pattern.cpp) when its inputs changed."""
    os.makedirs(GEN, exist_ok=True)
    hdr = os.path.join(GEN, "mi_pattern.h")
    srcs = [os.path.join(CSRC, "gen_mi_pattern.cpp"), os.path.join(CSRC, "mrt.cpp")]
    if not force and os.path.exists(hdr) and \
            all(os.path.getmtime(hdr) >= os.path.getmtime(x) for x in srcs + headers):
        return hdr
    exe = os.path.join(BUILD, "gen_mi_pattern")
    _run([CXX, "-O2", "-std=c++17", "-I", os.path.join(CUDA, "include"), *INCLUDES, *srcs, "-o", exe], verbose)
    text = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    if not os.path.exists(hdr) or open(hdr).read() != text:
        with open(hdr, "w") as fh:
            fh.write(text)
    else:
        os.utime(hdr)
    return hdr


def _stale(obj, src, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}):\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(verbose=False, ptxas_info=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    headers.append(_generate(headers, verbose, force))
    sources = [os.path.join(CSRC, s) for s, _ in CUDA_SOURCES] + [os.path.join(CSRC, s) for s in CXX_SOURCES]
    exes = [os.path.join(BIN, name) for _, name in EXECUTABLES]
    sources += [os.path.join(CSRC, s) for s, _ in EXECUTABLES]
    if not (force or ptxas_info) and all(os.path.exists(p) for p in [OUT] + exes):
        newest = max(os.path.getmtime(p) for p in sources + headers + [os.path.abspath(__file__)])
        if min(os.path.getmtime(p) for p in [OUT] + exes) >= newest:
            return OUT, ""
    objs = []
    logs = []
    for src, extra in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or ptxas_info or _stale(o, s, headers):
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-ccbin", CXX, "-Xcompiler", "-fPIC,-fvisibility=hidden",
                   "--expt-relaxed-constexpr", *INCLUDES, *extra, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            logs.append(_run(cmd, verbose))
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, s, headers):
            cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wno-unused-function",
                   "-I", os.path.join(CUDA, "include"), *INCLUDES, "-c", s, "-o", o]
            logs.append(_run(cmd, verbose))
    if force or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        tmp = OUT + ".tmp"
        cmd = [NVCC, *ARCH, "-ccbin", CXX, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs,
               "-cudart", "static", "-Xlinker", "--exclude-libs,ALL"]
        logs.append(_run(cmd, verbose))
        shutil.move(tmp, OUT)
    for src, name in EXECUTABLES:
        s = os.path.join(CSRC, src)
        exe = os.path.join(BIN, name)
        if force or _stale(exe, s, headers + [OUT]):
            cmd = [CXX, "-O2", "-std=c++17", "-Wall", *INCLUDES, s, "-o", exe, "-L", BIN, "-llbm",
                   "-Wl,-rpath,$ORIGIN"]
            logs.append(_run(cmd, verbose))
    return OUT, "".join(logs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print -Xptxas -v register/spill report")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    out, log = build(a.verbose, a.ptxas_info, a.force)
    if a.ptxas_info:
        print(log)
    print(out)


if __name__ == "__main__":
    sys.exit(main())

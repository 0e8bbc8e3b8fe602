"""Builds libfsb200.so (sm_100a) in-tree with nvcc.

    python -m fieldstitch_b200.build        # or __graft_entry__.build()

Each .cu under csrc/ is compiled for `-gencode arch=compute_100a,code=sm_100a` and linked into
fieldstitch_b200/libfsb200.so. detect.cu, describe.cu and geom.cu are compiled with --fmad=false so their
arithmetic rounds like the reference's (one rounding per operation).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfsb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "--expt-relaxed-constexpr"]
PER_FILE = {"detect.cu": ["--fmad=false"], "describe.cu": ["--fmad=false"], "geom.cu": ["--fmad=false"]}
SOURCES = ["api.cu", "pyramid.cu", "octave.cu", "detect.cu", "describe.cu", "match.cu", "tc_match.cu", "mlp.cu", "autotune.cu", "geom.cu", "prep.cu", "tracks.cu", "jpeg.cu", "ransac.cu"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, jobs=None, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "fsb200.h"))
    objs, procs = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if not _stale(obj, [path] + headers):
            continue
        cmd = [nvcc(), *ARCH, *COMMON, *PER_FILE.get(src, []), *extra, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out = p.communicate()[0].decode(errors="replace")
        if p.returncode != 0:
            failed.append((src, out))
        elif verbose and out.strip():
            print(out)
    if failed:
        raise RuntimeError("\n".join("nvcc failed on %s:\n%s" % f for f in failed))
    if procs or not os.path.exists(LIB):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, extra=[a for a in sys.argv[1:] if a != "-v"])
    print(LIB)

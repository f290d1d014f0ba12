"""Builds libnkr_b200.so in place: every csrc/*.cu compiled for sm_100a with nvcc
and linked into one shared library (the C ABI of include/nkr_b200.h).

    python nkr-zkp_b200/build.py [--force] [--verbose]

Objects go to nkr-zkp_b200/_build/; the library to nkr-zkp_b200/libnkr_b200.so.
A source is recompiled when it or any header under csrc/ or include/ is newer
than its object.  ptxas resource usage (registers, spills, shared memory) is
written to _build/ptxas.log.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnkr_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I", os.path.join(ROOT, "include"),
]


def _headers():
    out = []
    for d in (CSRC, HOST, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".h", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def _stale(src, obj, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in headers)


def _compile(src, obj):
    if src.endswith(".cpp"):
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include"),
               "-c", src, "-o", obj]
    else:
        cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    return src, p.returncode, p.stdout + p.stderr


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    srcs += sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp"))
    objs = [os.path.join(BUILD, os.path.splitext(os.path.basename(s))[0] + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(s, o, headers)]
    logs = []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for src, rc, log in ex.map(lambda so: _compile(*so), todo):
                logs.append(f"== {os.path.basename(src)}\n{log}")
                if rc != 0:
                    sys.stderr.write(log)
                    raise RuntimeError(f"nvcc failed on {src}")
        with open(os.path.join(BUILD, "ptxas.log"), "a") as f:
            f.write("\n".join(logs))
        if verbose:
            print("\n".join(logs))
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            sys.stderr.write(p.stdout + p.stderr)
            raise RuntimeError("link of libnkr_b200.so failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))

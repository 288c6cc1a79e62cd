"""Build recipe of the native library ``libopensc_b200.so`` (sm_100a).

Every ``csrc/*.cu`` file is compiled by ``nvcc -gencode arch=compute_100a,code=sm_100a
-lineinfo -O3`` into an object under ``_build/`` and the objects are linked into
``openspacecharge_b200/libopensc_b200.so`` in the source tree, so the library travels with
the repository snapshot.  Objects are rebuilt when their source or any header is newer.

Usage: ``python -m openspacecharge_b200.build [--force] [--jobs N] [--verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build", "opensc")
LIB = os.path.join(HERE, "libopensc_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-O3", "-I" + CSRC, "-I" + INCLUDE,
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> list[str]:
    # the system g++ (an alternative compiler wrapper may be first in $CXX)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return ["-ccbin", cand]
    return []


def _newest_header() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdr_t = _newest_header()
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs, todo = [], []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_t):
            todo.append((src, obj))

    def compile_one(so):
        src, obj = so
        cmd = [nvcc] + _host_cxx() + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r.returncode, r.stdout + r.stderr

    failed = []
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for src, rc, out in ex.map(compile_one, todo):
            if rc != 0:
                failed.append((src, out))
            elif verbose and out.strip():
                sys.stderr.write(f"--- {os.path.basename(src)}\n{out}\n")
    if failed:
        msg = "\n".join(f"=== {s}\n{o}" for s, o in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc] + _host_cxx() + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))

"""Builds libftsp.so (the engine and its C ABI) in-tree for sm_100a.

    python -m ftspolysol_b200.build [--force] [--verbose]

The library is written next to this file (ftspolysol_b200/libftsp.so) so it
travels with the source tree; nothing is installed into site-packages.
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
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libftsp.so")

SOURCES = ["engine_f32.cu", "engine_f64.cu", "abi.cu"]
HOST_SOURCES = ["host_model.cpp", "host_io.cpp", "host_run.cpp"]
HEADERS = ["fft_core.cuh", "passes.cuh", "chain_pairs.cuh", "learned.cuh", "engine.cuh", "host_model.h", "host_io.h"]
MAIN = os.path.join(HERE, "ftsp_main")
HOST_FLAGS = ["-O2", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-Wall"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC,-O2",
         "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else (shutil.which("nvcc") or "nvcc")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    if not os.path.exists(MAIN) or os.path.getmtime(MAIN) < t:
        return True
    deps = [os.path.join(CSRC, f) for f in SOURCES + HOST_SOURCES + HEADERS + ["main.cpp"]]
    deps += [os.path.join(INCLUDE, h) for h in ("ftsp.h", "ftsp_host.h")]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compiles each translation unit in parallel, then links libftsp.so."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    for src in SOURCES + HOST_SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        flags = ARCH + FLAGS if src.endswith(".cu") else HOST_FLAGS
        cmd = [nvcc()] + flags + ["-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
        if extra:
            cmd += list(extra)
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append(src)
            sys.stderr.write(out)
        elif verbose and out:
            print(out)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    link = [nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("linking libftsp.so failed")
    os.replace(LIB + ".tmp", LIB)
    # the reference-style executable: a thin main() over ftsp_main()
    exe = [nvcc(), "-O2", "-std=c++17", "-I", INCLUDE, os.path.join(CSRC, "main.cpp"), "-o", MAIN + ".tmp",
           "-L", HERE, "-lftsp", "-Xlinker", "-rpath,$ORIGIN"]
    res = subprocess.run(exe, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("linking ftsp_main failed")
    os.replace(MAIN + ".tmp", MAIN)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print register/smem usage (-Xptxas -v)")
    a = ap.parse_args()
    build(force=a.force or a.ptxas_info, verbose=a.verbose or a.ptxas_info,
          extra=["-Xptxas", "-v"] if a.ptxas_info else None)
    print(LIB)

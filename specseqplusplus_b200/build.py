"""Builds the engine in-tree for sm_100a (nvcc cross-compiles without a GPU).

Outputs (git-ignored, shipped with the source tree to the GPU host):
  libsspp.so      - CUDA engine + C ABI (include/sspp.h)
  libsspp_gen.so  - synthetic complex builders (input side)
  bin/specseq++   - drop-in command line (src/main.cu of the reference)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC,-O2",
                  "-I", os.path.join(ROOT, "include")]

ENGINE_SRC = ["sspp_engine.cu", "sspp_init.cu", "sspp_reduce.cu", "sspp_highclear.cu", "sspp_dual.cu", "sspp_collapse.cu", "sspp_build.cu", "sspp_xfer.cu", "sspp_tune.cpp", "sspp_server.cpp", "sspp_phat.cpp", "sspp_noalloc.cu", "sspp_io.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _objects(srcs, headers, objdir, flags, force, verbose):
    """Compiles each source to its own object in parallel (every object
    depends on all headers); returns the object paths."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(objdir, exist_ok=True)
    jobs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            jobs.append([NVCC] + flags + ["-c", "-o", obj, src])
    with ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for out in ex.map(_run, jobs):
            if verbose:
                print(out)
    return [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]


def build_engine(lib: str, objdir: str, extra_flags=(), force: bool = False, verbose: bool = False) -> None:
    """libsspp.so from per-file objects in objdir, compiled with NVFLAGS + extra_flags."""
    srcs = [os.path.join(CSRC, s) for s in ENGINE_SRC]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "sspp.h"))
    objs = _objects(srcs, headers, objdir, NVFLAGS + list(extra_flags), force, verbose)
    if force or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs)


def build(force: bool = False, verbose: bool = False) -> None:
    lib = os.path.join(HERE, "libsspp.so")
    build_engine(lib, os.path.join(HERE, "_build"), force=force, verbose=verbose)
    gen = os.path.join(HERE, "libsspp_gen.so")
    gsrc = [os.path.join(CSRC, "sspp_gen.cpp")]
    if force or _stale(gen, gsrc + [os.path.join(CSRC, "sspp_gen.h")]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-shared", "-o", gen] + gsrc)
    cli_src = os.path.join(CSRC, "sspp_cli.cpp")
    if os.path.exists(cli_src):
        os.makedirs(os.path.join(HERE, "bin"), exist_ok=True)
        cli = os.path.join(HERE, "bin", "specseq++")
        if force or _stale(cli, [cli_src, lib, os.path.join(ROOT, "include", "sspp.h")]):
            _run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", cli, cli_src,
                  "-L", HERE, "-lsspp", "-Wl,-rpath,$ORIGIN/.."])


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)

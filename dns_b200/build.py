"""Build the native parts of dns_b200 in-tree.

    python -m dns_b200.build            # library + CLI

Products (git-ignored, shipped with the tree):
    dns_b200/lib/libdns_b200.so   CUDA kernels + C ABI (sm_100a)
    dns_b200/bin/dns              drop-in CLI for slitvinov/dns main.c
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libdns_b200.so")
CLI = os.path.join(HERE, "bin", "dns")
INCLUDE = os.path.join(ROOT, "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps() -> list[str]:
    out = [os.path.join(INCLUDE, "dns_b200.h")]
    for f in os.listdir(CSRC):
        out.append(os.path.join(CSRC, f))
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_library(force: bool = False) -> str:
    if not force and not _stale(LIB, _deps()):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [_nvcc(), *NVCC_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}", "-c", src, "-o", obj]
        print("+", " ".join(cmd), flush=True)
        procs.append(subprocess.Popen(cmd))
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    _run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", tmp])
    os.replace(tmp, LIB)
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(HERE, "cli", "dns.c")
    if not force and not _stale(CLI, [src, LIB, os.path.join(INCLUDE, "dns_b200.h")]):
        return CLI
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cc = "gcc"  # the system compiler (links libm and libc only)
    _run([cc, "-std=gnu11", "-O2", "-Wall", f"-I{INCLUDE}", src,
          f"-L{os.path.dirname(LIB)}", "-ldns_b200", "-lm",
          "-Wl,-rpath,$ORIGIN/../lib", "-o", CLI])
    return CLI


def build_all(force: bool = False) -> None:
    build_library(force)
    build_cli(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)

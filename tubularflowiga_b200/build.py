"""Builds libtfiga_b200.so in-tree with nvcc for sm_100a (no JIT cache).

    python -m tubularflowiga_b200.build          # incremental
    python -m tubularflowiga_b200.build --clean

Objects go to tubularflowiga_b200/_build/, the library to
tubularflowiga_b200/lib/libtfiga_b200.so and the drop-in command to
tubularflowiga_b200/lib/iga_cuda_b200.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib"
LIBRARY = LIB / "libtfiga_b200.so"
COMMAND = LIB / "iga_cuda_b200"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "-I" + str(PKG.parent / "include")]
HOST_CXX = ["-ccbin", "g++"] if shutil.which("g++") else []


def sources():
    return sorted(SRC.glob("*.cu")) + sorted(p for p in SRC.glob("*.cpp") if p.name != "main.cpp")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    headers = list(SRC.glob("*.hpp")) + list(SRC.glob("*.cuh")) + [PKG.parent / "include" / "tfiga.h"]
    objects, commands = [], []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        objects.append(obj)
        if _stale(obj, [src] + headers):
            cmd = [NVCC] + HOST_CXX + ARCH + COMMON + ["-c", str(src), "-o", str(obj)]
            if src.suffix == ".cpp":
                cmd = [NVCC] + HOST_CXX + COMMON + ["-x", "c++", "-c", str(src), "-o", str(obj)]
            commands.append(cmd)
    procs = []
    for cmd in commands:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= (jobs or os.cpu_count() or 4):
            _wait(procs.pop(0))
    for p in procs:
        _wait(p)
    if _stale(LIBRARY, objects):
        cmd = [NVCC] + HOST_CXX + ARCH + ["-shared", "-o", str(LIBRARY)] + [str(o) for o in objects] + \
              ["-lcudart", "-Xlinker", "-rpath,$ORIGIN"]
        _run(cmd, verbose)
    main = SRC / "main.cpp"
    if main.exists() and _stale(COMMAND, [main, LIBRARY]):
        cmd = [NVCC] + HOST_CXX + COMMON + ["-x", "c++", str(main), "-o", str(COMMAND), "-L" + str(LIB),
                                             "-ltfiga_b200", "-Xlinker", "-rpath,$ORIGIN"]
        _run(cmd, verbose)
    return LIBRARY


def _wait(item):
    cmd, p = item
    out, _ = p.communicate()
    if p.returncode != 0:
        sys.stderr.write(out.decode(errors="replace"))
        raise RuntimeError("nvcc failed: " + " ".join(cmd))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        sys.stderr.write(r.stdout.decode(errors="replace"))
        raise RuntimeError("link failed: " + " ".join(cmd))


if __name__ == "__main__":
    if "--clean" in sys.argv:
        shutil.rmtree(BUILD, ignore_errors=True)
        shutil.rmtree(LIB, ignore_errors=True)
    print(build(verbose="-v" in sys.argv))

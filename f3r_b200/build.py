"""Build recipe for the f3r_b200 shared library (sm_100a only).

``python -m f3r_b200.build`` compiles ``csrc/*.cu`` and ``csrc/*.cpp`` with
nvcc into ``f3r_b200/libf3r_b200.so``, in place, so the library travels with
the source tree.  The C ABI is declared in ``include/f3r_b200.h``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libf3r_b200.so")
DRIVER_SRC = os.path.join(HERE, "driver", "f3r_run.cpp")
DRIVER = os.path.join(HERE, "bin", "f3r-run")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    "-ccbin", "/usr/bin/g++",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    hs += [os.path.join(inc, f) for f in os.listdir(inc)]
    return hs


def up_to_date() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(DRIVER):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(DRIVER))
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [DRIVER_SRC])


def build_driver(verbose: bool = False) -> str:
    """The command-line driver (bin/f3r-run), linked against the library with
    an rpath to it, so it runs from the source tree."""
    os.makedirs(os.path.dirname(DRIVER), exist_ok=True)
    cmd = [nvcc(), DRIVER_SRC, "-o", DRIVER, "-std=c++17", "-O2", "-ccbin", "/usr/bin/g++",
           "-I", os.path.join(os.path.dirname(HERE), "include"), "-L", HERE, "-lf3r_b200",
           "-Xlinker", "-rpath,$ORIGIN/.."]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and up_to_date():
        return LIB
    objs = []
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    procs = []
    for src in sources():
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + list(extra)
        if src.endswith(".cpp"):
            cmd += ["-x", "cu"]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    failed = []
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode()))
        elif verbose and out:
            print(out.decode())
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    link = [nvcc(), "-shared", "-o", LIB] + objs + ["-gencode", "arch=compute_100a,code=sm_100a",
                                                     "-Xcompiler", "-fopenmp", "-ccbin", "/usr/bin/g++"]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    build_driver(verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)

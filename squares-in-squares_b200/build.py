"""Build libsqs.so (CUDA sm_100a + C++ host runtime) in-tree with nvcc.

    python squares-in-squares_b200/build.py [--force] [--verbose]

Objects go to squares-in-squares_b200/_build/, the library to
squares-in-squares_b200/sqs/libsqs.so, the drop-in executables (packing,
seeded, certifier) to squares-in-squares_b200/bin/, ptxas resource usage (registers,
spills, shared memory) to _build/ptxas.log.  Only sources whose mtime (or
that of any header) changed are recompiled.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "sqs" / "libsqs.so"
BIN = PKG / "bin"
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
               "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]
# Kernels compiled without multiply-add contraction: the certifier, whose
# double-precision results must equal a C oracle bit for bit (the host
# compiler contracts none), and the FP64 polish, whose neighbour-list and
# all-pairs energies must agree bit for bit.
NO_FMA = {"certify_kernel.cu", "polish_kernel.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
    hm = _headers_mtime()
    objs, logs, changed = [], [], False
    for src in srcs:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hm):
            continue
        cmd = [nvcc(), *NVCC_COMMON, *GENCODE, "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cu":
            cmd += ["-Xptxas", "-v"]
            if src.name in NO_FMA:
                cmd += ["-fmad=false"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src.name}")
        (BUILD / (src.name + ".ptxas.log")).write_text(r.stdout + r.stderr)
        changed = True
    if changed or force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *GENCODE, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libsqs.so failed")
    log = "".join(p.read_text() for p in sorted(BUILD.glob("*.ptxas.log")))
    (BUILD / "ptxas.log").write_text(log)
    build_cli(force, verbose)
    return LIB


# Drop-in executables of the reference's search and certifier programs, on
# top of libsqs.so (found next to them through the run path).
CLI = {
    "packing": ("search.cpp", []),
    "seeded": ("search.cpp", ["-DSQS_FLAVOR_SEEDED"]),
    "certifier": ("certifier.cpp", []),
}


def build_cli(force: bool = False, verbose: bool = False) -> None:
    BIN.mkdir(exist_ok=True)
    for name, (src, defs) in CLI.items():
        exe, s = BIN / name, PKG / "cli" / src
        newest = max(s.stat().st_mtime, LIB.stat().st_mtime, (ROOT / "include" / "sqs.h").stat().st_mtime)
        if not force and exe.exists() and exe.stat().st_mtime >= newest:
            continue
        cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", *defs, "-I", str(ROOT / "include"), str(s),
               "-o", str(exe), "-L", str(LIB.parent), "-lsqs", "-Wl,-rpath,$ORIGIN/../sqs"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"build of {name} failed")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))


if __name__ == "__main__":
    main()

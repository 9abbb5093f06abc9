"""Build libmnmgdl.so (the engine's C-ABI library) for sm_100a with nvcc.

    python -m mnmgdatalog_b200.build [--force]

Objects go to mnmgdatalog_b200/_build/, the library to
mnmgdatalog_b200/libmnmgdl.so (in-tree, so it travels with the repository).
Rebuilds only what changed (sources or any header of csrc/ or include/).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmnmgdl.so")
BIN = os.path.join(PKG, "bin")
CLI_SRC = os.path.join(PKG, "cli", "dl_cli.cpp")
CLI_PROGRAMS = {"tc": 0, "sg": 1, "wcc": 2, "single_join": 3}

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC,
]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _compile(src: str, force: bool, extra: list[str]) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if force or not os.path.exists(obj) or os.path.getmtime(obj) < newest:
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, extra: list[str] | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = list(extra or [])
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, extra), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-Xlinker", "-z", "-Xlinker", "defs", "-o", tmp, *objs,
               "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_cli(force)
    if verbose:
        print(LIB)
    return LIB


def build_cli(force: bool = False) -> list[str]:
    """The reference-compatible command-line programs (mnmgdatalog_b200/bin/)."""
    os.makedirs(BIN, exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    outs = []
    for name, prog in CLI_PROGRAMS.items():
        exe = os.path.join(BIN, name)
        newest = max(os.path.getmtime(CLI_SRC), os.path.getmtime(LIB), os.path.getmtime(os.path.join(INCLUDE, "mnmgdl.h")))
        if force or not os.path.exists(exe) or os.path.getmtime(exe) < newest:
            cmd = [cxx, "-O2", "-std=c++17", f"-DDL_CLI_PROGRAM={prog}", "-I", INCLUDE, CLI_SRC, "-o", exe,
                   "-L", PKG, "-lmnmgdl", "-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
        outs.append(exe)
    return outs


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    if a.ptxas_info:
        os.makedirs(BUILD, exist_ok=True)
        for s in _sources():
            r = subprocess.run([nvcc(), *NVCC_FLAGS, *extra, "-c", s, "-o", os.devnull],
                               capture_output=True, text=True)
            sys.stdout.write(r.stderr)
        return 0
    build(force=a.force, verbose=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

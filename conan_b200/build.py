"""Builds the native parts of conan_b200 in-tree.

    python conan_b200/build.py          # library + CLI (the package itself
                                        # cannot be imported before this)
    python conan_b200/build.py --clean

Products (git-ignored, shipped with the tree):
    conan_b200/lib/libconan_pm.so   CUDA sm_100a kernels + the C ABI of include/conan_pm.h
    conan_b200/bin/conan            host CLI with the reference's `ic` and `run` commands

nvcc cross-compiles for sm_100a without a GPU; objects are rebuilt only when a
source or header is newer than the object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
CLI = PKG / "cli"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
BINDIR = PKG / "bin"
LIB = LIBDIR / "libconan_pm.so"
EXE = BINDIR / "conan"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                  "-Xcompiler", "-Wno-unknown-pragmas", f"-I{ROOT / 'include'}"]
CXX = shutil.which("g++") and "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def build(verbose: bool = False, extra_flags=()) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    BINDIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    sources = sorted(CSRC.glob("*.cu"))
    jobs = []
    objs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _newer(obj, [src, *headers, Path(__file__)]):
            jobs.append([NVCC, *NVFLAGS, *extra_flags, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd))
        list(ex.map(_run, jobs))
    if jobs or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcufft",
              "-Xlinker", f"-rpath,{CUDA_HOME / 'lib64'}"])
    cli_src = sorted(CLI.glob("*.cc"))
    cli_hdr = list(CLI.glob("*.hh")) + list((ROOT / "include").glob("*.h"))
    if cli_src and _newer(EXE, [*cli_src, *cli_hdr, LIB]):
        _run([CXX, "-std=c++17", "-O2", "-Wall", "-pthread", f"-I{ROOT / 'include'}", *map(str, cli_src),
              "-o", str(EXE), f"-L{LIBDIR}", "-lconan_pm", "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


def clean():
    for p in (BUILD, LIB, EXE):
        if p.is_dir():
            shutil.rmtree(p)
        elif p.exists():
            p.unlink()


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    if a.clean:
        clean()
    else:
        print(build(verbose=a.verbose))

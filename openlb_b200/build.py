"""Build recipe for liblbx.so (sm_100a) -- the CUDA library behind include/lbx.h.

    python -m openlb_b200.build            # compile what changed
    python -m openlb_b200.build --force    # rebuild everything

Each .cu under csrc/ is compiled by nvcc for sm_100a only (no PTX for other targets), and each
host-only .cpp by g++, into openlb_b200/_build/, then linked into openlb_b200/lib/liblbx.so.  The FP64 instantiation
units are compiled with -fmad=false: FP64 rounds like the reference's CPU build and the float
kernels fuse only where the source says so, identically in every kernel variant.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "liblbx.so"
INCLUDE = PKG.parent / "include"
PLATFORM = PKG / "platform"
HOST_EXAMPLES = {"cavity3d": PLATFORM / "cavity3d.cpp", "cavity2d": PLATFORM / "cavity2d.cpp"}

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills", "-I", str(INCLUDE), "-I", str(CSRC)]
# No implicit FMA contraction anywhere: FP64 keeps the reference's rounding, and the float
# kernels contract only where lbx_collision.cuh says so, identically in every kernel variant.
PER_UNIT = {}
COMMON.append("-fmad=false")


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; liblbx.so needs the CUDA toolkit to build")
    return cand


def _sources() -> list[Path]:
    """CUDA units (.cu, nvcc) and host-only units (.cpp, g++: the request server)."""
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers(src: Path) -> list[Path]:
    if src.suffix == ".cpp":
        return sorted(INCLUDE.glob("*.h"))
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "lbx.h"]


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if src.suffix == ".cpp":
        gxx = shutil.which("g++") or "/usr/bin/g++"
        cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-fPIC", "-pthread", "-I", str(INCLUDE), "-c", str(src),
               "-o", str(obj)]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"g++ failed for {src.name}:\n{proc.stdout}\n{proc.stderr}")
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *PER_UNIT.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{proc.stdout}\n{proc.stderr}")
    if verbose and proc.stderr:
        sys.stderr.write(proc.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile changed units and (re)link liblbx.so; returns the library path."""
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    todo = []
    for src in _sources():
        obj = BUILD / (src.stem + ".o")
        newest_header = max((p.stat().st_mtime for p in _headers(src)), default=0.0)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            todo.append(src)
    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as pool:
        list(pool.map(lambda s: _compile(s, verbose), todo))
    objs = [BUILD / (s.stem + ".o") for s in _sources()]
    if force or todo or not LIB.exists():
        cmd = [nvcc(), *ARCH, "-shared", "--cudart", "static", "-Xcompiler", "-pthread", "-o", str(LIB),
               *map(str, objs)]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed:\n{proc.stdout}\n{proc.stderr}")
    build_host_examples()
    return LIB


def build_host_examples() -> list[Path]:
    """C++ programs over the C++ host layer (platform/lbx.hpp), linked against liblbx.so with
    an rpath to it: g++, no CUDA headers."""
    gxx = shutil.which("g++") or "/usr/bin/g++"
    out = []
    for name, src in HOST_EXAMPLES.items():
        exe = LIB.parent / name
        deps = [src, PLATFORM / "lbx.hpp", INCLUDE / "lbx.h", LIB]
        if not exe.exists() or exe.stat().st_mtime < max(p.stat().st_mtime for p in deps):
            cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", str(INCLUDE), "-I", str(PLATFORM), str(src),
                   "-L", str(LIB.parent), "-llbx", "-Wl,-rpath,$ORIGIN", "-o", str(exe)]
            proc = subprocess.run(cmd, capture_output=True, text=True)
            if proc.returncode != 0:
                raise RuntimeError(f"g++ failed for {src.name}:\n{proc.stdout}\n{proc.stderr}")
        out.append(exe)
    return out


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="pass -Xptxas=-v (registers, spills)")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose, jobs=a.jobs))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

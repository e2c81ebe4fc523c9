"""Builds the engine in-tree: swifttn93_b200/lib/libtn93g.so (sm_100a kernels + the C ABI of include/tn93g.h) and
swifttn93_b200/bin/tn93g (the tn93 command line linked against it).

    python -m swifttn93_b200.build            # build (skips up-to-date outputs)
    python -m swifttn93_b200.build --force
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib" / "libtn93g.so"
CLI = PKG / "bin" / "tn93g"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# the C++ compiler on PATH (an exported CXX may point at a toolchain without the needed runtime)
HOSTCXX = "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DEVICE_SOURCES = ["engine.cu"]
HOST_SOURCES = ["tables.cpp", "logtable.cpp", "summary_json.cpp", "fasta.cpp"]
HEADERS = ["kernels.cuh", "tn93_math.cuh", "tables.h"]


def _newer(out: Path, deps) -> bool:
    if not out.exists():
        return False
    t = out.stat().st_mtime
    return all(Path(d).stat().st_mtime <= t for d in deps)


def _run(cmd, log: Path | None = None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.write_text(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-6000:] + r.stderr[-6000:])
        raise RuntimeError(f"build step failed: {' '.join(map(str, cmd[:3]))} ...")
    return r


def build_lib(force=False) -> Path:
    deps = [CSRC / s for s in DEVICE_SOURCES + HOST_SOURCES + HEADERS] + [REPO / "include" / "tn93g.h"]
    if not force and _newer(LIB, deps):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    objdir = PKG / "lib" / "_obj"
    objdir.mkdir(exist_ok=True)
    objs = []
    for s in DEVICE_SOURCES:
        o = objdir / (s + ".o")
        _run([NVCC, "-O3", *ARCH, "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xptxas", "-v", f"-I{REPO / 'include'}", f"-I{CSRC}", "-ccbin", HOSTCXX, "-c", str(CSRC / s),
              "-o", str(o)], log=objdir / (s + ".ptxas.log"))
        objs.append(o)
    for s in HOST_SOURCES:
        o = objdir / (s + ".o")
        _run([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", f"-I{REPO / 'include'}", f"-I{CSRC}",
              "-c", str(CSRC / s), "-o", str(o)])
        objs.append(o)
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, *ARCH, "-shared", "-ccbin", HOSTCXX, "-o", str(tmp), *map(str, objs), "-lquadmath",
          "-Xlinker", "-soname=libtn93g.so"])
    tmp.replace(LIB)
    return LIB


def build_cli(force=False) -> Path:
    lib = build_lib(force)
    deps = [CSRC / "cli.cpp", REPO / "include" / "tn93g.h", lib]
    if not force and _newer(CLI, deps):
        return CLI
    CLI.parent.mkdir(parents=True, exist_ok=True)
    tmp = CLI.with_name("tn93g.tmp")
    _run([HOSTCXX, "-O2", "-std=c++17", "-pthread", f"-I{REPO / 'include'}", str(CSRC / "cli.cpp"), "-o", str(tmp),
          f"-L{lib.parent}", "-ltn93g", "-Wl,-rpath,$ORIGIN/../lib"])
    tmp.replace(CLI)
    return CLI


def build_all(force=False):
    build_cli(force)
    return LIB, CLI


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(LIB)
    print(CLI)

"""Build recipe for the native library (libgpe_cuda.so, sm_100a) and the
C++ host driver.  Everything is built in-tree so the binaries travel with
the source tree; nvcc cross-compiles for sm_100a without a GPU.

    python -m gpe_b200.build          # incremental
    python -m gpe_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libgpe_cuda.so"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "--expt-relaxed-constexpr", "-I", str(INCLUDE)] + ARCH

CU_SOURCES = sorted(p.name for p in CSRC.glob("*.cu"))
CPP_SOURCES = sorted(p.name for p in CSRC.glob("*.cpp"))
HEADERS = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _newest(paths) -> float:
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    if src.suffix == ".cu":
        cmd = [NVCC, *NVFLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I", str(INCLUDE),
               "-I", "/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
    _run(cmd, verbose)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    hdr_time = _newest(HEADERS)
    jobs = []
    objs = []
    for name in CU_SOURCES + CPP_SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_time):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for f in [ex.submit(_compile, s, o, verbose) for s, o in jobs]:
                f.result()
    if force or jobs or not LIB.exists():
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcufft"], verbose)
    return LIB


BIN = PKG / "bin"
HOST_SRC = CSRC / "host" / "gpe_host.cpp"
HOST = BIN / "gpe_host"


def build_host(force: bool = False, verbose: bool = False) -> Path:
    """The C++ driver that runs the reference's time loop over the C ABI."""
    BIN.mkdir(exist_ok=True)
    if force or not HOST.exists() or HOST.stat().st_mtime < max(HOST_SRC.stat().st_mtime, LIB.stat().st_mtime):
        _run(["g++", "-std=c++17", "-O2", "-Wall", "-I", str(INCLUDE), str(HOST_SRC), "-o", str(HOST),
              "-L", str(LIBDIR), "-lgpe_cuda", "-Wl,-rpath,$ORIGIN/../lib"], verbose)
    return HOST


def build_oracle(verbose: bool = False) -> None:
    """The CPU oracle is test infrastructure; it has its own recipe."""
    _run(["make", "-s", "-C", str(ROOT / "oracle")], verbose)


def main(argv: list[str]) -> int:
    force = "--force" in argv
    verbose = "-v" in argv or "--verbose" in argv
    lib = build_library(force=force, verbose=verbose)
    host = build_host(force=force, verbose=verbose)
    print(f"built {lib} and {host}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))

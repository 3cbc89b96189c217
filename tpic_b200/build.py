"""Builds the sm_100a shared library tpic_b200/libtpicb200.so with nvcc.

Every kernel file is compiled for `-gencode arch=compute_100a,code=sm_100a`
with line info; the mover and the particle loader are compiled with
`-fmad=false` so that their arithmetic rounds every multiply and add on its
own, like the reference's expressions under strict IEEE evaluation. The library is built in-tree so
that it travels with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIBRARY = HERE / "libtpicb200.so"
DRIVER = HERE / "tpicb200_run"
DRIVER_SOURCE = HERE / "host" / "tpicb200_run.cpp"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]
PER_FILE = {"mover.cu": ["-fmad=false"], "load.cu": ["-fmad=false"]}
SOURCES = ["abi.cu", "mover.cu", "sort.cu", "deposit.cu", "fields.cu", "solver.cu", "mass_tc.cu", "cases.cu",
           "load.cu", "checkpoint.cu", "adjoint.cu", "output.cu", "gauss.cu"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else "nvcc"


def _compile(source: str) -> Path:
    obj = BUILD / (source + ".o")
    src = CSRC / source
    deps = [src] + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "tpicb200.h"]
    if obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, *PER_FILE.get(source, []), "-c", str(src), "-o", str(obj)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source}:\n{result.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objects = list(pool.map(_compile, SOURCES))
    newest = max(o.stat().st_mtime for o in objects)
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-lcudart"]
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"link failed:\n{result.stderr}")
    build_driver()
    if verbose:
        print(f"built {LIBRARY} and {DRIVER}")
    return LIBRARY


def build_driver() -> Path:
    """The C++ host driver tpicb200_run (g++, linked against the in-tree
    library and the CUDA runtime; no Python)."""
    cuda = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
    deps = [DRIVER_SOURCE, HERE.parent / "include" / "tpicb200.h", LIBRARY]
    if DRIVER.exists() and DRIVER.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", f"-I{cuda / 'include'}", str(DRIVER_SOURCE), "-o",
           str(DRIVER), f"-L{HERE}", "-ltpicb200", f"-L{cuda / 'lib64'}", "-lcudart", "-Wl,-rpath,$ORIGIN",
           f"-Wl,-rpath,{cuda / 'lib64'}"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0 or result.stderr.strip():
        raise RuntimeError(f"driver build failed or warned:\n{result.stderr}")
    return DRIVER


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)

"""Builds libmettle_cuda.so (and libmettle_cuda.a) in-tree for sm_100a.

Every CUDA and C++ source under csrc/ is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a``; objects go to csrc/_build/ and
are rebuilt only when a source or header is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = CSRC / "_build"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libmettle_cuda.so"
STATIC = HERE / "libmettle_cuda.a"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I", str(CSRC), "-I", str(INCLUDE)]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else (shutil.which("nvcc") or "nvcc")


def host_compiler() -> list[str]:
    # /usr/bin/g++ carries the full runtime; a CXX from the environment may not.
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if Path(gxx).exists() else []


def sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def headers() -> list[Path]:
    return [*CSRC.glob("*.h"), *CSRC.glob("*.cuh"), *INCLUDE.glob("*.h")]


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    newest = max([src.stat().st_mtime, *[h.stat().st_mtime for h in headers()]])
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [nvcc(), *host_compiler(), *ARCH, *CFLAGS, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd[cmd.index("-c") : cmd.index("-c")] = ["-x", "cu"] if False else []
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip() and verbose:
        print(res.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compiles every source and links the shared and static libraries."""
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread",
               "-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        # Static archive for a Rust build.rs (links with -lcudart_static).
        if STATIC.exists():
            STATIC.unlink()
        subprocess.run(["ar", "rcs", str(STATIC), *map(str, objs)], check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

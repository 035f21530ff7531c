"""Builds libpcc_gpu.so (sm_100a) in place from csrc/*.cu with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = ["pcc_api.cu", "pcc_scan_sort.cu", "pcc_detect.cu", "pcc_solver.cu", "pcc_planar.cu", "pcc_update.cu", "pcc_noalloc.cu",
           "pcc_serve.cu", "pcc_vtk.cu"]
OUT = PKG / "libpcc_gpu.so"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [PKG / "csrc" / s for s in SOURCES] + list((PKG / "csrc").glob("*.cuh")) + \
        list((PKG / "csrc").glob("*.hpp")) + [ROOT / "include" / "pcc_gpu.h"]
    return any(d.stat().st_mtime > t for d in deps)


CLI = PKG / "pcc_cellcollectives"


def build_cli(verbose: bool = False) -> Path:
    """The C++ command-line driver over the C ABI (links libpcc_gpu.so)."""
    src = PKG / "host" / "pcc_cellcollectives.cpp"
    deps = [src, PKG / "host" / "pcc_adapter.hpp", ROOT / "include" / "pcc_gpu.h", OUT]
    if CLI.exists() and all(d.stat().st_mtime <= CLI.stat().st_mtime for d in deps):
        return CLI
    cmd = ["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", f"-I{PKG / 'host'}", "-o", str(CLI), str(src),
           f"-L{PKG}", "-lpcc_gpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return CLI


OBJ_DIR = PKG / "_build"


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every source to an object in parallel (no device code crosses
    files), then links the shared library."""
    if not force and not needs_build():
        build_cli(verbose)
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    OBJ_DIR.mkdir(exist_ok=True)
    inc = [f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc'}"]
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]

    def compile_one(src: str) -> Path:
        obj = OBJ_DIR / (Path(src).stem + ".o")
        cmd = [nvcc(), *compile_flags, *inc, "-c", "-o", str(obj), str(PKG / "csrc" / src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(OUT) + ".tmp",
           *[str(o) for o in objs]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(OUT) + ".tmp", OUT)
    build_cli(verbose)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)

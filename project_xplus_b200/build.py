"""Builds the native library libxplus_b200.so (CUDA sm_100a kernels + C++ host code).

The library is compiled in-tree by nvcc with -gencode arch=compute_100a,code=sm_100a, so it
ships with the source tree.  The CUDA runtime is linked statically and libstdc++'s symbols
are kept private, so the library loads next to torch's own runtime without clashes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB_DIR = HERE / "lib"
LIB = LIB_DIR / "libxplus_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-O2,-Wall", "-Xptxas", "-O3"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + \
        [HERE.parent / "include" / "xplus_b200.h", Path(__file__), HERE / "exports.map"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile every source to an object, then link the shared library."""
    if not force and not needs_build():
        return LIB
    nvcc = nvcc_path()
    obj_dir = HERE / "_build"
    obj_dir.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = obj_dir / (src.name + ".o")
        objs.append(obj)
        if src.suffix == ".cu":
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        else:  # plain host C++ (no CUDA): the system compiler
            cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-c", str(src), "-o", str(obj)]
        procs.append((src, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, cmd, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src.name)
    if failed:
        raise RuntimeError(f"compilation failed: {failed}")
    link = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
            "-Xlinker", "--exclude-libs,ALL", "-Xlinker", f"--version-script={HERE / 'exports.map'}",
            "-Xcompiler", "-fPIC"]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

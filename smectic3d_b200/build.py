"""Build the sm_100a shared library ``libsmectic_b200.so`` in-tree.

Each translation unit under ``csrc/`` is compiled by nvcc for
``arch=compute_100a,code=sm_100a`` (in parallel) and linked into one
position-independent shared library next to this file, so that it travels
with the source tree.  No torch types cross the library boundary.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libsmectic_b200.so"
DRIVER = PKG / "smectic_run"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O2",
           f"-I{INCLUDE}"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = Path(cuda) / "bin" / "nvcc"
    return str(exe) if exe.exists() else (shutil.which("nvcc") or "nvcc")


def sources():
    return sorted(CSRC.glob("*.cu"))


def build_driver() -> Path:
    """g++ build of the host driver smectic_run against the in-tree library."""
    src = CSRC / "smectic_run.cpp"
    if DRIVER.exists() and DRIVER.stat().st_mtime > max(src.stat().st_mtime, LIB.stat().st_mtime):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", str(src), "-o", str(DRIVER), f"-L{PKG}", "-lsmectic_b200",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return DRIVER


def headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *headers()])


def _compile(src: Path, extra):
    obj = BUILD / (src.stem + ".o")
    if not _stale(obj, src):
        return obj, ""
    cmd = [nvcc(), *ARCH, *NVFLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, ptxas_info: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    objs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        futs = {ex.submit(_compile, s, extra): s for s in sources()}
        for f in cf.as_completed(futs):
            obj, log = f.result()
            objs.append(obj)
            if verbose and log:
                print(log, file=sys.stderr)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, sorted(objs)), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_driver()
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)

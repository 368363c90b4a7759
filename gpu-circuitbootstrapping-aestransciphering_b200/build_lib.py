"""Build libcbs_b200.so (sm_100a) in-tree.

Every .cu / .cpp under csrc/ is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into csrc/_build/ and linked
into ``libcbs_b200.so`` next to this file.  Incremental: a translation unit is rebuilt
when it or any header under csrc/ or include/ is newer than its object file.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libcbs_b200.so"
BUILD = CSRC / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                     "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC)]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libcbs_b200.so")
    return cand


def _host_cc() -> list[str]:
    # nvcc's host compiler: the system g++ (the image's /opt/gcc wrapper lacks libgomp)
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if Path(gxx).exists() else []


def sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def _headers_mtime() -> float:
    hs = [*CSRC.glob("*.cuh"), *CSRC.glob("*.h"), *(ROOT / "include").glob("*.h")]
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [_nvcc(), *_host_cc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, ptxas_info: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    hdr = _headers_mtime()
    todo, objs = [], []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if ptxas_info or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr):
            todo.append((src, obj))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
            for obj, err in ex.map(lambda t: _compile(t[0], t[1], extra), todo):
                if verbose or ptxas_info:
                    print(f"[build] {obj.name}\n{err}", file=sys.stderr)
    if todo or not OUT.exists():
        cmd = [_nvcc(), *_host_cc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(OUT)

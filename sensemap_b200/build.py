"""Build recipe for the engine's shared library (libsmvs.so, in-tree).

Compiles sensemap_b200/csrc with nvcc for sm_100a only. The translation units
are compiled in parallel and linked into ``sensemap_b200/libsmvs.so``; the
result is reused when no source is newer than it.
"""
from __future__ import annotations

import concurrent.futures as futures
import os
import shutil
import subprocess
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
LIB_PATH = PKG_DIR / "libsmvs.so"
BUILD_DIR = PKG_DIR / "_build"
INCLUDE_DIR = PKG_DIR.parent / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-v"]
NVCC_FLAGS = COMMON_FLAGS + ["--use_fast_math"]
# Units whose kernels must reproduce IEEE single-precision results exactly
# (no contraction into FMA, correctly rounded division and square root, no
# flush to zero): the cross-view filter's decisions and medians, and the
# depth tests of the initial maps, the fusion's consistency tests and medians.
EXACT_FLAGS = COMMON_FLAGS + ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
EXACT_UNITS = {"smvs_cross_filter.cu", "smvs_init_maps.cu", "smvs_fusion.cu", "smvs_pyramid.cu", "smvs_prior.cu"}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the engine needs the CUDA toolkit to build")


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _deps() -> list[Path]:
    return _sources() + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE_DIR.glob("*.h")) \
        + [Path(__file__)]


def needs_build() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def _compile(src: Path, nvcc: str) -> tuple[Path, str]:
    obj = BUILD_DIR / (src.name + ".o")
    flags = EXACT_FLAGS if src.name in EXACT_UNITS else NVCC_FLAGS
    cmd = [nvcc, *flags, *ARCH_FLAGS, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stderr}")
    return obj, res.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile libsmvs.so for sm_100a (no GPU needed). Returns its path."""
    if not force and not needs_build():
        return LIB_PATH
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    srcs = _sources()
    with futures.ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, nvcc), srcs))
    objs = [r[0] for r in results]
    if verbose:
        for _, log in results:
            print(log)
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))

"""Compile the REFERENCE's PatchMatch kernels into oracle/_ref/libref_pm.so.

Test infrastructure only (the second oracle). Sources are compiled where
they lie in the reference's source tree, named by the SMVS_REFERENCE_TREE
environment variable or --tree (nothing is copied): src/mvs/kernel_functions.cu
(through ref_kernels_n32.cu, which raises the 8-view cap to 32),
src/mvs/gpu_mat_ref_image.cu, src/mvs/gpu_mat_prng.cu and src/util/cudacc.cc,
plus this directory's ref_driver.cu, with the reference's own flags
(-O3 --use_fast_math, CMakeLists.txt:143) for sm_100a. Third-party headers the
reference includes are replaced by the small stand-ins in ref_shim/ (glog
CHECK macros, a boost::filesystem::path, base/reconstruction.h -> Eigen), and
Eigen comes from the reference's own bundled copy (3rdParty/VCG/eigenlib).
The library is built where the reference tree is and runs where a GPU is; the
reference tree is read at build time only. Without a tree the recipe does
nothing and exits 0.

    SMVS_REFERENCE_TREE=<reference checkout> python oracle/ref_build.py
"""
from __future__ import annotations

import concurrent.futures as futures
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("SMVS_REFERENCE_TREE", "")) if os.environ.get("SMVS_REFERENCE_TREE") else None
OUT = HERE / "_ref"
LIB = OUT / "libref_pm.so"
NVCC = "/usr/local/cuda/bin/nvcc"
FLAGS_BASE = ["-std=c++14", "-O3", "--use_fast_math", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-include", "vector", "-include", "cfloat", "-include", "algorithm"]


def _flags():
    return FLAGS_BASE + [f"-I{HERE / 'ref_shim'}", f"-I{REF / 'src'}", f"-I{REF / '3rdParty/VCG/eigenlib'}", "-w"]


def sources():
    return [HERE / "ref_kernels_n32.cu", REF / "src/mvs/gpu_mat_ref_image.cu", REF / "src/mvs/gpu_mat_prng.cu",
            REF / "src/util/cudacc.cc", HERE / "ref_shim/shim_string.cc", HERE / "ref_driver.cu"]


def build(force: bool = False) -> Path:
    if REF is None or not REF.exists():
        raise FileNotFoundError("reference tree not found: set SMVS_REFERENCE_TREE (or pass --tree)")
    deps = [p for p in sources()] + [Path(__file__), *HERE.glob("ref_shim/**/*")]
    if LIB.exists() and not force and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in deps if p.is_file()):
        return LIB
    OUT.mkdir(exist_ok=True)

    def compile_one(src: Path) -> Path:
        obj = OUT / (src.name + ".o")
        lang = ["-x", "cu"] if src.suffix == ".cc" else []
        res = subprocess.run([NVCC, *_flags(), *lang, "-c", str(src), "-o", str(obj)], capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"compiling {src} failed:\n{res.stderr[-4000:]}")
        return obj

    with futures.ThreadPoolExecutor(max_workers=6) as ex:
        objs = list(ex.map(compile_one, sources()))
    res = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(LIB),
                          *map(str, objs), "-lcudart"], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
    for o in objs:
        o.unlink()
    return LIB


if __name__ == "__main__":
    if "--tree" in sys.argv:
        REF = Path(sys.argv[sys.argv.index("--tree") + 1])
    if REF is None or not REF.exists():  # no reference tree here: nothing to check against
        print("reference tree not given or not found (SMVS_REFERENCE_TREE / --tree); reference kernels not built",
              file=sys.stderr)
        sys.exit(0)
    try:
        print(build(force="--force" in sys.argv))
    except Exception as exc:  # reported, not fatal: the engine build does not depend on it
        print(f"reference kernels not built: {exc}", file=sys.stderr)
        sys.exit(1)

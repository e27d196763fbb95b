"""Build recipe for the CPU oracle (oracle/_build/libsmvs_oracle.so).

Test infrastructure only. Plain gcc + OpenMP; x86-64-v3 (AVX2/FMA) so the
library built here also runs on the GPU hosts' CPUs.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

ORACLE_DIR = Path(__file__).resolve().parent
BUILD_DIR = ORACLE_DIR / "_build"
LIB_PATH = BUILD_DIR / "libsmvs_oracle.so"
# (source, extra flags). The cross-filter unit performs exactly the IEEE
# operations its CUDA counterpart spells out, so nothing may be contracted.
SOURCES = [(ORACLE_DIR / "smvs_oracle.c", []),
           (ORACLE_DIR / "smvs_oracle_filter.c", ["-ffp-contract=off"]),
           (ORACLE_DIR / "smvs_oracle_init.c", ["-ffp-contract=off"]),
           (ORACLE_DIR / "smvs_oracle_fusion.c", ["-ffp-contract=off"]),
           (ORACLE_DIR / "smvs_oracle_pyramid.c", ["-ffp-contract=off"]),
           (ORACLE_DIR / "smvs_oracle_prior.c", ["-ffp-contract=off"])]
DEPS = [src for src, _ in SOURCES] + [ORACLE_DIR / "smvs_oracle.h", ORACLE_DIR / "orc_pose.h",
                                      ORACLE_DIR.parent / "include" / "smvs.h", Path(__file__)]
CFLAGS = ["-std=c11", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-Wall", "-Wextra"]


def needs_build() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    return any(p.stat().st_mtime > t for p in DEPS)


def build(force: bool = False) -> Path:
    if not force and not needs_build():
        return LIB_PATH
    BUILD_DIR.mkdir(exist_ok=True)
    tmp = LIB_PATH.with_suffix(".so.tmp")
    errors = []
    # The system gcc ships libgomp; a CC wrapper may not, so it is the fallback.
    for cc in dict.fromkeys(c for c in (shutil.which("gcc"), os.environ.get("CC"), "cc") if c):
        objs, failed = [], None
        for src, extra in SOURCES:
            obj = BUILD_DIR / (src.stem + ".o")
            res = subprocess.run([cc, *CFLAGS, *extra, "-c", str(src), "-o", str(obj)], capture_output=True, text=True)
            if res.returncode != 0:
                failed = res.stderr
                break
            objs.append(str(obj))
        if failed is None:
            res = subprocess.run([cc, "-shared", "-fopenmp", *objs, "-o", str(tmp), "-lm"], capture_output=True,
                                 text=True)
            if res.returncode == 0:
                break
            failed = res.stderr
        errors.append(f"{cc}: {failed}")
    else:
        raise RuntimeError("oracle build failed:\n" + "\n".join(errors))
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True))

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
SOURCES = [ORACLE_DIR / "smvs_oracle.c"]
DEPS = SOURCES + [ORACLE_DIR / "smvs_oracle.h", ORACLE_DIR.parent / "include" / "smvs.h", Path(__file__)]
CFLAGS = ["-std=c11", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-Wall", "-Wextra"]


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
        cmd = [cc, *CFLAGS, *map(str, SOURCES), "-o", str(tmp), "-lm"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode == 0:
            break
        errors.append(f"{cc}: {res.stderr}")
    else:
        raise RuntimeError("oracle build failed:\n" + "\n".join(errors))
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True))

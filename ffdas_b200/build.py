"""Build libffdas_b200.so in-tree with nvcc for sm_100a.

Usage: python ffdas_b200/build.py [--force] [--jobs N] [--debug]
(run as a script: importing the package first would load the old library)

Every CUDA source under ffdas_b200/csrc is compiled separately (in parallel)
with the flags the reference also uses for arithmetic parity
(--ftz=true --fmad=true, CMakeLists.txt:74 of the reference) and linked into
one shared library exporting the C-ABI declared in include/ffdas.h.
The CUDA runtime is linked statically so the library only needs the driver.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libffdas_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--ftz=true", "--fmad=true",
    "-Xcompiler", "-fPIC,-fvisibility=hidden", "-Xptxas", "-v",
    "--expt-relaxed-constexpr", "-Dffdas_EXPORTS",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libffdas_b200.so")
    return exe


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _needs_build(force: bool) -> bool:
    if force or not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = _sources() + _headers() + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def _compile(src: Path, debug: bool) -> tuple[Path, str]:
    obj = BUILD / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
    if debug:
        cmd += ["-DFFDAS_DEVICE_CHECKS=1"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, jobs: int | None = None, debug: bool = False, verbose: bool = False) -> Path:
    """Compile and link the library if any source is newer than it."""
    if not _needs_build(force):
        return LIB
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = []
        for obj, log in ex.map(lambda s: _compile(s, debug), srcs):
            objs.append(obj)
            logs.append(log)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs),
           "-Xlinker", "-Bsymbolic", "-Xlinker", "--no-undefined", "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    (BUILD / "ptxas.log").write_text("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, debug=a.debug, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())

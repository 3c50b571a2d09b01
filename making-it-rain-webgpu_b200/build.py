"""Build the engine library, lib/libmdb200.so, for sm_100a.

  python making-it-rain-webgpu_b200/build.py [--verbose] [--ptxas-info]

nvcc compiles every kernel file and the host runtime in csrc/ in one
invocation, links the CUDA runtime statically, and writes the library in-tree
so it travels with the repository snapshot.  The build is skipped when the
library is newer than every source.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "lib" / "libmdb200.so"
INCLUDE = HERE.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def nvcc() -> str:
    for candidate in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found; the engine cannot be built without it")


def host_compiler() -> list[str]:
    # The image's default CXX may lack parts of its runtime; prefer the system g++.
    for candidate in ("/usr/bin/g++",):
        if Path(candidate).exists():
            return ["-ccbin", candidate]
    return []


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    built = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in sources() + headers() + [Path(__file__)])


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    if not force and up_to_date() and not ptxas_info:
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc(), *host_compiler(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-cudart", "static", "--expt-relaxed-constexpr",
           "-I", str(INCLUDE), "-o", str(LIB), *map(str, sources())]
    if ptxas_info:
        cmd.insert(1, "-Xptxas=-v")
    if verbose:
        print(" ".join(cmd))
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError("nvcc failed building libmdb200.so")
    if verbose or ptxas_info:
        sys.stderr.write(result.stderr)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    args = ap.parse_args()
    path = build(force=args.force, verbose=args.verbose, ptxas_info=args.ptxas_info)
    print(path)


if __name__ == "__main__":
    main()

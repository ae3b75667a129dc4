"""Build recipe for the in-tree CUDA library ``steam_b200/_lib/libsteam_b200.so``.

Compiles every ``steam_b200/csrc/*.cu`` for sm_100a with nvcc and links one
shared library exposing the C ABI declared in ``include/steam_b200.h``.  The
library is built in-tree so it travels with the repository snapshot.

Usage: ``python -m steam_b200.build [--force] [--verbose]``.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_DIR = PACKAGE_DIR.parent
CSRC = PACKAGE_DIR / "csrc"
INCLUDE = REPO_DIR / "include"
LIB_DIR = PACKAGE_DIR / "_lib"
LIB_PATH = LIB_DIR / "libsteam_b200.so"
BUILD_DIR = REPO_DIR / "_build"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "--std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"),
                 "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build steam_b200")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile (if stale) and return the path of the shared library."""
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objects = []
    for src in sources():
        obj = BUILD_DIR / (src.stem + ".o")
        objects.append(obj)
        if force or ptxas_info or _stale(obj, [src] + headers):
            cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, "-I", str(INCLUDE), "-c",
                   str(src), "-o", str(obj)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
            if verbose or ptxas_info:
                sys.stdout.write(res.stdout + res.stderr)
    if force or _stale(LIB_PATH, objects):
        cmd = [nvcc, *ARCH_FLAGS, "-shared", "-cudart", "static", "-o",
               str(LIB_PATH), *map(str, objects)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true",
                    help="rebuild with -Xptxas -v (registers, spills, smem)")
    args = ap.parse_args(argv)
    path = build(force=args.force, verbose=args.verbose, ptxas_info=args.ptxas_info)
    print(path)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

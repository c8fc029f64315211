"""Builds libqpb.so, the sm_100a backend, in-tree with nvcc.

    python -m qoraphasecu_b200.build [-v] [--force]

Objects go to ``_build/`` at the repository root; the shared library lands in
``qoraphasecu_b200/libqpb.so`` so that it travels with the source tree.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
BUILD = ROOT / "_build"
LIBRARY = PACKAGE / "libqpb.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH,
    "-O3",
    "-lineinfo",
    "-std=c++20",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-Wall",
    "-Xcompiler", "-g",
    "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", str(ROOT / "include"),
]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else "nvcc"


def _sources():
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def _headers():
    return [*CSRC.glob("*.cuh"), *CSRC.glob("*.hpp"), *(ROOT / "include").glob("*.h")]


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compiles every source for sm_100a and links libqpb.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objects = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objects.append(obj)
        stale = (
            force
            or not obj.exists()
            or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        )
        if stale:
            jobs.append((src, obj))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as pool:
            for f in [pool.submit(_compile, s, o, verbose) for s, o in jobs]:
                f.result()
    if jobs or force or not LIBRARY.exists():
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIBRARY


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("-v", "--verbose", action="store_true")
    parser.add_argument("--force", action="store_true")
    args = parser.parse_args(argv)
    print(build(verbose=args.verbose, force=args.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())

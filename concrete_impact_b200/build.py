"""Build recipe for the in-tree sm_100a shared library ``libcib200.so``.

The library is plain nvcc output (``-shared -Xcompiler -fPIC``) exposing the C ABI of
``include/cib200.h``; Python loads it with ctypes.  Objects are compiled in parallel and
only rebuilt when a source or header is newer than the object.

Usage: ``python -m concrete_impact_b200.build [--force] [-v]``.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_DIR = PACKAGE_DIR.parent
CSRC_DIR = PACKAGE_DIR / "csrc"
INCLUDE_DIR = REPO_DIR / "include"
BUILD_DIR = PACKAGE_DIR / "_build"
LIB_PATH = PACKAGE_DIR / "libcib200.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    "-Xptxas",
    "-warn-spills",
]


def nvcc_path() -> str:
    """Locate nvcc (CUDA_HOME, then /usr/local/cuda, then PATH)."""
    candidates = []
    if os.environ.get("CUDA_HOME"):
        candidates.append(Path(os.environ["CUDA_HOME"]) / "bin" / "nvcc")
    candidates.append(Path("/usr/local/cuda/bin/nvcc"))
    for candidate in candidates:
        if candidate.exists():
            return str(candidate)
    found = shutil.which("nvcc")
    if found is None:
        raise RuntimeError("nvcc not found; set CUDA_HOME.")
    return found


def _sources() -> list[Path]:
    return sorted(CSRC_DIR.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC_DIR.glob("*.cuh")) + sorted(INCLUDE_DIR.glob("*.h"))


def _newest(paths: list[Path]) -> float:
    return max((p.stat().st_mtime for p in paths), default=0.0)


def _compile(source: Path, verbose: bool, force: bool, header_time: float) -> Path:
    obj = BUILD_DIR / (source.stem + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(source.stat().st_mtime, header_time):
        return obj
    cmd = [nvcc_path(), *ARCH_FLAGS, *NVCC_FLAGS, f"-I{INCLUDE_DIR}", "-c", str(source), "-o", str(obj)]
    if verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{result.stderr}")
    if verbose and result.stderr:
        sys.stderr.write(result.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every ``csrc/*.cu`` for sm_100a and link ``libcib200.so``; return its path."""
    BUILD_DIR.mkdir(exist_ok=True)
    sources = _sources()
    header_time = _newest(_headers())
    workers = max(1, min(len(sources), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        objects = list(pool.map(lambda s: _compile(s, verbose, force, header_time), sources))
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < _newest(objects):
        tmp = LIB_PATH.with_suffix(".so.tmp")
        cmd = [nvcc_path(), *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objects), "-lcudart"]
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{result.stderr}")
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    parser.add_argument("-v", "--verbose", action="store_true", help="print ptxas resource usage")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()

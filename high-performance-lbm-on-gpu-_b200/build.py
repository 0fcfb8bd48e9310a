"""Build ``liblbm_b200.so`` in-tree with nvcc for sm_100a.

    python -m lbm_b200.build          (or: python high-performance-lbm-on-gpu-_b200/build.py)

Each ``csrc/*.cu`` compiles to an object in ``_build/`` in parallel, then the
objects link into ``liblbm_b200.so`` next to this file. ``-Xptxas -v``
output (registers, spills, shared memory per kernel) is kept in
``_build/ptxas.log``. A rebuild happens only when a source or header is newer
than the library.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
BUILD = HERE / "_build"
LIBRARY = HERE / "liblbm_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", f"-I{INCLUDE}"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build liblbm_b200.so")
    return path


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _inputs() -> list[Path]:
    return sources() + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h")) + [Path(__file__)]


def up_to_date() -> bool:
    if not LIBRARY.exists():
        return False
    built = LIBRARY.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in _inputs())


def _compile(src: Path) -> tuple[Path, str]:
    obj = BUILD / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{proc.stderr}")
    return obj, proc.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIBRARY
    BUILD.mkdir(exist_ok=True)
    jobs = min(len(sources()), os.cpu_count() or 4)
    with ThreadPoolExecutor(jobs) as pool:
        results = list(pool.map(_compile, sources()))
    objects = [obj for obj, _ in results]
    (BUILD / "ptxas.log").write_text("".join(log for _, log in results))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objects), "-lcudart"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{proc.stderr}")
    os.replace(tmp, LIBRARY)
    if verbose:
        print(f"built {LIBRARY}")
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

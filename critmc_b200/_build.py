"""Compile the CUDA sources of the package into ``critmc_b200/libcritmc_b200.so``.

Every ``csrc/*.cu`` file is compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) and linked into one shared library that
exports the C ABI declared in ``include/critmc_b200.h``.  Objects go to
``critmc_b200/_build/``; a file is recompiled when it or any header is newer
than its object.  nvcc cross-compiles, so this works on a machine without a GPU.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libcritmc_b200.so"
# bounds-checked flavour (-DCRITMC_CHECK, see critmc_check_report): own objects and library
BUILD_CHECK = PKG / "_build_check"
LIB_CHECK = PKG / "libcritmc_b200_check.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O2",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build critmc_b200")
    return exe


# translation units whose float arithmetic must match a host replay exactly
PER_FILE_FLAGS = {"on_models.cu": ["--fmad=false"], "ea_pt.cu": ["--fmad=false"], "flathist.cu": ["--fmad=false"],
                  "cluster.cu": ["--fmad=false"]}


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _compile(src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *PER_FILE_FLAGS.get(src.name, []), *extra, "-c", str(src),
           "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None, check: bool = False) -> Path:
    """Build the shared library (incrementally) and return its path.

    ``check``: the bounds-checked flavour (-DCRITMC_CHECK) into its own
    object folder and ``libcritmc_b200_check.so``."""
    extra = list(extra or [])
    build_dir, lib_path = BUILD, LIB
    if check:
        extra.append("-DCRITMC_CHECK")
        build_dir, lib_path = BUILD_CHECK, LIB_CHECK
    build_dir.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    newest_header = max((p.stat().st_mtime for p in _headers()), default=0.0)
    jobs = []
    objects = []
    for src in sources:
        obj = build_dir / (src.stem + ".o")
        objects.append(obj)
        stale = (
            force
            or not obj.exists()
            or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        )
        if stale:
            jobs.append((src, obj))
    if jobs:
        workers = max(1, min(len(jobs), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(workers) as ex:
            futs = [ex.submit(_compile, s, o, extra) for s, o in jobs]
            for f in futs:
                f.result()
        if verbose:
            print(f"compiled {[s.name for s, _ in jobs]}")
    if jobs or not lib_path.exists() or lib_path.stat().st_mtime < max(o.stat().st_mtime for o in objects):
        tmp = lib_path.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objects), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    import sys

    print(build(force="--force" in sys.argv, verbose=True, check="--check" in sys.argv))

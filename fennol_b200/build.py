"""Build the sm_100a shared library ``fennol_b200/lib/libfennol_b200.so``.

Every ``csrc/*.cu`` file is compiled by ``nvcc`` for ``sm_100a`` (the build
cross-compiles without a GPU) and linked into one shared library with a plain
C ABI (``include/fennol_b200.h``).  The library is built in-tree so it travels
with the source tree.

    python -m fennol_b200.build [--force] [--verbose]
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
LIBDIR = PKG / "lib"
LIBNAME = "libfennol_b200.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-diag-suppress", "177"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build fennol_b200")


def library_path() -> Path:
    return LIBDIR / LIBNAME


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _headers():
    return sorted(list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return t < src.stat().st_mtime or t < newest_header


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> Path:
    nvcc = nvcc_path()
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    srcs = _sources()
    jobs = []
    for src in srcs:
        obj = BUILD / (src.stem + ".o")
        if force or _stale(obj, src, newest_header):
            cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, *extra_flags, f"-I{INCLUDE}", f"-I{CSRC}",
                   "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        p = subprocess.run(cmd, capture_output=True, text=True)
        return src, p

    failed = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for src, p in ex.map(run, jobs):
                if verbose or p.returncode != 0:
                    sys.stderr.write(p.stdout + p.stderr)
                if p.returncode != 0:
                    failed.append(src.name)
    if failed:
        raise RuntimeError(f"nvcc failed for: {', '.join(failed)}")
    lib = library_path()
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    if force or jobs or not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-lcuda"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stdout + p.stderr)
        os.replace(tmp, lib)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()

"""Build the shearwave_b200 CUDA library in-tree.

    python -m shearwave_b200.build [--force] [--verbose]

Every ``csrc/*.cu`` file is compiled for sm_100a with nvcc and linked into
``shearwave_b200/_lib/libshearwave_b200.so`` (static CUDA runtime, plain C
ABI declared in ``include/shearwave_b200.h``).  Objects go to ``_build/``.
A file is recompiled when it or any header is newer than its object.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIBDIR = PKG / "_lib"
LIBNAME = "libshearwave_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-O3",
    "--expt-relaxed-constexpr",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build shearwave_b200")


def lib_path() -> Path:
    return LIBDIR / LIBNAME


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile and link the library; returns the path of the shared object."""
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    cc = nvcc()
    srcs = sorted(CSRC.glob("*.cu"))
    deps = _headers()
    flags = NVCC_FLAGS + (extra_flags or [])
    jobs = []
    objs = []
    for src in srcs:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            jobs.append([cc, *ARCH, *flags, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    out = lib_path()
    if force or jobs or not out.exists():
        tmp = out.with_suffix(".so.tmp")
        run([cc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)])
        os.replace(tmp, out)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else None
    p = build(force=a.force or a.ptxas_info, verbose=a.verbose or a.ptxas_info, extra_flags=extra)
    print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())

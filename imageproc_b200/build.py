"""Build the sm_100a shared library ``imageproc_b200/libimageproc_b200.so``.

Every ``csrc/*.cu`` file is compiled by nvcc for ``sm_100a`` only
(``-gencode arch=compute_100a,code=sm_100a``; no PTX for other targets, no
fast-math) and linked, with the static CUDA runtime, into one shared library
that exports the C ABI declared in ``include/imageproc_b200.h``. Objects go to
``imageproc_b200/_build/``; a source is recompiled when it or any header is
newer than its object.

Usage: python -m imageproc_b200.build [--verbose] [--ptxas-info]
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
BUILD = PKG / "_build"
LIB = PKG / "libimageproc_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build imageproc_b200")


def common_flags() -> list[str]:
    return ARCH + [
        "-O3", "-std=c++17", "-lineinfo",
        "-I", str(ROOT / "include"), "-I", str(CSRC),
        "-Xcompiler", "-fPIC,-fvisibility=hidden",
    ]


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(verbose: bool = False, ptxas_info: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr = _headers_mtime()
    cc = nvcc()

    def compile_one(src: Path) -> tuple[Path, str]:
        obj = BUILD / (src.stem + ".o")
        if obj.exists() and not ptxas_info and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr):
            return obj, ""
        cmd = [cc, *common_flags(), "-c", str(src), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stdout + r.stderr

    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, srcs))
    for obj, log in results:
        if log and (verbose or ptxas_info):
            print(f"--- {obj.name}\n{log}", file=sys.stderr)
    objs = [str(o) for o, _ in results]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *objs, "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    args = ap.parse_args()
    print(build(verbose=args.verbose, ptxas_info=args.ptxas_info))


if __name__ == "__main__":
    main()

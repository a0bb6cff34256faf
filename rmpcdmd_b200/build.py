"""Build the CUDA library for sm_100a in-tree.

Compiles every ``csrc/*.cu`` with nvcc into ``_build/`` objects and links
``_lib/librmpcd_b200.so``.  Objects are rebuilt when a source or any header
under ``csrc/`` or ``include/`` is newer than the object.

    python -m rmpcdmd_b200.build          # incremental
    python -m rmpcdmd_b200.build --clean  # from scratch
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
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "librmpcd_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the FP64 form reproduces the reference's separately rounded
# multiply/add sequence; every kernel is memory bound, so FMA buys nothing.
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O2", "--expt-relaxed-constexpr", "-I", str(INCLUDE)]


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr}\n{r.stdout}")
    return obj, r.stderr


def build(clean: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    extra = list(extra or [])
    if clean and BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr):
            todo.append((s, o))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            futs = [ex.submit(_compile, s, o, extra) for s, o in todo]
            for f in futs:
                obj, log = f.result()
                if verbose and log.strip():
                    print(f"[{obj.name}]\n{log}", file=sys.stderr)
    if todo or not LIB.exists():
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}\n{r.stdout}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    lib = build(clean=a.clean or a.ptxas_info, verbose=a.verbose or a.ptxas_info, extra=extra)
    print(lib)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

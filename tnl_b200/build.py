"""Build libtnlb200.so (all CUDA sources under csrc/) for sm_100a, in-tree.

    python tnl_b200/build.py          # incremental
    python tnl_b200/build.py --clean  # rebuild everything

Objects go to tnl_b200/_build/, the library to tnl_b200/_lib/libtnlb200.so
(both git-ignored; the built library travels with the working tree).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libtnlb200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr", "-Xptxas", "-O3", f"-I{INCLUDE}",
] + ARCH


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{p.stdout}\n{p.stderr}")
    return obj, p.stderr


def build(clean: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    extra = extra or []
    if clean and BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hm = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if clean or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hm):
            todo.append((s, o))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj, err in ex.map(lambda so: _compile(so[0], so[1], extra), todo):
                if verbose and err.strip():
                    print(f"[{obj.name}] {err}", file=sys.stderr)
    if todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs), "-lcudart_static",
               "-lrt", "-lpthread", "-ldl"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"link failed:\n{p.stdout}\n{p.stderr}")
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    extra = []
    if "--ptxas-verbose" in args:
        extra = ["-Xptxas", "-v"]
    lib = build(clean="--clean" in args, verbose="--verbose" in args or bool(extra), extra=extra)
    print(lib)

"""Builds the CUDA library ``gpu-assembly_b200/lib/librbf_b200.so`` for sm_100a.

Every ``csrc/*.cu`` file is one translation unit; every line of
``csrc/asm_variant_list.h`` becomes one more (a generated file that defines
that kernel shape), so the heavy, fully unrolled assembly kernels compile in
parallel. Objects are rebuilt only when a source or header is newer.

Usage: ``python -m rbf_b200.build [--jobs N] [--force]`` (with
``gpu-assembly_b200`` on ``sys.path``) or ``build()`` from Python.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent.parent  # gpu-assembly_b200/
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "librbf_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", f"-I{CSRC}", f"-I{INCLUDE}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _variant_lines():
    """(macro suffix, arguments) of every shape line of asm_variant_list.h."""
    text = (CSRC / "asm_variant_list.h").read_text()
    return re.findall(r"^RBFB_(VARIANT|BLK_VARIANT|BLK16_VARIANT)\((.*)\)\s*$", text, flags=re.M)


def _sources():
    """(source path, object path) of every translation unit."""
    gen = BUILD / "gen"
    gen.mkdir(parents=True, exist_ok=True)
    units = []
    for f in sorted(CSRC.glob("*.cu")):
        units.append((f, BUILD / (f.stem + ".o")))
    for kind, args in _variant_lines():
        name = args.split(",")[0].strip()
        src = gen / f"v_{name}.cu"
        body = ('#include "asm_variant_make.cuh"\n'
                f"RBFB_DEFINE_{kind}({args})\n")
        if not src.exists() or src.read_text() != body:
            src.write_text(body)
        units.append((src, BUILD / f"v_{name}.o"))
    return units


def _stale(obj: Path, src: Path, headers_mtime: float) -> bool:
    if not obj.exists():
        return True
    m = obj.stat().st_mtime
    return src.stat().st_mtime > m or headers_mtime > m


def _compile(src: Path, obj: Path):
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return src.name


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> Path:
    """Compile (incrementally) and link the library; returns its path."""
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    hmt = max((h.stat().st_mtime for h in headers), default=0.0)
    units = _sources()
    todo = [(s, o) for s, o in units if force or _stale(o, s, hmt)]
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for name in ex.map(lambda so: _compile(*so), todo):
                if verbose:
                    print(f"  compiled {name}", flush=True)
    objs = [str(o) for _, o in units]
    if force or todo or not LIB.exists():
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + objs + ["-lcudart_static", "-lrt",
                                                                       "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.jobs, a.force, verbose=True))


if __name__ == "__main__":
    sys.exit(main())

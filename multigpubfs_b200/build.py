"""Builds libmgbfs2.so in place for sm_100a (nvcc cross-compiles; no GPU needed).

    python -m multigpubfs_b200.build [--verbose]

The shared library is written next to this file (``_lib/libmgbfs2.so``) so it
travels with the source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
OUT_DIR = PACKAGE / "_lib"
LIBRARY = OUT_DIR / "libmgbfs2.so"
INCLUDE = PACKAGE.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", str(INCLUDE)]


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmgbfs2")
    return found


def sources():
    return sorted(CSRC.glob("*.cu"))


def _digest() -> str:
    h = hashlib.sha256()
    for p in sorted(list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def up_to_date() -> bool:
    stamp = OUT_DIR / "libmgbfs2.stamp"
    return LIBRARY.exists() and stamp.exists() and stamp.read_text() == _digest()


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    if not force and not ptxas_info and up_to_date():
        return LIBRARY
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    compiler = nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(src: Path):
        obj = obj_dir / (src.stem + ".o")
        cmd = [compiler, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        results = list(pool.map(compile_one, sources()))
    if ptxas_info:
        for _, err in results:
            sys.stdout.write(err)
    objs = [str(o) for o, _ in results]
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [compiler, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    tmp.replace(LIBRARY)
    (OUT_DIR / "libmgbfs2.stamp").write_text(_digest())
    return LIBRARY


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills/shared memory per kernel")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force, ptxas_info=a.ptxas_info))


if __name__ == "__main__":
    main()

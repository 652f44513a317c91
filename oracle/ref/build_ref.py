"""Builds the reference library from its own sources, where they lie, plus
the parity harness oracle/ref/ref_dump.cpp, into oracle/_ref/ (test
infrastructure, git-ignored; the built binary travels to the GPU machine).

Every .cu/.cpp under <reference>/src/gpjson is compiled with nvcc for sm_100a
as relocatable device code (the reference builds them with CUDA separable
compilation) and linked with the harness.  Nothing of the reference is copied
into this repository.

    python oracle/ref/build_ref.py [reference_root]

The reference checkout is the argument, else $GPJSON_REFERENCE_ROOT, else
the read-only mount this recipe was written against.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def reference_root() -> Path:
    """Where the reference project's sources are read from (they are never
    copied into this repository)."""
    return Path(os.environ.get("GPJSON_REFERENCE_ROOT", "/root/reference"))


def build(ref_root: str | None = None, verbose: bool = False) -> Path | None:
    ref = Path(ref_root) if ref_root else reference_root()
    src = ref / "src" / "gpjson"
    if not src.is_dir():
        return None
    obj = OUT / "obj"
    obj.mkdir(parents=True, exist_ok=True)
    flags = ARCH + ["-rdc=true", "-std=c++17", "--expt-relaxed-constexpr", "-O3",
                    "-I", str(ref / "include"), "-I", str(ref / "src")]
    sources = sorted(list(src.rglob("*.cu")) + list(src.rglob("*.cpp")))

    def one(s: Path) -> Path:
        o = obj / (str(s.relative_to(src)).replace("/", "__") + ".o")
        if not o.exists() or o.stat().st_mtime < s.stat().st_mtime:
            cmd = [NVCC] + flags + ["-x", "cu", "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True, capture_output=not verbose)
        return o

    with cf.ThreadPoolExecutor(os.cpu_count() or 4) as pool:
        objs = list(pool.map(one, sources))
    exe = OUT / "ref_dump"
    harness = HERE / "ref_dump.cpp"
    newest = max([o.stat().st_mtime for o in objs] + [harness.stat().st_mtime])
    if not exe.exists() or exe.stat().st_mtime < newest:
        hobj = OUT / "ref_dump.o"
        for cmd in ([NVCC] + flags + ["-x", "cu", "-c", str(harness), "-o", str(hobj)],
                    [NVCC] + ARCH + ["-rdc=true", str(hobj)] + [str(o) for o in objs] +
                    ["-o", str(exe)]):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True, capture_output=not verbose)
    return exe


if __name__ == "__main__":
    print(build(*(sys.argv[1:2] or []), verbose=True))

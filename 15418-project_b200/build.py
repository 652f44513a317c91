"""Build recipe for the gpjson_b200 native library (nvcc, sm_100a).

Outputs, in-tree so that they travel with the repository snapshot:
  15418-project_b200/lib/libgpjson_b200.so   kernels + C ABI
Run as a script or through __graft_entry__.build().
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libgpjson_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
          "-I", str(ROOT / "include"), "-I", str(CSRC)]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + \
        sorted((ROOT / "include").glob("*.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    LIBDIR.mkdir(parents=True, exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.name + ".o")
        objs.append(obj)
        cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT, text=True)))
    failed = []
    for cmd, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            print(out, end="", file=sys.stderr)
        if p.returncode:
            failed.append(cmd[-3])
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB.with_suffix(".so.tmp")
    link = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs),
            "-o", str(tmp)]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


CPP = PKG / "cpp"
CPP_LIB = LIBDIR / "libgpjson_cpp.so"
DRIVER = LIBDIR / "gpjson_driver"
CXX = os.environ.get("CXX", "g++")
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-I", str(CPP / "include"), "-I",
            str(ROOT / "include"), "-I", str(CUDA_HOME / "include")]
LDCUDA = ["-L", str(CUDA_HOME / "lib64"), "-lcudart_static", "-ldl", "-lrt", "-lpthread"]


def build_cpp(force: bool = False, verbose: bool = False) -> Path:
    """The reference-shaped C++ API (libgpjson_cpp.so) over the C ABI, and
    the gpjson_driver executable."""
    build_library(force=False, verbose=verbose)
    srcs = sorted((CPP / "src").glob("*.cpp"))
    deps = srcs + sorted((CPP / "src").glob("*.hpp")) + sorted((CPP / "include").rglob("*.hpp")) + \
        [LIB]
    if force or _stale(CPP_LIB, deps):
        cmd = [CXX, *CXXFLAGS, "-shared", *map(str, srcs), "-o", str(CPP_LIB), "-L", str(LIBDIR),
               "-lgpjson_b200", "-Wl,-rpath,$ORIGIN", *LDCUDA]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    app = CPP / "apps" / "gpjson_driver.cpp"
    if force or _stale(DRIVER, [app, CPP_LIB]):
        cmd = [CXX, *CXXFLAGS, str(app), "-o", str(DRIVER), "-L", str(LIBDIR), "-lgpjson_cpp",
               "-lgpjson_b200", "-Wl,-rpath,$ORIGIN", *LDCUDA]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return CPP_LIB


def build_cpp_test(src_dir: Path, out: Path) -> Path:
    """Compiles the C++ API test program (tests/cpp) against libgpjson_cpp."""
    build_cpp()
    srcs = sorted(src_dir.glob("*.cpp"))
    if _stale(out, srcs + [CPP_LIB]):
        out.parent.mkdir(parents=True, exist_ok=True)
        subprocess.run([CXX, *CXXFLAGS, *map(str, srcs), "-o", str(out), "-L", str(LIBDIR),
                        "-lgpjson_cpp", "-lgpjson_b200", f"-Wl,-rpath,{LIBDIR}", *LDCUDA],
                       check=True)
    return out


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_cpp(force="--force" in sys.argv, verbose=True)
    print(LIB)

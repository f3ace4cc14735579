"""Builds the in-tree CUDA library libp2r_b200.so for sm_100a (and the CPU oracle).

nvcc cross-compiles for sm_100a without a GPU, so this runs on any host with the CUDA
toolkit. Objects go to p2r_tests_b200/_build/, the library to p2r_tests_b200/.
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
LIB = PKG / "libp2r_b200.so"
ROOT = PKG.parent

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", "-I" + str(ROOT / "include")]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I" + str(ROOT / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libp2r_b200.so")


def cuda_home() -> Path:
    return Path(nvcc()).resolve().parent.parent


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "p2r.h"])


def extra_defines() -> list[str]:
    """Extra -D options for the CUDA sources, from P2R_DEFINES (e.g. "P2R_FAST_MATH")."""
    return ["-D" + d for d in os.environ.get("P2R_DEFINES", "").split() if d]


def _compile(src: Path, verbose_ptxas: bool) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    if src.suffix == ".cu":
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra_defines(), "-c", str(src), "-o", str(obj)]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = [os.environ.get("CXX", "g++"), *CXX_FLAGS, "-I" + str(cuda_home() / "include"),
               "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj, res.stdout + res.stderr


def build_library(force: bool = False, verbose_ptxas: bool = False, quiet: bool = True) -> Path:
    """Compiles every csrc/ source for sm_100a and links libp2r_b200.so (incremental)."""
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    newest = max(p.stat().st_mtime for p in srcs + headers() + [Path(__file__)])
    if LIB.exists() and not force and not verbose_ptxas and LIB.stat().st_mtime >= newest:
        return LIB
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    for _, log in results:
        if log.strip() and not quiet:
            print(log, file=sys.stderr)
    objs = [str(o) for o, _ in results]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


DRIVER_SRC = PKG / "driver" / "p2r_driver.cpp"
DRIVER = PKG / "p2r_driver"


def build_driver(force: bool = False) -> Path:
    """The C++ driver program (the reference's main over the C ABI), linked to the library."""
    lib = build_library()
    if DRIVER.exists() and not force and DRIVER.stat().st_mtime >= max(DRIVER_SRC.stat().st_mtime,
                                                                        lib.stat().st_mtime):
        return DRIVER
    cuda = cuda_home()
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-Wall", "-I" + str(ROOT / "include"),
           "-I" + str(cuda / "include"), str(DRIVER_SRC), "-o", str(DRIVER), "-L" + str(PKG), "-lp2r_b200",
           "-L" + str(cuda / "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + str(cuda / "lib64")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"driver build failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return DRIVER


def build_oracle() -> None:
    """Builds oracle/_build (always) and oracle/_ref from the reference checkout named by the
    P2R_REFDIR environment variable (skipped when it is unset; an existing oracle/_ref is kept)."""
    make = shutil.which("make")
    if make is None:
        raise RuntimeError("make not found")
    subprocess.run([make, "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)
    refdir = os.environ.get("P2R_REFDIR")
    if not refdir:
        return
    if not (Path(refdir) / "src" / "propagate-tor-test_tbb.cpp").exists():
        raise RuntimeError(f"P2R_REFDIR={refdir} holds no src/propagate-tor-test_tbb.cpp")
    subprocess.run([make, "-s", "-C", str(ROOT / "oracle"), "ref", f"REFDIR={refdir}"], check=True)


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv, quiet=False)
    build_driver(force="--force" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle()
    print(LIB)

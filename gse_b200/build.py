"""In-tree build of libgse_b200.so (nvcc, sm_100a) and the C++ drop-in check
program.  `python -m gse_b200.build` rebuilds when a source is newer than its
output."""
from __future__ import annotations

import glob
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libgse_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


CB_SRC = os.path.join(CSRC, "cufft_cb", "gse_green_cb.cu")
GEN = os.path.join(PKG, "_gen")
CB_HEADER = os.path.join(GEN, "gse_green_cb_fatbin.h")


def _deps():
    return (_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(INCLUDE, "*.h")) + [os.path.abspath(__file__), CB_SRC])


def build_callbacks(verbose: bool = False) -> None:
    """The cuFFT load callbacks as LTO code, embedded in a generated header
    (an array the library passes to cufftXtSetJITCallback)."""
    os.makedirs(GEN, exist_ok=True)
    fatbin = os.path.join(GEN, "gse_green_cb.fatbin")
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=lto_100a", "-dc", "-fatbin", "-O3",
           "-std=c++17", CB_SRC, "-o", fatbin]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    out = subprocess.run([os.path.join(CUDA_HOME, "bin", "bin2c"), "--name", "gse_green_cb_fatbin",
                          "--type", "char", fatbin], check=True, capture_output=True, text=True)
    with open(CB_HEADER + ".tmp", "w") as f:
        f.write("// generated by gse_b200/build.py from csrc/cufft_cb/gse_green_cb.cu\n")
        f.write(out.stdout)
    os.replace(CB_HEADER + ".tmp", CB_HEADER)


HASH_MARK = b"gse-b200-sources:"


def source_hash() -> str:
    """First 16 hex digits of a SHA-256 over the library's sources (the .cu
    and .cuh files, the public header, the cuFFT callback source), by path
    and content; compiled into the library as its build stamp."""
    h = hashlib.sha256()
    files = sorted(_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) +
                   glob.glob(os.path.join(INCLUDE, "*.h")) + [CB_SRC])
    for f in files:
        h.update(os.path.relpath(f, ROOT).encode())
        h.update(b"\0")
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def built_hash(path: str = LIB):
    """The source hash stamped into a library file at its build (None when
    the file or the stamp is missing); read from the file, not loaded."""
    if not os.path.exists(path):
        return None
    with open(path, "rb") as fh:
        data = fh.read()
    i = data.find(HASH_MARK)
    if i < 0:
        return None
    return data[i + len(HASH_MARK):i + len(HASH_MARK) + 16].decode("ascii", "replace")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    if any(os.path.getmtime(d) > t for d in deps):
        return True
    # file times can be lost in a copy; the stamp says which sources it came from
    return target == LIB and built_hash(target) != source_hash()


def nvcc_cmd(out=LIB):
    return ([NVCC] + ARCH + NVCC_FLAGS + [f'-DGSE_SOURCE_HASH="{source_hash()}"'] +
            ["-shared", "-I", INCLUDE, "-I", CSRC, "-I", GEN] +
            _sources() +
            ["-o", out, "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft",
             "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")])


def build_lib(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale(LIB, _deps()):
        return LIB
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    build_callbacks(verbose)
    tmp = LIB + ".tmp"
    cmd = nvcc_cmd(tmp)
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


CXX_DIR = os.path.join(PKG, "cxx")
CXX_CHECK = os.path.join(CXX_DIR, "gse_dropin_check")


def build_cxx_check(force: bool = False) -> str:
    """The drop-in C++ classes compiled into a small driver (gse_dropin_check)."""
    src = os.path.join(CXX_DIR, "gse_dropin_check.cpp")
    deps = [src] + glob.glob(os.path.join(CXX_DIR, "*.h")) + [LIB]
    if not force and not _stale(CXX_CHECK, deps):
        return CXX_CHECK
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", INCLUDE, "-I", CXX_DIR, src, "-o", CXX_CHECK,
                    "-L", PKG, "-lgse_b200", "-Wl,-rpath," + PKG], check=True)
    return CXX_CHECK


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_lib(force=force, verbose=verbose)
    if os.path.exists(os.path.join(CXX_DIR, "gse_dropin_check.cpp")):
        build_cxx_check(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
    print(LIB)

"""Build libparaclaws_b200.so in-tree with nvcc for sm_100a.

Every translation unit is compiled with --fmad=false: the FP64 parity code must round where
the reference's source rounds, and the mixed-precision code writes its multiply-adds out
explicitly so its bits do not depend on the kernel it is inlined into.
Host code is compiled with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libparaclaws_b200.so"
HEADERS = [ROOT / "include" / "paraclaws_b200.h"] + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh"))

# (source, allow FMA contraction)
SOURCES = [
    ("kernels_fp64.cu", False),
    ("kernels_gen.cu", False),
    ("kernels_aux.cu", False),
    ("kernels_mixed.cu", False),
    ("batch_fp64.cu", False),
    ("batch_mixed.cu", False),
    ("capi.cu", False),
    ("capi_batch.cu", False),
    ("noalloc.cu", False),
    ("selfcheck.cu", False),
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _flags(fmad: bool, verbose: bool) -> list:
    f = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "--fmad=" + ("true" if fmad else "false"),
         "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "--expt-relaxed-constexpr",
         "-I", str(ROOT / "include"), "-I", str(CSRC)]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s, _ in SOURCES] + HEADERS + [Path(__file__), HOST_SRC]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    BUILD.mkdir(exist_ok=True)
    objs = []
    for src, fmad in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        cmd = [nvcc(), "-c", str(CSRC / src), "-o", str(obj), *_flags(fmad, verbose)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", *ARCH, "-o", str(tmp), *objs, "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, LIB)
    build_host_driver()
    return LIB


HOST_SRC = PKG / "host" / "paraclaws_main.cpp"
HOST_BIN = PKG / "bin" / "paraclaws"


def build_host_driver() -> Path:
    """The C++ host program (main.f90 above the C ABI), linked against the in-tree library."""
    HOST_BIN.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "include"), str(HOST_SRC),
           "-L", str(PKG), "-lparaclaws_b200", "-Wl,-rpath,$ORIGIN/..", "-o", str(HOST_BIN)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("host driver build failed")
    return HOST_BIN


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

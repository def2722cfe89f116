"""Build of libmgp.so (the CUDA engine + C ABI) for sm_100a, in-tree.

The engine is compiled with --fmad=false: the stencil arithmetic must not contract
multiply-adds, so that FP64 results reproduce the reference's CPU arithmetic bit for bit.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
LIB = PKG / "libmgp.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "--fmad=false", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources())


DRIVERS = ROOT / "drivers"
FACADE = ROOT / "poisson"
APPS = ("fcycle", "vcycle", "mixed", "dirichlet", "neumann", "gaussseidel")


def driver_path(app: str, problem: int) -> Path:
    return DRIVERS / "bin" / f"{app}_p{problem}"


def build_drivers(problems=(1, 2, 3), force: bool = False) -> list:
    """The reference's six example executables over the C++ facade, one per test problem
    (compile-time PROBLEMn, as the reference's Makefile selects it)."""
    build()
    out = []
    deps = [DRIVERS / "mgp_drivers.cpp", DRIVERS / "problems.cpp", LIB] + sorted(FACADE.glob("*.h"))
    newest = max(p.stat().st_mtime for p in deps)
    (DRIVERS / "bin").mkdir(exist_ok=True)
    cxx = os.environ.get("CXX", "g++")
    for prob in problems:
        for app in APPS:
            exe = driver_path(app, prob)
            if not force and exe.exists() and exe.stat().st_mtime >= newest:
                out.append(exe)
                continue
            tmp = exe.with_suffix(".tmp")
            subprocess.check_call([cxx, "-std=c++17", "-O2", f"-DMGP_APP_{app.upper()}", f"-DPROBLEM{prob}",
                                   f"-I{FACADE}", f"-I{INCLUDE}", str(DRIVERS / "mgp_drivers.cpp"),
                                   str(DRIVERS / "problems.cpp"), f"-L{PKG}", "-lmgp",
                                   "-Wl,-rpath,$ORIGIN/../../mgp", "-o", str(tmp)])
            os.replace(tmp, exe)
            out.append(exe)
    return out


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *NVCC_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}", "-o", str(tmp)] + [str(p) for p in sorted(CSRC.glob("*.cu"))]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB

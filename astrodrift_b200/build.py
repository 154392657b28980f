"""Build the native parts of astrodrift_b200 in-tree.

* ``astrodrift_b200/_lib/libdrift_b200.so`` -- the C ABI of ``include/drift_b200.h``:
  sm_100a integration kernels (one unit without multiply-add contraction, one
  with) and the host-side launch/context code, static CUDA runtime.
* ``astrodrift_b200/_drift*.so`` -- the pybind11 module with the C++ host layer
  (container graph, stage dispatch, argument validation) that calls the C ABI.

Each target is rebuilt only when its inputs or flags change.  Run as
``python -m astrodrift_b200.build`` or through ``__graft_entry__.build()``.
"""

from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = CSRC / "host"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIBDIR = PKG / "_lib"
LIB = LIBDIR / "libdrift_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + [
    "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
    "-I", str(CSRC), "-I", str(INCLUDE),
]
CUDA_UNITS = {
    # precision-exact kernels: no contraction, IEEE division/sqrt, no flush-to-zero
    "drift_kernels_exact": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "drift_kernels_fma": ["-fmad=true", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    # discrete adjoint (gradients: contraction allowed)
    "drift_adjoint": ["-fmad=true", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "drift_capi": [],
    "drift_tuning": [],
    "drift_server": [],
}


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _cxx() -> str:
    # The image's default C++ compiler; an inherited CC/CXX may point at a
    # toolchain without its runtime support files.
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("g++ not found")


def _deps(paths: list[Path]) -> str:
    h = hashlib.sha256()
    for p in sorted(paths):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()


def _stale(target: Path, key: str) -> bool:
    stamp = BUILD / (target.name + ".stamp")
    return not target.exists() or not stamp.exists() or stamp.read_text() != key


def _mark(target: Path, key: str) -> None:
    (BUILD / (target.name + ".stamp")).write_text(key)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ... ({r.returncode})")
    if verbose and r.stderr.strip():
        sys.stderr.write(r.stderr)


def build_library(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))
    objs: list[Path] = []
    jobs = []
    for unit, flags in CUDA_UNITS.items():
        src = CSRC / f"{unit}.cu"
        obj = BUILD / f"{unit}.o"
        objs.append(obj)
        key = _deps([src] + headers) + " ".join(NVCC_COMMON + flags)
        if _stale(obj, key):
            cmd = [_nvcc()] + NVCC_COMMON + flags + ["-c", str(src), "-o", str(obj)]
            jobs.append((obj, key, cmd))
    def one(job):
        obj, key, cmd = job
        _run(cmd, verbose)
        _mark(obj, key)

    with ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        for f in [ex.submit(one, j) for j in jobs]:
            f.result()
    link_key = _deps(objs) + "link-v1"
    if _stale(LIB, link_key):
        cmd = [_nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [str(o) for o in objs] + [
            "-Xlinker", "-soname=libdrift_b200.so"]
        _run(cmd, verbose)
        _mark(LIB, link_key)
    return LIB


def extension_path() -> Path:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return PKG / f"_drift{suffix}"


def build_extension(verbose: bool = False) -> Path:
    import pybind11

    BUILD.mkdir(exist_ok=True)
    target = extension_path()
    srcs = sorted(HOST.glob("*.cpp"))
    headers = sorted(HOST.glob("*.h")) + sorted(INCLUDE.glob("*.h"))
    flags = [
        "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-Wall",
        f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}",
        f"-I{INCLUDE}", f"-I{HOST}",
    ]
    key = _deps(srcs + headers + [LIB]) + " ".join(flags)
    if _stale(target, key):
        cmd = [_cxx()] + flags + [str(s) for s in srcs] + [
            f"-L{LIBDIR}", "-ldrift_b200", "-Wl,-rpath,$ORIGIN/_lib", "-o", str(target)]
        _run(cmd, verbose)
        _mark(target, key)
    return target


def build_all(verbose: bool = False) -> None:
    build_library(verbose)
    build_extension(verbose)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    print(f"built {LIB} and {extension_path()}")

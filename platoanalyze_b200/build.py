"""Build the CUDA library (sm_100a) and the C++ adapter test into the source tree.

    python -m platoanalyze_b200.build          # library only
    python -m platoanalyze_b200.build --all    # + C++ adapter test binary

Outputs: platoanalyze_b200/lib/libplato_b200.so (loaded by the ctypes binding and by C/C++
callers through include/plato_b200.h) and tests/cpp/_build/test_adapter.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libplato_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O3", "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _host_cxx() -> str:
    # plain system g++ (some images point $CXX at a wrapper without libgomp specs)
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_library(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(INCLUDE.glob("*.h"))
    jobs = []
    objs = []
    for src in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            if src.suffix == ".cu":
                cmd = [nvcc] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
            else:
                cmd = [nvcc, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}",
                       "-c", str(src), "-o", str(obj)]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd))
        list(ex.map(_run, jobs))
    if jobs or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-cudart", "static"])
    return LIB


def build_adapter_test() -> Path:
    out_dir = ROOT / "tests" / "cpp" / "_build"
    out_dir.mkdir(parents=True, exist_ok=True)
    src = ROOT / "tests" / "cpp" / "test_adapter.cpp"
    exe = out_dir / "test_adapter"
    if src.exists() and _stale(exe, [src, INCLUDE / "plato_b200.h", INCLUDE / "plato_b200.hpp", LIB]):
        _run([_nvcc(), "-O2", "-std=c++17", f"-I{INCLUDE}", str(src), "-o", str(exe),
              f"-L{LIB.parent}", "-lplato_b200", f"-Xlinker=-rpath,{LIB.parent}"])
    return exe


def build_oracle() -> Path:
    odir = ROOT / "oracle"
    _run(["make", "-s", "-C", str(odir), f"ORACLE_CXX={_host_cxx()}"])
    return odir / "_build" / "libplato_oracle.so"


if __name__ == "__main__":
    build_library(verbose="-v" in sys.argv)
    if "--all" in sys.argv:
        build_adapter_test()
        build_oracle()
    print(LIB)

"""Build libwos_b200.so and the `wos` command line for sm_100a.

    python -m walk_on_spheres_b200.build [--force] [--verbose]

Kernels are compiled with nvcc for `-gencode arch=compute_100a,code=sm_100a`
(the exact-path translation unit additionally with --fmad=false so FP64
arithmetic rounds like the reference's x86-64 build); host C++ with g++;
everything is linked with a static CUDA runtime so the library loads with no
CUDA libraries on the loader path.  Outputs stay in the package tree
(lib/, bin/) so they travel with the sources; objects go to _build/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libwos_b200.so"
CLI = PKG / "bin" / "wos"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc") if (CUDA_HOME / "bin" / "nvcc").exists() else "nvcc"
CXX = os.environ.get("CXX", "g++")

NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I", str(INCLUDE), "-I", str(CSRC)]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-pthread", "-Wall", "-Wextra", "-Wno-unused-parameter",
             "-I", str(CUDA_HOME / "include"), "-I", str(INCLUDE), "-I", str(CSRC)]

CUDA_UNITS = {
    "kernels_exact.cu": ["--fmad=false"],
    "kernels_fast.cu": [],
    "kernels_adjoint.cu": [],
    # host code that includes the device headers' type definitions
    "context.cpp": ["-x", "cu"],
    "heat_api.cpp": ["-x", "cu"],
    "batch.cpp": ["-x", "cu"],
    "transient.cpp": ["-x", "cu"],
    "stationary.cpp": ["-x", "cu"],
    "noalloc.cu": [],
    # the device tree build repeats the host build's FP64 expressions
    "scene_build_gpu.cu": ["--fmad=false"],
}
HOST_UNITS = ["scene_build.cpp", "obj_reader.cpp", "runner.cpp", "h5_writer.cpp", "host_api.cpp"]
CLI_UNITS = ["cli_main.cpp"]


def _headers() -> list[Path]:
    return list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}{r.stderr}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libwos_b200")
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    CLI.parent.mkdir(exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for src, extra in CUDA_UNITS.items():
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            cmd = [NVCC] + NVCC_FLAGS + extra + (["-Xptxas", "-v"] if ptxas_info else []) + \
                  ["-c", str(CSRC / src), "-o", str(obj)]
            jobs.append(cmd)
    for src in HOST_UNITS + CLI_UNITS:
        obj = BUILD / (src + ".o")
        if src in HOST_UNITS:
            objs.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            jobs.append([CXX] + CXX_FLAGS + ["-c", str(CSRC / src), "-o", str(obj)])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    if force or jobs or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] +
             [str(o) for o in objs] + ["-lpthread"], verbose)
    cli_obj = BUILD / "cli_main.cpp.o"
    if force or jobs or _stale(CLI, [cli_obj, LIB]):
        _run([CXX, "-o", str(CLI), str(cli_obj), str(LIB), "-Wl,-rpath,$ORIGIN/../lib",
              "-lpthread"], verbose)
    if ptxas_info:
        print("\n".join(l for l in "".join(logs).splitlines() if "ptxas" in l or "Used" in l))
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register / spill usage")
    a = ap.parse_args(argv)
    lib = build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())

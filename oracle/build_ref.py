"""TEST INFRASTRUCTURE ONLY: compile the reference's own FastEddy CUDA path into oracle/_ref.

Builds oracle/_ref/fe_ref_harness from the reference sources where they lie (the
reference tree is read-only and is never copied), the single-rank MPI shim and netCDF
stub in oracle/refshim, and oracle/ref_harness.c. The reference sources are compiled
for sm_100a with their own flags (-std=c++11, relocatable device code, device link),
replacing only -arch=sm_70. The result runs only on a GPU box; building needs no GPU.

Also builds oracle/_ref/fe_ref_io from the reference's host modules and its binary output
writer (IO/io_binary.c, compiled as part of IO/io.c) with oracle/ref_io.c: no CUDA, it runs on any machine.

usage: python oracle/build_ref.py [REFERENCE_SRC_DIR]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "refshim")
DEFAULT_SRC = "/root/reference/SRC"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

C_SOURCES = [
    "PARAMETERS/parameters.c", "PARAMETERS/hashTable.c", "FEMPI/fempi.c", "MEM_UTILS/mem_utils.c", "IO/io.c",
    "IO/ioVarsList.c", "GRID/grid.c", "GRID/CUDA/cuda_grid.c", "HYDRO_CORE/hydro_core.c",
    "HYDRO_CORE/CUDA/cuda_hydroCore.c", "TIME_INTEGRATION/time_integration.c",
    "TIME_INTEGRATION/CUDA/cuda_timeInt.c", "FECUDA/fecuda.c",
]
CU_SOURCES = [
    "GRID/CUDA/cuda_gridDevice.cu", "HYDRO_CORE/CUDA/cuda_hydroCoreDevice.cu",
    "TIME_INTEGRATION/CUDA/cuda_timeIntDevice.cu", "FECUDA/fecuda_Device.cu",
]
INC_DIRS = ["TIME_INTEGRATION", "TIME_INTEGRATION/CUDA", "HYDRO_CORE", "HYDRO_CORE/CUDA", "GRID", "GRID/CUDA", "FECUDA",
            "IO", "MEM_UTILS", "FEMPI", "PARAMETERS"]
DEFINES = ["-DCUB_IGNORE_DEPRECATED_CPP_DIALECT", "-DTHRUST_IGNORE_DEPRECATED_CPP_DIALECT"]


def _run(cmd: list[str], cwd: str | None = None) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True, cwd=cwd)
    if res.returncode != 0:
        raise RuntimeError("reference build step failed:\n" + " ".join(cmd) + "\n" + res.stdout[-4000:] + res.stderr[-4000:])


def _obj(rel: str) -> str:
    return os.path.join(OUT, "obj", rel.replace("/", "__").rsplit(".", 1)[0] + ".o")


def build(src: str = DEFAULT_SRC, verbose: bool = False) -> str:
    exe = os.path.join(OUT, "fe_ref_harness")
    if not os.path.isdir(src):
        if os.path.exists(exe):
            return exe
        raise FileNotFoundError(f"reference sources not found at {src}")
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    inc = ["-I" + SHIM] + ["-I" + os.path.join(src, d) for d in INC_DIRS] + ["-I/usr/local/cuda/include"]
    objs = []
    for rel in C_SOURCES:
        o = _obj(rel)
        if not os.path.exists(o):
            cmd = ["gcc", "-O2", "-m64", "-w", *DEFINES, *inc, "-c", os.path.join(src, rel), "-o", o]
            if verbose:
                print(os.path.basename(rel), flush=True)
            _run(cmd)
        objs.append(o)
    cu_objs = []
    for rel in CU_SOURCES:
        o = _obj(rel)
        if not os.path.exists(o):
            cmd = [NVCC, *ARCH, "-m64", "-std=c++11", "-O3", "-w", *DEFINES, *inc, "-dc",
                   os.path.join(src, rel), "-o", o]
            if verbose:
                print(os.path.basename(rel), flush=True)
            _run(cmd)
        cu_objs.append(o)
    for name in ("mpi_stub.c", "netcdf_stub.c"):
        o = os.path.join(OUT, "obj", name[:-2] + ".o")
        _run(["gcc", "-O2", "-I" + SHIM, "-c", os.path.join(SHIM, name), "-o", o])
        objs.append(o)
    ho = os.path.join(OUT, "obj", "ref_harness.o")
    _run(["gcc", "-O2", "-m64", *inc, "-c", os.path.join(HERE, "ref_harness.c"), "-o", ho])
    objs.append(ho)
    dl = os.path.join(OUT, "obj", "devlink.o")
    _run([NVCC, *ARCH, "-dlink", *cu_objs, "-o", dl])
    _run([NVCC, *ARCH, "-o", exe, *objs, *cu_objs, "-lm", "-lstdc++"])
    build_io(src, inc)
    return exe


# host modules the binary-output checker needs (no CUDA wrappers, no FECUDA)
IO_SOURCES = [
    "PARAMETERS/parameters.c", "PARAMETERS/hashTable.c", "FEMPI/fempi.c", "MEM_UTILS/mem_utils.c", "IO/io.c",
    "IO/ioVarsList.c", "GRID/grid.c", "HYDRO_CORE/hydro_core.c", "TIME_INTEGRATION/time_integration.c",
]  # IO/io.c includes io_binary.c (io.c:202)


def build_io(src: str, inc: list[str]) -> str:
    exe = os.path.join(OUT, "fe_ref_io")
    objs = []
    for rel in IO_SOURCES:
        o = _obj(rel)
        if not os.path.exists(o):
            _run(["gcc", "-O2", "-m64", "-w", *DEFINES, *inc, "-c", os.path.join(src, rel), "-o", o])
        objs.append(o)
    for name in ("mpi_stub.c", "netcdf_stub.c"):
        objs.append(os.path.join(OUT, "obj", name[:-2] + ".o"))
    io = os.path.join(OUT, "obj", "ref_io.o")
    _run(["gcc", "-O2", "-m64", *inc, "-c", os.path.join(HERE, "ref_io.c"), "-o", io])
    _run(["gcc", "-o", exe, *objs, io, "-lm"])
    return exe


# The reference's CUDA layer: the four device translation units and the thin C wrappers over them.
# The drop-in build leaves exactly these out and links the repository's libraries in their place.
CUDA_WRAPPERS = ["FECUDA/fecuda.c", "GRID/CUDA/cuda_grid.c", "HYDRO_CORE/CUDA/cuda_hydroCore.c",
                 "TIME_INTEGRATION/CUDA/cuda_timeInt.c"]
ENGINE_LIBS = os.path.join(os.path.dirname(HERE), "fasteddy-model_b200", "_build")


def build_dropin(src: str = DEFAULT_SRC) -> str:
    """oracle/_ref/fe_dropin_harness: the same driver sequence (ref_harness.c) and the same
    reference host modules as fe_ref_harness, with the reference's CUDA layer replaced by
    libfe_refabi.so + libfe_engine.so, linked as a FastEddy user would (-rdynamic exports the
    driver's globals to the library). Needs fe_ref_harness's objects (build() first) and the
    repository's libraries."""
    exe = os.path.join(OUT, "fe_dropin_harness")
    objs = [_obj(rel) for rel in C_SOURCES if rel not in CUDA_WRAPPERS]
    objs += [os.path.join(OUT, "obj", n) for n in ("mpi_stub.o", "netcdf_stub.o", "ref_harness.o")]
    missing = [o for o in objs if not os.path.exists(o)]
    if missing:
        if not os.path.isdir(src):
            raise FileNotFoundError("reference objects not built: " + ", ".join(missing))
        build(src)
    rpath = "$ORIGIN/" + os.path.relpath(ENGINE_LIBS, OUT)
    _run(["gcc", "-o", exe, *objs, "-rdynamic", "-L" + ENGINE_LIBS, "-lfe_refabi", "-lfe_engine",
          "-Wl,-rpath," + rpath, "-lm"])
    return exe


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC, verbose=True))
    print(build_dropin(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC))

"""Build the native libraries of the package in-tree (they travel with the source tree).

    _build/libfe_engine.so   CUDA engine for sm_100a (nvcc), C ABI of include/fasteddy_b200.h
    _build/libfe_refabi.so   reference-named drop-in entry points (reads the FastEddy globals)
    _build/libfe_host.so     host C layer: parameter file, grid, base state, initial state

Run as a module or call build(); rebuilds only what is older than its sources.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build")
INC = os.path.join(ROOT, "include")
ENGINE_DIR = os.path.join(HERE, "csrc", "engine")
HOST_DIR = os.path.join(HERE, "csrc", "host")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)


def _sources(d: str, exts: tuple[str, ...]) -> list[str]:
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def build(verbose: bool = False) -> dict[str, str]:
    os.makedirs(OUT, exist_ok=True)
    libs = {
        "engine": os.path.join(OUT, "libfe_engine.so"),
        "refabi": os.path.join(OUT, "libfe_refabi.so"),
        "host": os.path.join(OUT, "libfe_host.so"),
    }
    hdr = [os.path.join(INC, "fasteddy_b200.h")]
    eng_src = _sources(ENGINE_DIR, (".cu",))
    eng_deps = eng_src + _sources(ENGINE_DIR, (".cuh", ".h")) + hdr
    if _stale(libs["engine"], eng_deps):
        # one object per translation unit, compiled concurrently (the stage kernel's instantiations
        # are split by RK stage over fe_march_s*.cu), then one shared library
        objdir = os.path.join(OUT, "obj")
        os.makedirs(objdir, exist_ok=True)
        procs, objs = [], []
        for src in eng_src:
            obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
            objs.append(obj)
            cmd = [_nvcc(), *NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INC,
                   "-I" + ENGINE_DIR, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        errors = []
        for cmd, pr in procs:
            out, _ = pr.communicate()
            if pr.returncode != 0:
                errors.append(" ".join(cmd) + "\n" + out)
        if errors:
            raise RuntimeError("build step failed:\n" + "\n".join(errors))
        cmd = [_nvcc(), *NVCC_ARCH, "-shared", "-o", libs["engine"], *objs, "-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        _run(cmd)
    host_src = [os.path.join(HOST_DIR, f) for f in ("fe_params.c", "fe_host.c")]
    host_deps = host_src + _sources(HOST_DIR, (".h",))
    if _stale(libs["host"], host_deps):
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-I" + INC, "-I" + HOST_DIR, "-o", libs["host"],
               *host_src, "-lm"]
        if verbose:
            print(" ".join(cmd), flush=True)
        _run(cmd)
    abi_src = [os.path.join(HOST_DIR, "fe_refabi.c")]
    if _stale(libs["refabi"], abi_src + host_deps + hdr + [libs["engine"]]):
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-I" + INC, "-I" + HOST_DIR, "-o", libs["refabi"],
               *abi_src, "-L" + OUT, "-lfe_engine", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        _run(cmd)
    return libs


if __name__ == "__main__":
    out = build(verbose="-v" in sys.argv)
    for k, v in out.items():
        print(k, v)

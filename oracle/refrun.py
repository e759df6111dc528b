"""TEST INFRASTRUCTURE ONLY: run the reference's own CUDA build (oracle/_ref/fe_ref_harness)
on inputs produced by the host layer, for parity checks and the reference timing arm.

Inputs and outputs are exchanged as raw float32 files in the reference layout.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "fe_ref_harness")
# the same driver and host modules with the repository's libraries as the CUDA layer
DROPIN = os.path.join(HERE, "_ref", "fe_dropin_harness")


def available(exe: str = HARNESS) -> bool:
    return os.path.exists(exe) and os.access(exe, os.X_OK)


def _write_inputs(d: str, inp: dict) -> None:
    for k, v in inp.items():
        if v is None:
            continue
        np.ascontiguousarray(v, dtype=np.float32).tofile(os.path.join(d, k + ".bin"))


def _run(param_text: str, inp: dict | None, mode: str, n: int, timeout: float, qv: str | None = None,
         files: dict | None = None, exe: str = HARNESS) -> tuple[str, str]:
    """Run the harness in a fresh directory. inp = None keeps the reference's own initial state
    (its grid, base state and theta perturbations); qv = "qv:SFC,TOP,ZTOP" then sets its q_v
    profile. files = {name: bytes} are written into the directory first (e.g. a topoFile named
    by the parameter text as ./name)."""
    if not available(exe):
        raise FileNotFoundError(f"{os.path.basename(exe)} not built (python oracle/build_ref.py)")
    work = tempfile.mkdtemp(prefix="feref_")
    ind, outd = os.path.join(work, "in"), os.path.join(work, "out")
    os.makedirs(ind)
    os.makedirs(outd)
    os.makedirs(os.path.join(work, "output"), exist_ok=True)
    pf = os.path.join(work, "params.in")
    with open(pf, "w") as f:
        f.write(param_text)
    for name, blob in (files or {}).items():
        with open(os.path.join(work, name), "wb") as f:
            f.write(blob)
    if inp is not None:
        _write_inputs(ind, inp)
    cmd = [exe, pf, ind if inp is not None else "-", outd, mode, str(n)] + ([qv] if qv else [])
    res = subprocess.run(cmd, capture_output=True, text=True, cwd=work, timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"reference harness failed ({res.returncode}):\n{res.stdout[-3000:]}\n{res.stderr[-3000:]}")
    return outd, res.stdout


def run(param_text: str, inp: dict, nsteps: int, shape: tuple[int, int, int], ntke: int, nmoist: int,
        timeout: float = 900.0, exe: str = HARNESS) -> dict:
    """Advance `nsteps` RK3 steps with the reference build (or, exe = DROPIN, with the reference's
    driver and host modules over this repository's libraries); returns the state (float32)."""
    outd, _ = _run(param_text, inp, "run", nsteps, timeout, exe=exe)
    nx, ny, nz = shape
    rd = lambda name, nf: np.fromfile(os.path.join(outd, name + ".bin"), dtype=np.float32).reshape(nf, nx, ny, nz)
    out = {"hydroFlds": rd("hydroFlds", 5), "pres": rd("pres", 1)[0]}
    out["sgstke"] = rd("sgstke", 1) if ntke else None
    out["moist"] = rd("moist", nmoist) if nmoist else None
    for name in ("fricVel", "htFlux", "invOblen", "tskin"):
        p = os.path.join(outd, name + ".bin")
        if os.path.exists(p):
            out[name] = np.fromfile(p, dtype=np.float32).reshape(nx, ny)
    _read_forcing(outd, shape, ntke, nmoist, out)
    return out


def _read_forcing(outd: str, shape: tuple[int, int, int], ntke: int, nmoist: int, out: dict) -> None:
    nx, ny, nz = shape
    for name, nf in (("hydroFrhs", 5), ("sgstkeFrhs", ntke), ("moistFrhs", nmoist), ("taus", 9),
                     ("moistTaus", 3 * nmoist)):
        p = os.path.join(outd, name + ".bin")
        if nf and os.path.exists(p):
            out[name] = np.fromfile(p, dtype=np.float32).reshape(nf, nx, ny, nz)


def frhs(param_text: str, inp: dict, stage: int, shape: tuple[int, int, int], ntke: int, nmoist: int,
         timeout: float = 900.0, exe: str = HARNESS) -> dict:
    """One tendency evaluation of RK stage `stage` on `inp` by the reference build
    (cuda_hydroCoreDeviceBuildFrhs): hydroFrhs, sgstkeFrhs, moistFrhs, taus, moistTaus, pres.
    The parameter text must set hydroForcingWrite = 1 and hydroSubGridWrite = 1."""
    outd, _ = _run(param_text, inp, "frhs", stage, timeout, exe=exe)
    nx, ny, nz = shape
    out = {"pres": np.fromfile(os.path.join(outd, "pres.bin"), dtype=np.float32).reshape(nx, ny, nz)}
    _read_forcing(outd, shape, ntke, nmoist, out)
    return out


def time_steps(param_text: str, inp: dict | None, k: int, timeout: float = 1800.0, qv: str | None = None,
               files: dict | None = None) -> dict:
    """Wall time per RK3 step of the reference build (difference of K- and 2K-step batches).
    inp = None: the reference's own initial state (see _run)."""
    _, stdout = _run(param_text, inp, "time", k, timeout, qv, files)
    for line in stdout.splitlines()[::-1]:
        line = line.strip()
        if line.startswith("{") and "ms_per_step" in line:
            return json.loads(line)
    raise RuntimeError("no timing line from the reference harness:\n" + stdout[-2000:])

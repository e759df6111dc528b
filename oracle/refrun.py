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


def available() -> bool:
    return os.path.exists(HARNESS) and os.access(HARNESS, os.X_OK)


def _write_inputs(d: str, inp: dict) -> None:
    for k, v in inp.items():
        if v is None:
            continue
        np.ascontiguousarray(v, dtype=np.float32).tofile(os.path.join(d, k + ".bin"))


def _run(param_text: str, inp: dict, mode: str, n: int, timeout: float) -> tuple[str, str]:
    if not available():
        raise FileNotFoundError("reference harness not built (python oracle/build_ref.py)")
    work = tempfile.mkdtemp(prefix="feref_")
    ind, outd = os.path.join(work, "in"), os.path.join(work, "out")
    os.makedirs(ind)
    os.makedirs(outd)
    os.makedirs(os.path.join(work, "output"), exist_ok=True)
    pf = os.path.join(work, "params.in")
    with open(pf, "w") as f:
        f.write(param_text)
    _write_inputs(ind, inp)
    res = subprocess.run([HARNESS, pf, ind, outd, mode, str(n)], capture_output=True, text=True, cwd=work,
                         timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"reference harness failed ({res.returncode}):\n{res.stdout[-3000:]}\n{res.stderr[-3000:]}")
    return outd, res.stdout


def run(param_text: str, inp: dict, nsteps: int, shape: tuple[int, int, int], ntke: int, nmoist: int,
        timeout: float = 900.0) -> dict:
    """Advance `nsteps` RK3 steps with the reference build; returns its state (float32)."""
    outd, _ = _run(param_text, inp, "run", nsteps, timeout)
    nx, ny, nz = shape
    rd = lambda name, nf: np.fromfile(os.path.join(outd, name + ".bin"), dtype=np.float32).reshape(nf, nx, ny, nz)
    out = {"hydroFlds": rd("hydroFlds", 5), "pres": rd("pres", 1)[0]}
    out["sgstke"] = rd("sgstke", 1) if ntke else None
    out["moist"] = rd("moist", nmoist) if nmoist else None
    for name in ("fricVel", "htFlux", "invOblen", "tskin"):
        p = os.path.join(outd, name + ".bin")
        if os.path.exists(p):
            out[name] = np.fromfile(p, dtype=np.float32).reshape(nx, ny)
    return out


def time_steps(param_text: str, inp: dict, k: int, timeout: float = 1800.0) -> dict:
    """Wall time per RK3 step of the reference build (difference of K- and 2K-step batches)."""
    _, stdout = _run(param_text, inp, "time", k, timeout)
    for line in stdout.splitlines()[::-1]:
        line = line.strip()
        if line.startswith("{") and "ms_per_step" in line:
            return json.loads(line)
    raise RuntimeError("no timing line from the reference harness:\n" + stdout[-2000:])

"""TEST INFRASTRUCTURE ONLY: Python binding of the FP64 CPU oracle (oracle/fe_oracle.c).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg only, as the
checker of the CUDA path. Builds oracle/_build/libfe_oracle.so with gcc on first use.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libfe_oracle.so")
_lib = None

c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)


def build(openmp: bool = False) -> str:
    """Compile the oracle (plain C, libm only); returns the library path."""
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(HERE, "fe_oracle.c"), os.path.join(HERE, "fe_oracle.h"),
            os.path.join(ROOT, "include", "fasteddy_b200.h")]
    if os.path.exists(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs):
        return LIB
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"), "-I" + HERE,
           "-o", LIB, os.path.join(HERE, "fe_oracle.c"), "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)
    return LIB


def _load():
    global _lib
    if _lib is not None:
        return _lib
    lib = ctypes.CDLL(build())
    vp = ctypes.c_void_p
    ip = ctypes.c_int
    fp = c_float_p
    dp = c_double_p
    sig = {
        "ora_create": (ip, [vp, ctypes.POINTER(vp)]),
        "ora_destroy": (None, [vp]),
        "ora_set_grid": (ip, [vp, fp, fp, fp, fp, fp, fp]),
        "ora_set_base_state": (ip, [vp, fp]),
        "ora_set_state": (ip, [vp, fp, fp, fp]),
        "ora_set_state_f64": (ip, [vp, dp, dp, dp]),
        "ora_set_surface": (ip, [vp, fp, fp, fp, fp, fp, fp, fp]),
        "ora_set_clock": (ip, [vp, ctypes.c_double, ip]),
        "ora_set_decomposition": (ip, [vp, ip, ip]),
        "ora_build_frhs": (ip, [vp, ip]),
        "ora_rk_stage": (ip, [vp, ip]),
        "ora_step": (ip, [vp, ip]),
        "ora_get_state": (ip, [vp, dp, dp, dp, dp]),
        "ora_get_frhs": (ip, [vp, dp, dp, dp, dp]),
        "ora_get_surface": (ip, [vp, dp, dp, dp, dp, dp, dp, dp, dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _f(a):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.ctypes.data_as(c_float_p), a


class Oracle:
    """FP64 serial restatement of one FastEddy domain (reference layout, halo-inclusive)."""

    def __init__(self, cfg) -> None:
        self.lib = _load()
        self.h = ctypes.c_void_p()
        rc = self.lib.ora_create(ctypes.cast(ctypes.pointer(cfg), ctypes.c_void_p), ctypes.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"ora_create failed ({rc})")
        self.shape = (cfg.Nx + 6, cfg.Ny + 6, cfg.Nz + 6)
        self.ntke = 1 if (cfg.turbulenceSelector > 0 and cfg.TKESelector > 0) else 0
        self.nmoist = cfg.moistureNvars if cfg.moistureSelector > 0 else 0
        self._keep = []

    def close(self) -> None:
        if self.h:
            self.lib.ora_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def _p(self, a):
        if a is None:
            return None
        p, arr = _f(a)
        self._keep.append(arr)
        return p

    def set_inputs(self, inp: dict, simTime: float = 0.0, simTime_it: int = 0) -> None:
        L = self.lib
        L.ora_set_grid(self.h, *(self._p(inp[k]) for k in ("zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac")))
        L.ora_set_base_state(self.h, self._p(inp["baseState"]))
        L.ora_set_surface(self.h, *(self._p(inp.get(k)) for k in ("z0m", "z0t", "htFlux", "tskin", "fricVel",
                                                                    "qFlux", "qskin")))
        L.ora_set_state(self.h, self._p(inp["hydroFlds"]), self._p(inp.get("sgstke")), self._p(inp.get("moist")))
        L.ora_set_clock(self.h, simTime, simTime_it)
        self._keep.clear()

    def set_decomposition(self, peer_x: bool, peer_y: bool) -> None:
        """Keep the caller-written x / y halo columns (a slab of a decomposed domain)."""
        self.lib.ora_set_decomposition(self.h, int(peer_x), int(peer_y))

    def set_state_f64(self, hydro, sgstke=None, moist=None) -> None:
        d = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        H, E, M = d(hydro), d(sgstke) if self.ntke else None, d(moist) if self.nmoist else None
        p = lambda a: None if a is None else a.ctypes.data_as(c_double_p)
        self.lib.ora_set_state_f64(self.h, p(H), p(E), p(M))

    def set_clock(self, simTime: float, simTime_it: int) -> None:
        self.lib.ora_set_clock(self.h, simTime, simTime_it)

    def step(self, n: int = 1) -> None:
        self.lib.ora_step(self.h, n)

    def rk_stage(self, stage: int) -> None:
        self.lib.ora_rk_stage(self.h, stage)

    def build_frhs(self, stage: int) -> dict:
        self.lib.ora_build_frhs(self.h, stage)
        return self.last_frhs()

    def last_frhs(self) -> dict:
        """The tendencies and SGS stresses of the last evaluation (after step(): those of the last
        RK stage of the last step, what the reference copies back after a batch)."""
        nx, ny, nz = self.shape
        F = np.empty((5, nx, ny, nz))
        Fe = np.empty((1, nx, ny, nz)) if self.ntke else None
        Fm = np.empty((self.nmoist, nx, ny, nz)) if self.nmoist else None
        T = np.empty((9, nx, ny, nz))
        d = lambda a: None if a is None else a.ctypes.data_as(c_double_p)
        self.lib.ora_get_frhs(self.h, d(F), d(Fe), d(Fm), d(T))
        return {"hydroFrhs": F, "sgstkeFrhs": Fe, "moistFrhs": Fm, "taus": T}

    def get_state(self) -> dict:
        nx, ny, nz = self.shape
        H = np.empty((5, nx, ny, nz))
        E = np.empty((1, nx, ny, nz)) if self.ntke else None
        M = np.empty((self.nmoist, nx, ny, nz)) if self.nmoist else None
        P = np.empty((nx, ny, nz))
        d = lambda a: None if a is None else a.ctypes.data_as(c_double_p)
        self.lib.ora_get_state(self.h, d(H), d(E), d(M), d(P))
        return {"hydroFlds": H, "sgstke": E, "moist": M, "pres": P}

    def get_surface(self) -> dict:
        nx, ny, _ = self.shape
        names = ("cd", "ch", "fricVel", "htFlux", "invOblen", "tskin", "qFlux", "qskin")
        out = {k: np.empty((nx, ny)) for k in names}
        self.lib.ora_get_surface(self.h, *(out[k].ctypes.data_as(c_double_p) for k in names))
        return out

"""ctypes bindings of the native libraries (host layer, drop-in ABI, engine).

The product path is native: the engine kernels run on the GPU through libfe_engine.so.
Nothing here computes physics; a missing library or a missing GPU raises instead of
falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import build as _build

_LIBS: dict[str, ctypes.CDLL] = {}

SGS_NIN = 11      # FE_SGS_NIN
SGS_NOUT = 9      # FE_SGS_NOUT
KERNEL_CELL = 0   # FE_KERNEL_CELL
KERNEL_MARCH = 1  # FE_KERNEL_MARCH

c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)


class FeConfig(ctypes.Structure):
    """Mirror of `fe_config` in include/fasteddy_b200.h (same field order and types)."""

    _fields_ = [
        ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int), ("Nh", ctypes.c_int),
        ("dX", ctypes.c_float), ("dY", ctypes.c_float), ("dZ", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("simTime_itRestart", ctypes.c_int),
        ("hydroBCs", ctypes.c_int),
        ("pgfSelector", ctypes.c_int), ("buoyancySelector", ctypes.c_int), ("coriolisSelector", ctypes.c_int),
        ("turbulenceSelector", ctypes.c_int), ("TKESelector", ctypes.c_int), ("TKEAdvSelector", ctypes.c_int),
        ("TKEAdvSelector_b_hyb", ctypes.c_float), ("c_s", ctypes.c_float), ("c_k", ctypes.c_float),
        ("advectionSelector", ctypes.c_int),
        ("b_hyb", ctypes.c_float),
        ("diffusionSelector", ctypes.c_int), ("filterSelector", ctypes.c_int), ("lsfSelector", ctypes.c_int),
        ("surflayerSelector", ctypes.c_int),
        ("surflayer_z0", ctypes.c_float), ("surflayer_z0t", ctypes.c_float), ("surflayer_wth", ctypes.c_float),
        ("surflayer_tr", ctypes.c_float), ("surflayer_wq", ctypes.c_float), ("surflayer_qr", ctypes.c_float),
        ("surflayer_qskin_input", ctypes.c_int), ("surflayer_stab", ctypes.c_int), ("surflayer_idealsine", ctypes.c_int),
        ("surflayer_ideal_ts", ctypes.c_float), ("surflayer_ideal_te", ctypes.c_float),
        ("surflayer_ideal_amp", ctypes.c_float),
        ("surflayer_ideal_qts", ctypes.c_float), ("surflayer_ideal_qte", ctypes.c_float),
        ("surflayer_ideal_qamp", ctypes.c_float),
        ("moistureSelector", ctypes.c_int), ("moistureNvars", ctypes.c_int), ("moistureAdvSelectorQv", ctypes.c_int),
        ("moistureAdvSelectorQv_b", ctypes.c_float),
        ("moistureAdvSelectorQi", ctypes.c_int), ("moistureSGSturb", ctypes.c_int), ("moistureCond", ctypes.c_int),
        ("moistureCondTscale", ctypes.c_float),
        ("moistureCondBasePres", ctypes.c_int),
        ("moistureMPcallTscale", ctypes.c_float),
        ("dampingLayerSelector", ctypes.c_int),
        ("dampingLayerDepth", ctypes.c_float),
        ("U_g", ctypes.c_float), ("V_g", ctypes.c_float), ("z_Ug", ctypes.c_float), ("z_Vg", ctypes.c_float),
        ("Ug_grad", ctypes.c_float), ("Vg_grad", ctypes.c_float),
        ("corioConstHorz", ctypes.c_float), ("corioConstVert", ctypes.c_float), ("corioLS_fact", ctypes.c_float),
        ("physics_oneRKonly", ctypes.c_int),
        ("temp_grnd", ctypes.c_float), ("pres_grnd", ctypes.c_float),
        ("R_gas", ctypes.c_float), ("R_vapor", ctypes.c_float), ("Rv_Rg", ctypes.c_float), ("cp_gas", ctypes.c_float),
        ("cv_gas", ctypes.c_float), ("accel_g", ctypes.c_float), ("R_cp", ctypes.c_float), ("cp_R", ctypes.c_float),
        ("cp_cv", ctypes.c_float), ("refPressure", ctypes.c_float), ("kappa", ctypes.c_float), ("L_v", ctypes.c_float),
        ("filter_6th_coeff", ctypes.c_float),
        ("lsf_horMnSubTerms", ctypes.c_int), ("lsf_freq", ctypes.c_float),
        *[(f"lsf_{v}_{p}", ctypes.c_float) for v in ("w", "th", "qv") for p in ("surf", "lev1", "lev2", "zlev1", "zlev2")],
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class FeNoallocArgs(ctypes.Structure):
    """Mirror of `fe_noalloc_args` (device pointers)."""

    _fields_ = [(n, ctypes.c_void_p) for n in ("zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac", "baseState", "state",
                                                "surface", "frhs")]


class FeError(RuntimeError):
    pass


def _declare(lib: ctypes.CDLL, name: str, restype, argtypes) -> None:
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes


def load(rebuild: bool = True) -> dict[str, ctypes.CDLL]:
    """Load (building first if needed) libfe_host, libfe_engine and libfe_refabi."""
    if _LIBS:
        return _LIBS
    paths = _build.build() if rebuild else {
        k: os.path.join(_build.OUT, f"libfe_{k}.so") for k in ("engine", "refabi", "host")}
    host = ctypes.CDLL(paths["host"], mode=ctypes.RTLD_GLOBAL)
    engine = ctypes.CDLL(paths["engine"], mode=ctypes.RTLD_GLOBAL)
    refabi = ctypes.CDLL(paths["refabi"], mode=ctypes.RTLD_GLOBAL)
    vp = ctypes.c_void_p
    ip = ctypes.c_int
    fp = c_float_p
    for name, res, args in [
        ("fe_host_load_params_file", ip, [ctypes.c_char_p]),
        ("fe_host_load_params_text", ip, [ctypes.c_char_p]),
        ("fe_host_unused_params", ip, [ctypes.c_char_p, ip]),
        ("fe_host_set_topography", ip, [fp, ip, ip]),
        ("fe_host_gaussian_hill", ip, [ctypes.c_float, ctypes.c_float]),
        ("fe_host_write_topofile", ip, [ctypes.c_char_p]),
        ("fe_host_init", ip, [ctypes.c_ulonglong]),
        ("fe_host_set_qv_profile", ip, [ctypes.c_float, ctypes.c_float, ctypes.c_float]),
        ("fe_host_cleanup", None, []),
        ("fe_host_field_elems", ctypes.c_size_t, []),
        ("fe_host_plane_elems", ctypes.c_size_t, []),
        ("fe_host_last_message", ctypes.c_char_p, []),
        ("fe_host_write_binary", ip, [ctypes.c_char_p, ip]),
        ("fe_host_write_netcdf", ip, [ctypes.c_char_p, ip]),
    ]:
        _declare(host, name, res, args)
    for name, res, args in [
        ("fe_config_defaults", None, [ctypes.POINTER(FeConfig)]),
        ("fe_config_derive", None, [ctypes.POINTER(FeConfig), ctypes.c_float]),
        ("fe_device_count", ip, []),
        ("fe_create", ip, [ctypes.POINTER(FeConfig), ip, ctypes.POINTER(vp)]),
        ("fe_destroy", ip, [vp]),
        ("fe_device_bytes", ctypes.c_size_t, [vp]),
        ("fe_set_grid", ip, [vp, fp, fp, fp, fp, fp, fp]),
        ("fe_set_base_state", ip, [vp, fp]),
        ("fe_set_state", ip, [vp, fp, fp, fp]),
        ("fe_set_surface", ip, [vp, fp, fp, fp, fp, fp, fp, fp]),
        ("fe_set_clock", ip, [vp, ctypes.c_float, ip]),
        ("fe_get_clock", ip, [vp, fp, ctypes.POINTER(ip)]),
        ("fe_advance", ip, [vp, ip]),
        ("fe_sync", ip, [vp]),
        ("fe_stream", vp, [vp]),
        ("fe_get_state", ip, [vp, fp, fp, fp, fp]),
        ("fe_get_surface", ip, [vp, fp, fp, fp, fp, fp, fp, fp, fp]),
        ("fe_build_frhs", ip, [vp, ip]),
        ("fe_get_frhs", ip, [vp, fp, fp, fp, fp]),
        ("fe_set_forcing_capture", ip, [vp, ip]),
        ("fe_get_sgs_fluxes", ip, [vp, fp, fp]),
        ("fe_check_config", ip, [ctypes.POINTER(FeConfig)]),
        ("fe_count_nonfinite", ip, [vp, ctypes.POINTER(ctypes.c_longlong)]),
        ("fe_domain_means", ip, [vp, c_double_p]),
        ("fe_set_tiling", ip, [vp, ip, ip, ip]),
        ("fe_set_stage_kernel", ip, [vp, ip, ip, ip]),
        ("fe_set_sgs_kernel", ip, [vp, ip]),
        ("fe_set_sgs_shape", ip, [vp, ip, ip]),
        ("fe_get_sgs_shape", ip, [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]),
        ("fe_get_stage_kernel", ip, [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]),
        ("fe_autotune", ip, [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]),
        ("fe_launch_count", ctypes.c_longlong, [vp]),
        ("fe_time_stage_kernel", ip, [vp, ip, fp]),
        ("fe_host_register", ip, [vp, ctypes.c_size_t]),
        ("fe_host_unregister", ip, [vp]),
        ("fe_ensemble_create", ip, [ctypes.POINTER(vp), ip, ctypes.POINTER(vp)]),
        ("fe_ensemble_advance", ip, [vp, ip]),
        ("fe_ensemble_sync", ip, [vp]),
        ("fe_ensemble_stream", vp, [vp]),
        ("fe_ensemble_destroy", ip, [vp]),
        ("fe_ensemble_set_batched", ip, [vp, ip]),
        ("fe_ensemble_is_batched", ip, [vp]),
        ("fe_ensemble_launch_count", ctypes.c_longlong, [vp]),
        ("fe_slab_group_create", ip, [ctypes.POINTER(vp), ip, ip, ctypes.POINTER(vp)]),
        ("fe_ipc_handle_bytes", ctypes.c_size_t, []),
        ("fe_arena_ipc_handle", ip, [vp, vp, ctypes.c_size_t]),
        ("fe_set_halo_peers", ip, [vp, ip, ip, ctypes.POINTER(vp)]),
        ("fe_clear_halo_peers", ip, [vp]),
        ("fe_comm_unique_id_bytes", ctypes.c_size_t, []),
        ("fe_comm_unique_id", ip, [vp, ctypes.c_size_t]),
        ("fe_comm_create", ip, [vp, ip, ip, ip, ctypes.POINTER(vp)]),
        ("fe_comm_destroy", ip, [vp]),
        ("fe_set_halo_comm", ip, [vp, vp]),
        ("fe_last_error", ctypes.c_char_p, []),
        ("fe_noalloc_max_cells", ctypes.c_longlong, []),
        ("fe_checkpoint_bytes", ctypes.c_size_t, [vp]),
        ("fe_checkpoint_save", ip, [vp, vp, ctypes.c_size_t]),
        ("fe_checkpoint_load", ip, [vp, vp, ctypes.c_size_t]),
        ("fe_mlp_param_count", ctypes.c_longlong, []),
        ("fe_mlp_create", ip, [ip, ctypes.c_ulonglong, ctypes.POINTER(vp)]),
        ("fe_mlp_destroy", ip, [vp]),
        ("fe_mlp_set_params", ip, [vp, fp]),
        ("fe_mlp_get_params", ip, [vp, fp]),
        ("fe_mlp_set_norm", ip, [vp, fp, fp, fp, fp]),
        ("fe_mlp_get_norm", ip, [vp, fp, fp, fp, fp]),
        ("fe_mlp_set_data", ip, [vp, fp, fp, ctypes.c_longlong, ctypes.c_ulonglong, ip]),
        ("fe_mlp_gradient", ip, [vp, ctypes.c_longlong, ctypes.c_longlong, fp, c_double_p]),
        ("fe_mlp_train", ip, [vp, ip, ctypes.c_longlong, ctypes.c_float, c_double_p]),
        ("fe_mlp_predict", ip, [vp, fp, ctypes.c_longlong, fp]),
        ("fe_mlp_time", ip, [vp, ip, ctypes.c_longlong, ip, fp]),
        ("fe_mlp_check", ip, [vp]),
        ("fe_set_sgs_mlp", ip, [vp, vp]),
        ("fe_sgs_sample", ip, [vp, ctypes.c_longlong, fp, fp, fp]),
        ("fe_coarsen", ip, [vp, vp, fp]),
        ("fe_frhs_noalloc", ip, [ctypes.POINTER(FeConfig), ip, ctypes.c_float, ip, ctypes.POINTER(FeNoallocArgs), vp]),
        ("fe_noalloc_last_error", ctypes.c_char_p, []),
    ]:
        _declare(engine, name, res, args)
    for name in ("fecuda_Init", "fecuda_DeallocateHaloBuffers", "fecuda_Cleanup", "cuda_gridInit", "cuda_gridCleanup",
                 "cuda_hydroCoreInit", "cuda_hydroCoreCleanup", "cuda_timeIntInit", "cuda_timeIntCleanup",
                 "cuda_timeIntHydroInitDevice", "cuda_timeIntHydroSynchFromDevice"):
        _declare(refabi, name, ip, [])
    _declare(refabi, "fecuda_SetBlocksPerGrid", ip, [ip, ip, ip])
    _declare(refabi, "fecuda_AllocateHaloBuffers", ip, [ip, ip, ip, ip])
    _declare(refabi, "cuda_timeIntCommence", ip, [ip])
    _declare(refabi, "cuda_hydroCoreDeviceBuildFrhs", ip, [ctypes.c_float, ip, ip, ctypes.c_float, ip, ip])
    _declare(refabi, "fe_refabi_domain", vp, [])
    _declare(refabi, "fe_refabi_fill_config", None, [ctypes.POINTER(FeConfig)])
    _LIBS.update(host=host, engine=engine, refabi=refabi)
    return _LIBS


def pin(a: Optional[np.ndarray]) -> None:
    """Page-lock a host array (cudaHostRegister) so copies to and from the device run at full
    link speed; undo with unpin() before the array is freed."""
    if a is not None:
        _check(load()["engine"].fe_host_register(a.ctypes.data_as(ctypes.c_void_p), a.nbytes), "fe_host_register")


def unpin(a: Optional[np.ndarray]) -> None:
    if a is not None:
        _check(load()["engine"].fe_host_unregister(a.ctypes.data_as(ctypes.c_void_p)), "fe_host_unregister")


def _fptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(c_float_p)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = _LIBS["engine"].fe_last_error().decode(errors="replace")
        raise FeError(f"{what} failed with code {rc}: {msg}")


# ---------------------------------------------------------------- host layer
class Host:
    """The repository's host C layer: FastEddy parameter file -> grid, base state, initial state.

    Arrays are numpy views of the host globals the drop-in ABI reads (reference layout).
    """

    def __init__(self) -> None:
        self.libs = load()
        self.h = self.libs["host"]

    def load_params_text(self, text: str) -> None:
        nerr = self.h.fe_host_load_params_text(text.encode())
        if nerr != 0:
            raise FeError(f"{nerr} parameter error(s): {self.h.fe_host_last_message().decode()}")

    def load_params_file(self, path: str) -> None:
        nerr = self.h.fe_host_load_params_file(path.encode())
        if nerr != 0:
            raise FeError(f"parameter file {path}: {nerr} error(s): {self.h.fe_host_last_message().decode()}")

    def unused_params(self) -> list[str]:
        buf = ctypes.create_string_buffer(8192)
        self.h.fe_host_unused_params(buf, len(buf))
        return buf.value.decode().split()

    def gaussian_hill(self, height: float, halfwidth: float) -> None:
        if self.h.fe_host_gaussian_hill(height, halfwidth) != 0:
            raise FeError(self.h.fe_host_last_message().decode())

    def set_topography(self, topo: np.ndarray) -> None:
        t = np.ascontiguousarray(topo, dtype=np.float32)
        if self.h.fe_host_set_topography(_fptr(t), t.shape[0], t.shape[1]) != 0:
            raise FeError(self.h.fe_host_last_message().decode())

    def write_binary(self, path: str | None = None, tstep: int = 0) -> None:
        """Write the host state in FastEddy's raw binary output format (one file per output
        step, io_binary.c:19-132); path None: <outPath><outFileBase>_rank_0.<tstep>."""
        if self.h.fe_host_write_binary(path.encode() if path else None, tstep) != 0:
            raise FeError(self.h.fe_host_last_message().decode())

    def write_netcdf(self, path: str | None = None, tstep: int = 0) -> None:
        """Write the host state as FastEddy's netCDF output (interior cells, dimensions time,
        zIndex, yIndex, xIndex; io_netcdf.c:392-717) in the classic 64-bit-offset container;
        path None: <outPath><outFileBase>.<tstep>."""
        if self.h.fe_host_write_netcdf(path.encode() if path else None, tstep) != 0:
            raise FeError(self.h.fe_host_last_message().decode())

    def write_topofile(self, path: str) -> None:
        if self.h.fe_host_write_topofile(path.encode()) != 0:
            raise FeError("topography not set")

    def init(self, seed: int = 12345) -> None:
        if self.h.fe_host_init(ctypes.c_ulonglong(seed)) != 0:
            raise FeError(self.h.fe_host_last_message().decode())

    def set_qv_profile(self, q_sfc: float, q_top: float, z_top: float) -> None:
        if self.h.fe_host_set_qv_profile(q_sfc, q_top, z_top) != 0:
            raise FeError("moisture not enabled")

    def gi(self, name: str) -> int:
        return ctypes.c_int.in_dll(self.h, name).value

    def gf(self, name: str) -> float:
        return ctypes.c_float.in_dll(self.h, name).value

    def set_gi(self, name: str, v: int) -> None:
        ctypes.c_int.in_dll(self.h, name).value = int(v)

    def set_gf(self, name: str, v: float) -> None:
        ctypes.c_float.in_dll(self.h, name).value = float(v)

    @property
    def shape(self) -> tuple[int, int, int]:
        nh = self.gi("Nh")
        return (self.gi("Nxp") + 2 * nh, self.gi("Nyp") + 2 * nh, self.gi("Nzp") + 2 * nh)

    def array(self, name: str, nfields: int = 1, two_d: bool = False) -> np.ndarray:
        """numpy view of a global float* host array (no copy)."""
        p = c_float_p.in_dll(self.h, name)
        if not p:
            raise FeError(f"host array {name} not allocated")
        nx, ny, nz = self.shape
        shape = (nfields, nx, ny) if two_d else (nfields, nx, ny, nz)
        cnt = int(np.prod(shape))
        buf = (ctypes.c_float * cnt).from_address(ctypes.addressof(p.contents))
        return np.frombuffer(buf, dtype=np.float32).reshape(shape)

    def config(self) -> FeConfig:
        cfg = FeConfig()
        self.libs["refabi"].fe_refabi_fill_config(ctypes.byref(cfg))
        return cfg

    def nfields(self) -> tuple[int, int]:
        cfg = self.config()
        ntke = 1 if (cfg.turbulenceSelector > 0 and cfg.TKESelector > 0) else 0
        nm = cfg.moistureNvars if cfg.moistureSelector > 0 else 0
        return ntke, nm

    def inputs(self) -> dict[str, np.ndarray]:
        """Copies of every host input of the hot path."""
        ntke, nm = self.nfields()
        d = {
            "zPos": self.array("zPos")[0].copy(), "J31": self.array("J31")[0].copy(),
            "J32": self.array("J32")[0].copy(), "J33": self.array("J33")[0].copy(),
            "D_Jac": self.array("D_Jac")[0].copy(), "invD_Jac": self.array("invD_Jac")[0].copy(),
            "baseState": self.array("hydroBaseStateFlds", 2).copy(),
            "hydroFlds": self.array("hydroFlds", 5).copy(),
        }
        d["sgstke"] = self.array("sgstkeScalars", 1).copy() if ntke else None
        d["moist"] = self.array("moistScalars", nm).copy() if nm else None
        for nm2 in ("z0m", "z0t", "htFlux", "tskin", "fricVel", "qFlux", "qskin"):
            d[nm2] = self.array(nm2, 1, two_d=True)[0].copy()
        return d

    def cleanup(self) -> None:
        self.h.fe_host_cleanup()


# ---------------------------------------------------------------- engine domain
class Domain:
    """One B200 domain (engine handle). Arrays in and out use the reference layout."""

    def __init__(self, cfg: FeConfig, device: int = 0) -> None:
        self.libs = load()
        self.e = self.libs["engine"]
        if self.e.fe_device_count() <= 0:
            raise FeError("no CUDA device visible: the engine has no CPU path")
        self.cfg = cfg
        h = ctypes.c_void_p()
        _check(self.e.fe_create(ctypes.byref(cfg), device, ctypes.byref(h)), "fe_create")
        self.h = h
        self.shape = (cfg.Nx + 6, cfg.Ny + 6, cfg.Nz + 6)
        self.ntke = 1 if (cfg.turbulenceSelector > 0 and cfg.TKESelector > 0) else 0
        self.nmoist = cfg.moistureNvars if cfg.moistureSelector > 0 else 0

    def close(self) -> None:
        if self.h:
            self.e.fe_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def set_inputs(self, inp: dict, simTime: float = 0.0, simTime_it: int = 0) -> None:
        f32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)
        g = {k: f32(inp[k]) for k in ("zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac")}
        _check(self.e.fe_set_grid(self.h, *(_fptr(g[k]) for k in ("zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac"))),
               "fe_set_grid")
        _check(self.e.fe_set_base_state(self.h, _fptr(f32(inp["baseState"]))), "fe_set_base_state")
        surf = [f32(inp.get(k)) for k in ("z0m", "z0t", "htFlux", "tskin", "fricVel", "qFlux", "qskin")]
        _check(self.e.fe_set_surface(self.h, *(_fptr(a) for a in surf)), "fe_set_surface")
        self.set_state(inp["hydroFlds"], inp.get("sgstke"), inp.get("moist"))
        _check(self.e.fe_set_clock(self.h, simTime, simTime_it), "fe_set_clock")

    def set_state(self, hydro, sgstke=None, moist=None) -> None:
        f32 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)
        _check(self.e.fe_set_state(self.h, _fptr(f32(hydro)), _fptr(f32(sgstke) if self.ntke else None),
                                   _fptr(f32(moist) if self.nmoist else None)), "fe_set_state")

    def advance(self, nsteps: int, sync: bool = True) -> None:
        _check(self.e.fe_advance(self.h, nsteps), "fe_advance")
        if sync:
            self.sync()

    def sync(self) -> None:
        _check(self.e.fe_sync(self.h), "fe_sync")

    def stream(self) -> int:
        return int(self.e.fe_stream(self.h) or 0)

    def state_buffers(self) -> dict[str, np.ndarray]:
        """Empty host arrays of the shapes get_state() returns (to pass as `out`)."""
        nx, ny, nz = self.shape
        return {"hydroFlds": np.empty((5, nx, ny, nz), np.float32),
                "sgstke": np.empty((1, nx, ny, nz), np.float32) if self.ntke else None,
                "moist": np.empty((self.nmoist, nx, ny, nz), np.float32) if self.nmoist else None,
                "pres": np.empty((nx, ny, nz), np.float32)}

    def get_state(self, out: dict | None = None) -> dict[str, np.ndarray]:
        """The state (flux form, reference layout) and perturbation pressure; into `out`
        (from state_buffers(), e.g. page-locked with pin()) when given."""
        b = out if out is not None else self.state_buffers()
        hydro, tke, moist, pres = b["hydroFlds"], b["sgstke"], b["moist"], b["pres"]
        _check(self.e.fe_get_state(self.h, _fptr(hydro), _fptr(tke), _fptr(moist), _fptr(pres)), "fe_get_state")
        return {"hydroFlds": hydro, "sgstke": tke, "moist": moist, "pres": pres}

    def get_surface(self) -> dict[str, np.ndarray]:
        nx, ny, _ = self.shape
        names = ("cd", "ch", "fricVel", "htFlux", "invOblen", "tskin", "qFlux", "qskin")
        out = {k: np.empty((nx, ny), np.float32) for k in names}
        _check(self.e.fe_get_surface(self.h, *(_fptr(out[k]) for k in names)), "fe_get_surface")
        return out

    def build_frhs(self, stage: int, taus: bool = True) -> dict[str, np.ndarray]:
        _check(self.e.fe_build_frhs(self.h, stage), "fe_build_frhs")
        nx, ny, nz = self.shape
        F = np.empty((5, nx, ny, nz), np.float32)
        Fe = np.empty((1, nx, ny, nz), np.float32) if self.ntke else None
        Fm = np.empty((self.nmoist, nx, ny, nz), np.float32) if self.nmoist else None
        taus = np.empty((9, nx, ny, nz), np.float32) if taus else None
        _check(self.e.fe_get_frhs(self.h, _fptr(F), _fptr(Fe), _fptr(Fm), _fptr(taus)), "fe_get_frhs")
        return {"hydroFrhs": F, "sgstkeFrhs": Fe, "moistFrhs": Fm, "taus": taus}

    def set_forcing_capture(self, on: bool) -> None:
        """Keep the last RK stage's tendencies of the last step of every later advance."""
        _check(self.e.fe_set_forcing_capture(self.h, 1 if on else 0), "fe_set_forcing_capture")

    def last_forcing(self) -> dict[str, np.ndarray]:
        """Tendencies kept by the last advance (set_forcing_capture) and the SGS fluxes of the
        last physics stage: hydroFrhs, sgstkeFrhs, moistFrhs, taus, moistTaus."""
        nx, ny, nz = self.shape
        F = np.empty((5, nx, ny, nz), np.float32)
        Fe = np.empty((1, nx, ny, nz), np.float32) if self.ntke else None
        Fm = np.empty((self.nmoist, nx, ny, nz), np.float32) if self.nmoist else None
        _check(self.e.fe_get_frhs(self.h, _fptr(F), _fptr(Fe), _fptr(Fm), None), "fe_get_frhs")
        out = {"hydroFrhs": F, "sgstkeFrhs": Fe, "moistFrhs": Fm}
        out.update(self.sgs_fluxes())
        return out

    def sgs_fluxes(self) -> dict[str, np.ndarray]:
        """SGS stresses/heat fluxes (9) and moisture SGS fluxes (3 per species, when the
        configuration has them) of the last physics stage."""
        nx, ny, nz = self.shape
        cfg = self.cfg
        taus = np.empty((9, nx, ny, nz), np.float32) if cfg.turbulenceSelector > 0 else None
        mt = None
        if cfg.turbulenceSelector > 0 and self.nmoist and cfg.moistureSGSturb > 0:
            mt = np.empty((3 * self.nmoist, nx, ny, nz), np.float32)
        if taus is not None:
            _check(self.e.fe_get_sgs_fluxes(self.h, _fptr(taus), _fptr(mt)), "fe_get_sgs_fluxes")
        return {"taus": taus, "moistTaus": mt}

    def nonfinite(self) -> int:
        c = ctypes.c_longlong()
        _check(self.e.fe_count_nonfinite(self.h, ctypes.byref(c)), "fe_count_nonfinite")
        return int(c.value)

    def means(self) -> np.ndarray:
        out = np.zeros(5 + self.ntke + self.nmoist, np.float64)
        _check(self.e.fe_domain_means(self.h, out.ctypes.data_as(c_double_p)), "fe_domain_means")
        return out

    def set_tiling(self, tk: int, tj: int, ti: int) -> None:
        _check(self.e.fe_set_tiling(self.h, tk, tj, ti), "fe_set_tiling")

    def clock(self) -> tuple[float, int]:
        t, it = ctypes.c_float(), ctypes.c_int()
        _check(self.e.fe_get_clock(self.h, ctypes.byref(t), ctypes.byref(it)), "fe_get_clock")
        return float(t.value), int(it.value)

    def checkpoint(self) -> bytes:
        """State, surface planes and clock as one byte string (fe_checkpoint_save)."""
        n = int(self.e.fe_checkpoint_bytes(self.h))
        buf = ctypes.create_string_buffer(n)
        _check(self.e.fe_checkpoint_save(self.h, buf, n), "fe_checkpoint_save")
        return buf.raw

    def restore(self, blob: bytes) -> None:
        """Resume from a checkpoint (the grid and base state must already be set)."""
        buf = ctypes.create_string_buffer(blob, len(blob))
        _check(self.e.fe_checkpoint_load(self.h, buf, len(blob)), "fe_checkpoint_load")

    def set_sgs_mlp(self, mlp: Optional["Mlp"]) -> None:
        """Learned SGS stresses from `mlp` (None: the TKE closure)."""
        _check(self.e.fe_set_sgs_mlp(self.h, mlp.h if mlp is not None else None), "fe_set_sgs_mlp")
        self._mlp = mlp  # keep the network alive while the domain uses it

    def sgs_sample(self, every: int = 1) -> dict[str, np.ndarray]:
        """Closure inputs X (n x 11), stresses tau (n x 9) and rho of every `every`-th interior cell."""
        cells = (self.cfg.Nx * self.cfg.Ny * self.cfg.Nz + every - 1) // every
        X = np.empty((cells, SGS_NIN), np.float32)
        tau = np.empty((cells, SGS_NOUT), np.float32)
        rho = np.empty(cells, np.float32)
        _check(self.e.fe_sgs_sample(self.h, every, _fptr(X), _fptr(tau), _fptr(rho)), "fe_sgs_sample")
        return {"X": X, "tau": tau, "rho": rho}

    def coarsen_into(self, coarse: "Domain") -> np.ndarray:
        """2x2x2 box filter of this (fine) state into `coarse`; returns the subfilter targets tau/rho."""
        cells = coarse.cfg.Nx * coarse.cfg.Ny * coarse.cfg.Nz
        tgt = np.empty((cells, SGS_NOUT), np.float32)
        _check(self.e.fe_coarsen(self.h, coarse.h, _fptr(tgt)), "fe_coarsen")
        return tgt

    def set_stage_kernel(self, kind: str, tj: int = 0, ni: int = 0) -> None:
        """kind 'march' (tiles of 32 levels x tj rows marching ni planes) or 'cell'."""
        code = {"cell": KERNEL_CELL, "march": KERNEL_MARCH}[kind]
        _check(self.e.fe_set_stage_kernel(self.h, code, tj, ni), "fe_set_stage_kernel")

    def set_sgs_kernel(self, rows: int) -> None:
        """Last-stage SGS physics as one fused kernel with tiles of `rows` rows (8 or 16), or
        (rows = 0) as the separate kernels."""
        _check(self.e.fe_set_sgs_kernel(self.h, int(rows)), "fe_set_sgs_kernel")

    def set_sgs_shape(self, rows: int, ni: int) -> None:
        """The fused SGS kernel's tile rows (8 or 16; 0 = the separate kernels) and planes per block."""
        _check(self.e.fe_set_sgs_shape(self.h, int(rows), int(ni)), "fe_set_sgs_shape")

    def sgs_shape(self) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(self.e.fe_get_sgs_shape(self.h, ctypes.byref(a), ctypes.byref(b)), "fe_get_sgs_shape")
        return a.value, b.value

    def stage_kernel(self) -> tuple[str, int, int]:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.e.fe_get_stage_kernel(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "fe_get_stage_kernel")
        return ("march" if a.value == KERNEL_MARCH else "cell"), b.value, c.value

    def autotune(self) -> tuple[str, int, int]:
        """Time the candidate stage-kernel forms/shapes, keep the fastest, return (kind, tj, ni|ti)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(self.e.fe_autotune(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "fe_autotune")
        return self.stage_kernel()

    def time_stage_kernel(self, reps: int = 10) -> float:
        """Mean ms per launch of the fused dynamics stage kernel (CUDA events)."""
        ms = ctypes.c_float()
        _check(self.e.fe_time_stage_kernel(self.h, reps, ctypes.byref(ms)), "fe_time_stage_kernel")
        return float(ms.value)

    def launch_count(self) -> int:
        return int(self.e.fe_launch_count(self.h))

    def device_bytes(self) -> int:
        return int(self.e.fe_device_bytes(self.h))


class Ensemble:
    """Several domains of one device advanced by one captured CUDA graph per step batch."""

    def __init__(self, members: list[Domain]) -> None:
        self.libs = load()
        self.e = self.libs["engine"]
        self.members = members
        arr = (ctypes.c_void_p * len(members))(*[m.h.value for m in members])
        h = ctypes.c_void_p()
        _check(self.e.fe_ensemble_create(arr, len(members), ctypes.byref(h)), "fe_ensemble_create")
        self.h = h

    def advance(self, nsteps: int, sync: bool = True) -> None:
        _check(self.e.fe_ensemble_advance(self.h, nsteps), "fe_ensemble_advance")
        if sync:
            _check(self.e.fe_ensemble_sync(self.h), "fe_ensemble_sync")

    def stream(self) -> int:
        return int(self.e.fe_ensemble_stream(self.h) or 0)

    def set_batched(self, on: bool) -> None:
        """Work-list launches over all members (when they allow it) or one graph branch per member."""
        _check(self.e.fe_ensemble_set_batched(self.h, int(on)), "fe_ensemble_set_batched")

    def batched(self) -> bool:
        """Whether the advances so far used the work-list launches."""
        return bool(self.e.fe_ensemble_is_batched(self.h))

    def launch_count(self) -> int:
        return int(self.e.fe_ensemble_launch_count(self.h))

    def close(self) -> None:
        if self.h:
            self.e.fe_ensemble_destroy(self.h)
            self.h = ctypes.c_void_p()


class Mlp:
    """The learned SGS closure (fe_mlp handle): parameters, training set, Adam, prediction."""

    def __init__(self, device: int = 0, seed: int = 1) -> None:
        self.libs = load()
        self.e = self.libs["engine"]
        h = ctypes.c_void_p()
        _check(self.e.fe_mlp_create(device, seed, ctypes.byref(h)), "fe_mlp_create")
        self.h = h
        self.nparams = int(self.e.fe_mlp_param_count())

    def close(self) -> None:
        if self.h:
            self.e.fe_mlp_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.empty(self.nparams, np.float32)
        _check(self.e.fe_mlp_get_params(self.h, _fptr(p)), "fe_mlp_get_params")
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        _check(self.e.fe_mlp_set_params(self.h, _fptr(p)), "fe_mlp_set_params")

    def norm(self) -> dict[str, np.ndarray]:
        a = [np.empty(SGS_NIN, np.float32), np.empty(SGS_NIN, np.float32), np.empty(SGS_NOUT, np.float32),
             np.empty(SGS_NOUT, np.float32)]
        _check(self.e.fe_mlp_get_norm(self.h, *(_fptr(x) for x in a)), "fe_mlp_get_norm")
        return dict(zip(("in_mu", "in_sig", "out_mu", "out_sig"), a))

    def set_norm(self, in_mu, in_sig, out_mu, out_sig) -> None:
        a = [np.ascontiguousarray(x, np.float32) for x in (in_mu, in_sig, out_mu, out_sig)]
        _check(self.e.fe_mlp_set_norm(self.h, *(_fptr(x) for x in a)), "fe_mlp_set_norm")

    def set_data(self, X: np.ndarray, T: np.ndarray, seed: int = 7, fit_norm: bool = True) -> None:
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        assert X.shape[1] == SGS_NIN and T.shape == (X.shape[0], SGS_NOUT)
        _check(self.e.fe_mlp_set_data(self.h, _fptr(X), _fptr(T), X.shape[0], seed, 1 if fit_norm else 0),
               "fe_mlp_set_data")

    def gradient(self, first: int, count: int) -> tuple[np.ndarray, float]:
        g = np.empty(self.nparams, np.float32)
        loss = ctypes.c_double()
        _check(self.e.fe_mlp_gradient(self.h, first, count, _fptr(g), ctypes.byref(loss)), "fe_mlp_gradient")
        return g, float(loss.value)

    def train(self, steps: int, batch: int, lr: float) -> np.ndarray:
        hist = np.zeros(steps, np.float64)
        _check(self.e.fe_mlp_train(self.h, steps, batch, lr, hist.ctypes.data_as(c_double_p)), "fe_mlp_train")
        return hist

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        Y = np.empty((X.shape[0], SGS_NOUT), np.float32)
        _check(self.e.fe_mlp_predict(self.h, _fptr(X), X.shape[0], _fptr(Y)), "fe_mlp_predict")
        return Y

    def time(self, train: bool, batch: int, reps: int = 10) -> float:
        ms = ctypes.c_float()
        _check(self.e.fe_mlp_time(self.h, 1 if train else 0, batch, reps, ctypes.byref(ms)), "fe_mlp_time")
        return float(ms.value)


def read_binary(path: str) -> dict[str, np.ndarray]:
    """Records of a FastEddy raw binary output file (io_binary.c:59-126), in file order: name ->
    float32 array of the halo-inclusive extents (nx, ny, nz) or (nx, ny)."""
    out: dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        (nlen,) = np.frombuffer(data, np.int32, 1, pos)
        name = data[pos + 4:pos + 4 + int(nlen)].decode()
        pos += 4 + int(nlen)
        (nd,) = np.frombuffer(data, np.int32, 1, pos)
        ext = tuple(int(e) for e in np.frombuffer(data, np.int32, int(nd), pos + 4))
        pos += 4 + 4 * int(nd)
        cnt = int(np.prod(ext))
        out[name] = np.frombuffer(data, np.float32, cnt, pos).reshape(ext).copy()
        pos += 4 * cnt
    return out

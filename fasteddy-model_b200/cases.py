"""FastEddy parameter files for the benchmark cases, written in the reference's key format.

Each case is a plain FastEddy parameter file (the same keys an existing FastEddy user
writes), so the host layer, the drop-in ABI and the reference build all read the same
input. Sizes can be shrunk for tests; the physics settings stay those of the case.

  cbl_dry        dry convective boundary layer, flat terrain (the 128x128x64 case)
  cbl_moist_hill moist CBL over a Gaussian hill with Rayleigh damping (the 512x512x128 case)
  abl_neutral    neutral ABL member of the batched ensemble
  cbl_hill_dry   large dry CBL over the hill (the 1024x1024x256 case)
  bomex          moist CBL, flat, with the selectors of FastEddy's BOMEX tutorial (HYB34 for q_v,
                 explicit filter, large-scale forcing with slab-mean subsidence, mixing-ratio
                 condensation on the base pressure)
"""
from __future__ import annotations

import math
import re

# Coriolis parameter f = 1e-4 s^-1: FastEddy takes a latitude, f = 2*Omega*sin(lat)
F_CORIOLIS = 1.0e-4
LAT_F1EM4 = math.degrees(math.asin(F_CORIOLIS / 1.45842e-4))

_BASE = """Description = {desc}
numProcsX = 1
numProcsY = 1
tBx = 1
tBy = {tby}
tBz = {tbz}
inPath =
inFile =
outPath = ./output/
outFileBase = FE_B200
frqOutput = {nt}
ioOutputMode = 1
Nx = {nx}
Ny = {ny}
Nz = {nz}
Nh = 3
d_xi = {dx}
d_eta = {dy}
d_zeta = {dz}
coordHorizHalos = 1
topoFile = {topo}
verticalDeformSwitch = 0
verticalDeformFactor = 1.0
verticalDeformQuadCoeff = 0.0
timeMethod = 0
Nt = {nt}
dt = {dt}
NtBatch = {nt}
hydroBCs = 2
hydroForcingWrite = 0
hydroSubGridWrite = 0
hydroForcingLog = 0
advectionSelector = 3
b_hyb = 0.0
moistureSelector = {moist}
moistureNvars = 2
moistureAdvSelectorQv = 3
moistureAdvSelectorQv_b = 0.0
moistureAdvSelectorQi = 2
moistureSGSturb = 1
moistureCond = 2
moistureCondTscale = 1.0
moistureCondBasePres = 0
moistureMPcallTscale = 1.0
surflayer_wq = 0.0
surflayer_qr = 0.0
coriolisSelector = 1
coriolisLatitude = {lat:.10f}
turbulenceSelector = 1
TKESelector = 1
TKEAdvSelector = 3
TKEAdvSelector_b_hyb = 0.0
c_s = 0.18
c_k = 0.10
diffusionSelector = 0
nu_0 = 0.0
filterSelector = 0
filter_6th_coeff = 0.03
dampingLayerSelector = {damp}
dampingLayerDepth = {dampdepth}
surflayerSelector = 1
surflayer_z0 = {z0}
surflayer_z0t = {z0}
surflayer_wth = {wth}
surflayer_tr = 0.0
surflayer_idealsine = 0
stabilityScheme = 1
temp_grnd = 300.0
pres_grnd = 100000.0
zStableBottom = {zsb}
stableGradient = 0.008
zStableBottom2 = 6000.0
stableGradient2 = 0.08
zStableBottom3 = 50000.0
stableGradient3 = 0.003
thetaPerturbationSwitch = {pert}
thetaHeight = 400.0
thetaAmplitude = 0.25
U_g = {ug}
V_g = 0.0
z_Ug = 10000.0
z_Vg = 10000.0
Ug_grad = 0.0
Vg_grad = 0.0
lsfSelector = 0
lsf_horMnSubTerms = 0
lsf_freq = 1.0
lsf_w_surf = 0.0
lsf_w_lev1 = 0.0
lsf_w_lev2 = 0.0
lsf_w_zlev1 = 100.0
lsf_w_zlev2 = 200.0
lsf_th_surf = 0.0
lsf_th_lev1 = 0.0
lsf_th_lev2 = 0.0
lsf_th_zlev1 = 100.0
lsf_th_zlev2 = 200.0
lsf_qv_surf = 0.0
lsf_qv_lev1 = 0.0
lsf_qv_lev2 = 0.0
lsf_qv_zlev1 = 100.0
lsf_qv_zlev2 = 200.0
physics_oneRKonly = 1
"""


# Selectors of the BOMEX tutorial (tutorials/examples/Example04_BOMEX.in) applied to the moist case.
BOMEX = dict(moistureAdvSelectorQv=2, moistureCond=3, moistureCondBasePres=1, filterSelector=1, filter_6th_coeff=0.03,
             lsfSelector=1, lsf_horMnSubTerms=1, lsf_freq=1.0, lsf_w_surf=0.0, lsf_w_lev1=-23.4, lsf_w_lev2=0.0,
             lsf_w_zlev1=1500.0, lsf_w_zlev2=2100.0, lsf_th_surf=-0.0833333, lsf_th_lev1=-0.0833333, lsf_th_lev2=0.0,
             lsf_th_zlev1=1500.0, lsf_th_zlev2=3000.0, lsf_qv_surf=-0.0432, lsf_qv_lev1=-0.0432, lsf_qv_lev2=0.0,
             lsf_qv_zlev1=300.0, lsf_qv_zlev2=500.0, surflayer_wq=0.052)


# Time step. The cases ask for dx = dy = 20 m, dz = 10 m and dt = 0.05 s, but the
# explicit acoustic step of this model is unstable there: c*dt*sqrt(dx^-2+dy^-2+dz^-2)
# = 347*0.05*0.1225 = 2.1 exceeds the RK3 limit sqrt(3), and the reference build, the FP64
# oracle and this engine all overflow after ~30 steps. dt = 0.025 s (1.06) is stable; the
# work per step is unchanged.
DT_STABLE = 0.025


def exact_tb(ny: int, nz: int, max_threads: int = 256) -> tuple[int, int]:
    """(tBy, tBz) dividing the halo-inclusive extents exactly: tBz the largest divisor of Nz+6
    within CUDA's 64-thread limit on a block's z extent, tBy the largest divisor of Ny+6 that
    keeps the block at most `max_threads` threads (the reference's register-heavy kernels)."""
    nzh, nyh = nz + 6, ny + 6
    tbz = max(t for t in range(1, min(nzh, 64) + 1) if nzh % t == 0)
    tby = max(t for t in range(1, nyh + 1) if nyh % t == 0 and t * tbz <= max_threads)
    return tby, tbz


def param_text(case: str, nx: int, ny: int, nz: int, *, dx: float = 20.0, dz: float = 10.0, dt: float = DT_STABLE,
               nt: int = 100, topo: str = "", ug: float = 10.0, z0: float = 0.05, tb: tuple[int, int] | None = None,
               params: dict | None = None) -> str:
    """Parameter file text of `case` at the given size.

    tb = (tBy, tBz) sets the reference build's thread-block shape; by default the
    tutorials' (4, 64). A shape that divides the halo-inclusive extents exactly avoids
    the reference's out-of-range threads (see oracle/refrun.py).
    params = {key: value} overrides keys of the case (e.g. advectionSelector, filterSelector);
    every key must already be in the file."""
    tby, tbz = tb if tb is not None else (4, 64)
    ztop = nz * dz - 0.5 * dz
    if case == "cbl_dry":
        kw = dict(desc="dry CBL, flat terrain", moist=0, damp=0, dampdepth=100.0, wth=0.35, zsb=600.0, pert=1)
    elif case == "cbl_moist_hill":
        kw = dict(desc="moist CBL over a Gaussian hill", moist=1, damp=1, dampdepth=round(0.2 * nz * dz, 3),
                  wth=0.35, zsb=600.0, pert=1)
    elif case == "cbl_hill_dry":
        kw = dict(desc="dry CBL over a Gaussian hill", moist=0, damp=1, dampdepth=round(0.2 * nz * dz, 3),
                  wth=0.35, zsb=600.0, pert=1)
    elif case == "bomex":
        kw = dict(desc="BOMEX-configured moist CBL, flat terrain", moist=1, damp=1, dampdepth=round(0.2 * nz * dz, 3),
                  wth=0.008, zsb=600.0, pert=1)
        params = dict(BOMEX, **(params or {}))
    elif case == "abl_neutral":
        kw = dict(desc="neutral ABL ensemble member", moist=0, damp=0, dampdepth=100.0, wth=0.0,
                  zsb=round(0.8 * ztop, 3), pert=1)
    else:
        raise ValueError(f"unknown case {case}")
    text = _BASE.format(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dz, dt=dt, nt=nt, topo=topo, lat=LAT_F1EM4, ug=ug,
                        z0=z0, tby=tby, tbz=tbz, **kw)
    for key, value in (params or {}).items():
        text, n = re.subn(rf"^{re.escape(key)} = .*$", f"{key} = {value}", text, flags=re.M)
        if n != 1:
            raise ValueError(f"{key} is not a key of the {case} parameter file")
    return text


# Gaussian hill of the terrain cases: height 200 m, half-width 1 km (h = 200 * 2^-(r/1km)^2)
HILL_HEIGHT = 200.0
HILL_HALFWIDTH = 1000.0
# Water vapour profile of the moist case: 14 g/kg at the surface, 4 g/kg at 1.5 km
QV_SFC, QV_TOP, QV_ZTOP = 14.0, 4.0, 1500.0


def setup_host(case: str, nx: int, ny: int, nz: int, seed: int = 12345, hill_halfwidth: float | None = None,
               hill_height: float = HILL_HEIGHT, qv: tuple[float, float, float] | None = None, **kw):
    """Load the case into the host layer (grid, base state, initial state). Returns the Host.

    qv = (q_sfc, q_top, z_top) overrides the water-vapour profile of the moist case
    (tests use a supersaturated one to exercise the saturation adjustment)."""
    from .runtime import Host

    host = Host()
    host.load_params_text(param_text(case, nx, ny, nz, **kw))
    if case in ("cbl_moist_hill", "cbl_hill_dry"):
        host.gaussian_hill(hill_height, HILL_HALFWIDTH if hill_halfwidth is None else hill_halfwidth)
    host.init(seed)
    if case in ("cbl_moist_hill", "bomex"):
        host.set_qv_profile(*(qv if qv is not None else (QV_SFC, QV_TOP, QV_ZTOP)))
    return host

"""The host layer's inputs of the CUDA path against the reference's own host code on the same
parameter file: coordinates and metrics (SRC/GRID/grid.c:386-803), the hydrostatic base state
and initial state (SRC/HYDRO_CORE/hydro_core.c:1053-1250), the surface arrays
(hydro_core.c:835-860). The reference side is oracle/_ref/fe_ref_io in its dump mode, built from
the reference's host modules by oracle/build_ref.py; it runs without a GPU.

Tolerances. Coordinates and metrics follow the reference's float expressions and must be equal
bit for bit, halos included. The base state is integrated in FP64 here and in float (with
double pow) by the reference, so rho_BS and (rho theta)_BS agree to the reference's float
rounding (relative 1e-6). The theta perturbations of the two programs come from different random
streams (splitmix64 here, the C library's rand() there), so with perturbations on only their
support and bound are compared: the same cells (interior, z <= thetaHeight) are perturbed, by at
most thetaAmplitude; without perturbations the whole initial state is compared.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, interior, rel_l2

REF_IO = os.path.join(ROOT, "oracle", "_ref", "fe_ref_io")


def _reference_dump(text: str, shape, tmp_path, files: dict | None = None) -> dict:
    work = tmp_path / "ref"
    work.mkdir()
    (work / "output").mkdir()
    pf = work / "params.in"
    pf.write_text(text)
    for name, blob in (files or {}).items():
        (work / name).write_bytes(blob)
    out = work / "dump"
    out.mkdir()
    res = subprocess.run([REF_IO, str(pf), str(out), "dump"], capture_output=True, text=True, cwd=str(work),
                         timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    nx, ny, nz = shape
    got = {}
    for p in out.iterdir():
        a = np.fromfile(str(p), dtype=np.float32)
        n3 = nx * ny * nz
        got[p.stem] = a.reshape(-1, nx, ny, nz) if a.size % n3 == 0 and a.size >= n3 else a.reshape(-1, nx, ny)
    return got


def _ours(host) -> dict:
    ntke, nm = host.nfields()
    d = {n: host.array(n)[0] for n in ("xPos", "yPos", "zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac")}
    d["topoPos"] = host.array("topoPos", 1, two_d=True)[0]
    d["baseState"] = host.array("hydroBaseStateFlds", 2)
    d["hydroFlds"] = host.array("hydroFlds", 5)
    if ntke:
        d["sgstke"] = host.array("sgstkeScalars", 1)
    for n in ("tskin", "fricVel", "htFlux", "z0m", "z0t", "qskin", "qFlux"):
        d[n] = host.array(n, 1, two_d=True)[0]
    return d


@pytest.mark.parametrize("case,kw", [
    ("cbl_dry", {}),
    ("cbl_hill_dry", dict(hill_halfwidth=120.0, hill_height=40.0)),
    ("cbl_moist_hill", dict(hill_halfwidth=150.0, hill_height=30.0)),
])
@pytest.mark.parametrize("pert", [0, 1])
def test_initial_inputs_match_the_reference_host_code(fe, tmp_path, case, kw, pert):
    if not os.path.exists(REF_IO):
        pytest.skip("reference host program not built (python oracle/build_ref.py)")
    nx, ny, nz = 24, 20, 48  # 475 m deep: the 400 m perturbation layer and the air above it
    params = {"thetaPerturbationSwitch": pert}
    host = fe.cases.setup_host(case, nx, ny, nz, params=params, **kw)
    files, topo = {}, ""
    if "hill" in case:
        host.write_topofile(str(tmp_path / "hill.topo"))
        files["hill.topo"] = (tmp_path / "hill.topo").read_bytes()
        topo = "./hill.topo"
    text = fe.cases.param_text(case, nx, ny, nz, topo=topo, params=params)
    ref = _reference_dump(text, host.shape, tmp_path, files)
    ours = _ours(host)

    # grid: coordinates, terrain and metrics bit for bit (halo-inclusive, as both build them)
    for name in ("xPos", "yPos", "zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac"):
        np.testing.assert_array_equal(ours[name], ref[name][0], err_msg=name)
    np.testing.assert_array_equal(ours["topoPos"], ref["topoPos"][0])
    # base state: FP64 here, float in the reference
    for f in range(2):
        assert rel_l2(interior(ours["baseState"][f]), interior(ref["baseState"][f])) < 1e-6, f
    # initial state
    rho_o, rho_r = ours["hydroFlds"][0], ref["hydroFlds"][0]
    assert rel_l2(interior(rho_o), interior(rho_r)) < 1e-6
    for f in (1, 2, 3):
        assert rel_l2(interior(ours["hydroFlds"][f]), interior(ref["hydroFlds"][f])) < 1e-6, f
    th_o = interior(ours["hydroFlds"][4]).astype(np.float64) / interior(rho_o)
    th_r = interior(ref["hydroFlds"][4]).astype(np.float64) / interior(rho_r)
    th_bs = interior(ref["baseState"][1]).astype(np.float64) / interior(ref["baseState"][0])
    if pert == 0:
        assert rel_l2(th_o, th_r) < 1e-6
    else:
        amp = 0.25
        below = interior(ref["zPos"][0]) <= 400.0
        for th in (th_o, th_r):
            dth = th - th_bs
            # the bound to the float rounding of rho theta / rho (~300 K * 1e-7)
            assert np.abs(dth[below]).max() <= amp + 1e-4 and np.abs(dth[below]).max() > 0.5 * amp
            assert np.abs(dth[~below]).max() < 1e-4  # only the cells the reference perturbs
    if "sgstke" in ref:
        assert rel_l2(interior(ours["sgstke"][0]), interior(ref["sgstke"][0])) < 1e-6
    for name in ("tskin", "fricVel", "htFlux", "z0m", "z0t"):
        np.testing.assert_allclose(ours[name][3:-3, 3:-3], ref[name][0][3:-3, 3:-3], rtol=1e-6, err_msg=name)
    host.cleanup()

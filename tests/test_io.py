"""FastEddy's raw binary output (io_binary.c:19-132) written by the host layer, checked byte for
byte against the reference's own writer (oracle/_ref/fe_ref_io, built by oracle/build_ref.py
from the reference's host modules; it needs no GPU) on identical host arrays."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

REF_IO = os.path.join(ROOT, "oracle", "_ref", "fe_ref_io")

# every registered array of the host layer: (file name for the reference program, host symbol,
# fields, 2-D)
ARRAYS = [("xPos", "xPos", 1, False), ("yPos", "yPos", 1, False), ("zPos", "zPos", 1, False),
          ("topoPos", "topoPos", 1, True), ("hydroFlds", "hydroFlds", 5, False), ("hydroPres", "hydroPres", 1, False),
          ("hydroFldsFrhs", "hydroFldsFrhs", 5, False), ("sgstke", "sgstkeScalars", 1, False),
          ("sgstkeFrhs", "sgstkeScalarsFrhs", 1, False), ("taus", "hydroTauFlds", 9, False),
          ("tskin", "tskin", 1, True), ("fricVel", "fricVel", 1, True), ("htFlux", "htFlux", 1, True),
          ("invOblen", "invOblen", 1, True), ("z0m", "z0m", 1, True), ("z0t", "z0t", 1, True),
          ("qskin", "qskin", 1, True), ("qFlux", "qFlux", 1, True)]


def _host(fe, case, params, outdir):
    host = fe.Host()
    text = fe.cases.param_text(case, 8, 6, 6, params=params).replace("outPath = ./output/", f"outPath = {outdir}/")
    host.load_params_text(text)
    host.init(5)
    return host, text


@pytest.mark.parametrize("case,params", [
    ("cbl_moist_hill", dict(hydroForcingWrite=1, hydroSubGridWrite=1)),  # every optional record
    ("cbl_dry", {}),  # the default record list
])
def test_binary_output_matches_the_reference_writer(fe, tmp_path, case, params):
    if not os.path.exists(REF_IO):
        pytest.skip("reference IO program not built (python oracle/build_ref.py)")
    ours, ref, ind = tmp_path / "ours", tmp_path / "ref", tmp_path / "in"
    for d in (ours, ref, ind):
        d.mkdir()
    host, text = _host(fe, case, params, ours)
    ntke, nm = host.nfields()
    rng = np.random.default_rng(11)
    arrays = list(ARRAYS)
    if nm:
        arrays += [("moist", "moistScalars", nm, False), ("moistFrhs", "moistScalarsFrhs", nm, False),
                   ("moistTaus", "moistTauFlds", 3 * nm, False)]
    for fname, sym, nf, two_d in arrays:
        if sym.startswith("sgstke") and not ntke:
            continue
        a = host.array(sym, nf, two_d)
        if sym in ("hydroPres", "hydroFldsFrhs", "sgstkeScalarsFrhs", "hydroTauFlds", "invOblen", "moistScalarsFrhs",
                   "moistTauFlds"):
            a[...] = rng.standard_normal(a.shape).astype(np.float32)  # fields the initial state leaves at 0
        a.tofile(str(ind / f"{fname}.bin"))
    host.write_binary(None, 7)
    (tmp_path / "ref.in").write_text(text.replace(f"outPath = {ours}/", f"outPath = {ref}/"))
    res = subprocess.run([REF_IO, str(tmp_path / "ref.in"), str(ind), "7"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    name = "FE_B200_rank_0.7"
    mine, theirs = (ours / name).read_bytes(), (ref / name).read_bytes()
    assert len(mine) == len(theirs)
    assert mine == theirs
    recs = fe.read_binary(str(ours / name))
    state = host.array("hydroFlds", 5)
    np.testing.assert_array_equal(recs["rho"], state[0])
    np.testing.assert_array_equal(recs["u"], state[1] / state[0])
    assert ("Tau11" in recs) == bool(params) and ("F_theta" in recs) == bool(params)
    host.cleanup()


@pytest.mark.parametrize("case,params", [("cbl_moist_hill", dict(hydroForcingWrite=1, hydroSubGridWrite=1)), ("cbl_dry", {})])
def test_netcdf_output_has_the_reference_data_model(fe, tmp_path, case, params):
    """The netCDF output (io_netcdf.c:392-717) read back by an independent reader (scipy's
    classic-format netcdf_file): dimensions time (one record), zIndex, yIndex, xIndex; int
    coordinate variables 0..N-1; the registered variables in the binary file's order, float over
    (time, z, y, x) or (time, y, x), holding the binary record's interior cells transposed."""
    from scipy.io import netcdf_file

    host, _ = _host(fe, case, params, tmp_path)
    rng = np.random.default_rng(3)
    for sym, nf in (("hydroPres", 1), ("hydroFldsFrhs", 5), ("hydroTauFlds", 9)):
        a = host.array(sym, nf)
        a[...] = rng.standard_normal(a.shape).astype(np.float32)
    host.write_binary(str(tmp_path / "out.bin"))
    host.write_netcdf(None, 3)
    recs = fe.read_binary(str(tmp_path / "out.bin"))
    nx, ny, nz = (e - 6 for e in host.shape)
    with netcdf_file(str(tmp_path / "FE_B200.3"), "r", mmap=False) as nc:
        assert nc.version_byte == 2
        assert nc.dimensions == {"time": None, "zIndex": nz, "yIndex": ny, "xIndex": nx}
        assert "time" not in nc.variables  # a dimension only, as in the reference
        names = [k for k in nc.variables if k not in ("zIndex", "yIndex", "xIndex")]
        assert names == list(recs)
        for d, n in (("zIndex", nz), ("yIndex", ny), ("xIndex", nx)):
            np.testing.assert_array_equal(nc.variables[d][:], np.arange(n))
            assert nc.variables[d].typecode() == "i"
        for name, rec in recs.items():
            var = nc.variables[name]
            assert var.typecode() == "f"
            got = np.asarray(var[:])
            assert got.shape[0] == 1
            if rec.ndim == 3:
                assert var.dimensions == ("time", "zIndex", "yIndex", "xIndex")
                np.testing.assert_array_equal(got[0], rec[3:-3, 3:-3, 3:-3].transpose(2, 1, 0))
            else:
                assert var.dimensions == ("time", "yIndex", "xIndex")
                np.testing.assert_array_equal(got[0], rec[3:-3, 3:-3].T)
    host.cleanup()


def test_restart_from_netcdf_output(fe, tmp_path):
    """An inFile restart (FastEddy.c:202-243, io_netcdf.c:106-390, time_integration.c:95-105) from
    the netCDF output of a perturbed state: the step comes from the name's suffix, the grid from
    the file's topography, rho and the surface planes come back exactly, the flux-form fields
    ((phi/rho) * rho) to one rounding, and the surface planes get their periodic halos."""
    a, text = _host(fe, "cbl_moist_hill", {}, tmp_path)
    a.gaussian_hill(12.0, 50.0)
    a.init(5)
    rng = np.random.default_rng(9)
    H = a.array("hydroFlds", 5)
    H[1:4] += rng.standard_normal(H[1:4].shape).astype(np.float32)
    M = a.array("moistScalars", 2)
    M[1] = np.abs(rng.standard_normal(M[1].shape)).astype(np.float32) * 1e-3
    for nm in ("tskin", "htFlux", "fricVel"):
        p = a.array(nm, 1, True)
        p[...] = rng.random(p.shape).astype(np.float32)
    a.write_netcdf(str(tmp_path / "RUN.40"))
    ia = {k: (v.copy() if v is not None else None) for k, v in a.inputs().items()}
    ta = a.array("topoPos", 1, True).copy()
    a.cleanup()

    b = fe.Host()
    b.load_params_text(text.replace("inPath =\n", f"inPath = {tmp_path}/\n").replace("inFile =\n", "inFile = RUN.40\n"))
    b.init(5)
    ib = b.inputs()
    assert b.gi("simTime_itRestart") == 40 and b.gi("simTime_it") == 40
    I = (Ellipsis, slice(3, -3), slice(3, -3), slice(3, -3))
    np.testing.assert_array_equal(b.array("topoPos", 1, True)[0, 3:-3, 3:-3], ta[0, 3:-3, 3:-3])
    np.testing.assert_allclose(ib["zPos"], ia["zPos"], rtol=1e-6)
    np.testing.assert_array_equal(ib["hydroFlds"][0][I], ia["hydroFlds"][0][I])
    for f in range(1, 5):
        np.testing.assert_allclose(ib["hydroFlds"][f][I], ia["hydroFlds"][f][I], rtol=2.5e-7, atol=1e-30)
    for f in range(2):
        np.testing.assert_allclose(ib["moist"][f][I], ia["moist"][f][I], rtol=2.5e-7, atol=1e-30)
    np.testing.assert_allclose(ib["sgstke"][0][I], ia["sgstke"][0][I], rtol=2.5e-7, atol=1e-30)
    for nm in ("tskin", "htFlux", "fricVel", "z0m"):
        np.testing.assert_array_equal(ib[nm][3:-3, 3:-3], ia[nm][3:-3, 3:-3])
        np.testing.assert_array_equal(ib[nm], np.pad(ib[nm][3:-3, 3:-3], 3, mode="wrap"))  # periodic halos
    b.cleanup()


def test_restart_rejects_a_mismatched_file(fe, tmp_path):
    a, text = _host(fe, "cbl_dry", {}, tmp_path)
    a.write_netcdf(str(tmp_path / "RUN.8"))
    a.cleanup()
    b = fe.Host()
    small = fe.cases.param_text("cbl_dry", 8, 6, 4).replace("outPath = ./output/", f"outPath = {tmp_path}/")
    b.load_params_text(small.replace("inPath =\n", f"inPath = {tmp_path}/\n").replace("inFile =\n", "inFile = RUN.8\n"))
    with pytest.raises(fe.FeError, match="parameters ask for"):
        b.init(5)


def test_restart_rejects_a_variable_in_another_dimension_order(fe, tmp_path):
    """A variable whose dimensions are not (time, zIndex, yIndex, xIndex) -- here u written as
    (time, xIndex, yIndex, zIndex) by scipy's independent writer -- is refused with a message, not
    read transposed into the state."""
    from scipy.io import netcdf_file

    a, text = _host(fe, "cbl_dry", {}, tmp_path)
    a.write_netcdf(str(tmp_path / "GOOD.8"))
    a.cleanup()
    with netcdf_file(str(tmp_path / "GOOD.8"), "r", mmap=False) as src, \
            netcdf_file(str(tmp_path / "BAD.8"), "w", version=2) as dst:
        for name, size in src.dimensions.items():
            dst.createDimension(name, size)
        for name, var in src.variables.items():
            dims = var.dimensions
            data = var.data.copy()
            if name == "u":
                dims = ("time", "xIndex", "yIndex", "zIndex")
                data = np.ascontiguousarray(data.transpose(0, 3, 2, 1))
            out = dst.createVariable(name, var.data.dtype, dims)
            out[:] = data
    b = fe.Host()
    b.load_params_text(text.replace("inPath =\n", f"inPath = {tmp_path}/\n").replace("inFile =\n", "inFile = BAD.8\n"))
    with pytest.raises(fe.FeError, match="dimension"):
        b.init(5)

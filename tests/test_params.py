"""Parameter-file reader: the reference's input format and query semantics
(SRC/PARAMETERS/parameters.c:81-200 parsing, :265-450 typed queries)."""
from __future__ import annotations

import pytest


def test_case_file_parses_with_no_unused_keys(fe):
    host = fe.Host()
    host.load_params_text(fe.cases.param_text("cbl_dry", 16, 12, 8))
    assert host.unused_params() == []
    assert host.gi("Nx") == 16 and host.gi("Ny") == 12 and host.gi("Nz") == 8
    assert host.gi("advectionSelector") == 3 and host.gi("TKESelector") == 1
    assert abs(host.gf("dt") - 0.025) < 1e-9
    # derived constants (hydro_core.c:941-967): f = 2*Omega*sin(lat) = 1e-4
    assert abs(host.gf("corioConstHorz") - 1e-4) < 1e-9
    assert abs(host.gf("cp_gas") - (287.04 + 718.0)) < 1e-3


def test_comments_blank_values_and_unused_keys(fe):
    host = fe.Host()
    text = fe.cases.param_text("cbl_dry", 8, 8, 8) + "\n# a comment line\nmyExtraKey = 3 # not a FastEddy key\n"
    host.load_params_text(text)
    assert host.unused_params() == ["myExtraKey"]


def test_duplicate_key_is_an_error(fe):
    host = fe.Host()
    with pytest.raises(fe.FeError):
        host.load_params_text(fe.cases.param_text("cbl_dry", 8, 8, 8) + "Nx = 9\n")


def test_missing_mandatory_key_is_an_error(fe):
    host = fe.Host()
    text = "\n".join(l for l in fe.cases.param_text("cbl_dry", 8, 8, 8).splitlines() if not l.startswith("d_zeta"))
    with pytest.raises(fe.FeError, match="d_zeta"):
        host.load_params_text(text)


def test_out_of_range_value_is_an_error(fe):
    host = fe.Host()
    text = fe.cases.param_text("cbl_dry", 8, 8, 8).replace("thetaAmplitude = 0.25", "thetaAmplitude = 5.0")
    with pytest.raises(fe.FeError, match="thetaAmplitude"):
        host.load_params_text(text)


def test_multi_rank_decomposition_rejected(fe):
    host = fe.Host()
    text = fe.cases.param_text("cbl_dry", 8, 8, 8).replace("numProcsX = 1", "numProcsX = 2")
    with pytest.raises(fe.FeError, match="numProcsX"):
        host.load_params_text(text)


def test_optional_key_keeps_default(fe):
    host = fe.Host()
    text = "\n".join(l for l in fe.cases.param_text("cbl_dry", 8, 8, 8).splitlines()
                     if not l.startswith("physics_oneRKonly"))
    host.load_params_text(text)
    assert host.gi("physics_oneRKonly") == 1


def test_parameter_file_on_disk(fe, tmp_path):
    p = tmp_path / "case.in"
    p.write_text(fe.cases.param_text("cbl_moist_hill", 8, 8, 8))
    host = fe.Host()
    host.load_params_file(str(p))
    assert host.gi("moistureSelector") == 1 and host.gi("moistureNvars") == 2
    with pytest.raises(fe.FeError):
        host.load_params_file(str(tmp_path / "missing.in"))

"""Checks against golden vectors produced by the reference's own CUDA build
(tests/golden/make_reference_golden.py, run on a B200 with oracle/_ref).

The CPU test pins the FP64 oracle to the reference's outputs; the GPU test checks the
engine against the same vectors. Tolerances: the reference computes in FP32, so its
state after one step differs from FP64 by FP32 rounding (see test_gpu_engine.py); the
reference's own run-to-run spread is stored with the vectors and added to the bound.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import ROOT, interior, rel_l2
from oracle.pyoracle import Oracle

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _load(name):
    import importlib.util

    spec = importlib.util.spec_from_file_location("mkgold", os.path.join(GOLDEN, "make_reference_golden.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    path = os.path.join(GOLDEN, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden vectors {path} not generated")
    return mk, np.load(path)


GOLDEN_CASES = ["cbl_dry", "moist_hill", "dry_quick_filter", "moist_weno3_filter", "dry_hyb34", "moist_centred_filter",
                "dry_upwind_filter", "moist_lsf", "dry_lsf_no_subsidence"]

TOL = {1: [1e-6, 1e-5, 2e-3, 2e-3, 1e-6], 10: [2e-6, 2e-5, 5e-3, 5e-3, 2e-6]}


def _compare(state, gold, n, spread):
    for f in range(5):
        ref = gold[f"hydro_{n}"][f]
        bound = TOL[n][f] + 4 * spread[f] / max(np.abs(ref).max(), 1e-30)
        assert rel_l2(interior(state["hydroFlds"][f]), ref) < bound, (n, f)
    # TKE and q_l: FP32 noise against the reference is ~3e-5; a wrong advection scheme for either
    # field moves it by 1e-3 to 1e-2 in 10 steps
    if f"tke_{n}" in gold:
        assert rel_l2(interior(state["sgstke"][0]), gold[f"tke_{n}"][0]) < 2e-4, (n, "tke")
    if f"moist_{n}" in gold:
        assert rel_l2(interior(state["moist"][0]), gold[f"moist_{n}"][0]) < 2e-6
        assert rel_l2(interior(state["moist"][1]), gold[f"moist_{n}"][1]) < 2e-4, (n, "q_l")


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_build(fe, name):
    mk, gold = _load(name)
    host, inp = mk.make_inputs(name)
    assert mk.input_digest(inp) == str(gold["input_sha256"]), "host layer changed the golden inputs"
    o = Oracle(host.config())
    o.set_inputs(inp)
    o.step(1)
    _compare(o.get_state(), gold, 1, gold["self_absdiff_1"])
    o.step(9)
    _compare(o.get_state(), gold, 10, gold["self_absdiff_10"])
    host.cleanup()


# Mistakes planted in the oracle (a scheme or the filter switched): each must fail the
# comparison with the reference build's vectors, so the vectors pin the option they exercise.
PLANTED = [("dry_quick_filter", "advectionSelector", 3), ("dry_quick_filter", "filterSelector", 0),
           ("moist_weno3_filter", "advectionSelector", 5), ("moist_weno3_filter", "moistureAdvSelectorQi", 2),
           ("dry_hyb34", "b_hyb", 0.0), ("dry_hyb34", "TKEAdvSelector", 3),
           ("moist_centred_filter", "moistureAdvSelectorQv", 3), ("moist_centred_filter", "filterSelector", 0),
           ("dry_upwind_filter", "TKEAdvSelector", 3), ("dry_upwind_filter", "advectionSelector", 1),
           ("moist_lsf", "lsfSelector", 0), ("moist_lsf", "lsf_horMnSubTerms", 0), ("moist_lsf", "lsf_freq", 0.075),
           ("dry_lsf_no_subsidence", "lsfSelector", 0), ("dry_lsf_no_subsidence", "lsf_freq", 0.075)]


@pytest.mark.parametrize("name,key,value", PLANTED)
def test_golden_vectors_reject_a_wrong_option(fe, name, key, value):
    mk, gold = _load(name)
    host, inp = mk.make_inputs(name)
    cfg = host.config()
    setattr(cfg, key, value)
    o = Oracle(cfg)
    o.set_inputs(inp)
    o.step(10)
    with pytest.raises(AssertionError):
        _compare(o.get_state(), gold, 10, gold["self_absdiff_10"])
    host.cleanup()


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_engine_matches_reference_build(fe, name):
    mk, gold = _load(name)
    host, inp = mk.make_inputs(name)
    assert mk.input_digest(inp) == str(gold["input_sha256"])
    d = fe.Domain(host.config())
    d.set_inputs(inp)
    d.advance(1)
    _compare(d.get_state(), gold, 1, gold["self_absdiff_1"])
    d.advance(9)
    _compare(d.get_state(), gold, 10, gold["self_absdiff_10"])
    d.close()
    host.cleanup()


# Tendencies of one evaluation per RK stage on the initial state (cases without large-scale
# forcing). Engine against reference: both FP32 with the same operator order, momentum
# tendencies agree to ~1e-6; the advected scalars' (a small divergence of large fluxes) to ~1e-4,
# because the reference forms its advective face values in double precision. The FP64 oracle
# against the reference: to the FP32 noise of the perturbation pressure and of the fluxes, 1e-3
# (2e-3 for the stresses), as the oracle tendency tests use. On flat terrain the mass tendency
# is zero up to rounding and is bounded in absolute terms.
FRHS_CASES = [c for c in GOLDEN_CASES if "lsf" not in c]


def _compare_frhs(g: dict, gold, stage: int, flat: bool, tight: bool) -> None:
    tm = 1e-5 if tight else 1e-3  # momentum
    tt = 1e-5 if tight else 2e-3  # stresses
    ref = gold[f"frhs_{stage}"]
    scale = np.abs(ref[4]).max() / 300.0  # the theta tendency's size in mass units
    for f in range(5):
        a = interior(g["hydroFrhs"][f]).astype(np.float64)
        if f == 0 and flat:
            assert np.abs(a - ref[0]).max() <= 1e-5 * scale + 1e-7, (stage, f)
        elif np.abs(ref[f]).max() > 0:
            assert rel_l2(a, ref[f]) < (1e-3 if f in (0, 4) else tm), (stage, f)
        else:
            assert np.abs(a).max() < 1e-6, (stage, f)
    if f"tkefrhs_{stage}" in gold and np.abs(gold[f"tkefrhs_{stage}"]).max() > 0:
        assert rel_l2(interior(g["sgstkeFrhs"][0]), gold[f"tkefrhs_{stage}"][0]) < 1e-3, (stage, "tke")
    if f"moistfrhs_{stage}" in gold:
        for m in range(gold[f"moistfrhs_{stage}"].shape[0]):
            r = gold[f"moistfrhs_{stage}"][m]
            if np.abs(r).max() > 0:
                assert rel_l2(interior(g["moistFrhs"][m]), r) < 1e-3, (stage, "moist", m)
    if stage == 2 and g.get("taus") is not None:
        for t in range(9):
            r = gold["taus_2"][t]
            if np.abs(r).max() > 0:
                assert rel_l2(interior(g["taus"][t]), r) < tt, ("tau", t)


@pytest.mark.parametrize("name", FRHS_CASES)
def test_oracle_tendency_matches_reference_build(fe, name):
    mk, gold = _load(name)
    if "frhs_0" not in gold:
        pytest.skip("golden vectors without tendencies")
    host, inp = mk.make_inputs(name)
    assert mk.input_digest(inp) == str(gold["input_sha256"])
    for stage in (0, 1, 2):
        o = Oracle(host.config())
        o.set_inputs(inp)
        _compare_frhs(o.build_frhs(stage), gold, stage, "hill" not in name, tight=False)
        o.close()
    host.cleanup()


@pytest.mark.gpu
@pytest.mark.parametrize("name", FRHS_CASES)
def test_engine_tendency_matches_reference_build(fe, name):
    mk, gold = _load(name)
    if "frhs_0" not in gold:
        pytest.skip("golden vectors without tendencies")
    host, inp = mk.make_inputs(name)
    assert mk.input_digest(inp) == str(gold["input_sha256"])
    for stage in (0, 1, 2):
        d = fe.Domain(host.config())
        d.set_inputs(inp)
        _compare_frhs(d.build_frhs(stage), gold, stage, "hill" not in name, tight=True)
        d.close()
    host.cleanup()

"""Generate the reference-build golden vectors in tests/golden (run on a GPU box).

Runs the reference's own CUDA build (oracle/_ref, built by oracle/build_ref.py) on small
seeded cases produced by the host layer and stores its prognostic state after 1 and 10
RK3 steps and (cases without large-scale forcing) its tendency of every RK stage on the
initial state with the SGS stresses of the physics stage, so the FP64 oracle and the engine
are checked against the reference's own outputs. The reference runs with a thread-block shape that divides the halo-inclusive
extents (no out-of-range threads), twice, and the run-to-run difference is stored too.

usage: python tests/golden/make_reference_golden.py OUTDIR [CASE ...]
"""
from __future__ import annotations

import hashlib
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
fe = importlib.import_module("fasteddy-model_b200")
from oracle import refrun  # noqa: E402

# BOMEX-shaped large-scale forcing with rates ~50 times the tutorial's, so that 10 steps of it move
# the state well beyond FP32 noise (the reference accepts rates up to 1e4 per hour)
LSF = dict(lsfSelector=1, lsf_horMnSubTerms=1, lsf_freq=0.05, lsf_w_surf=0.0, lsf_w_lev1=-2000.0, lsf_w_lev2=0.0,
           lsf_w_zlev1=50.0, lsf_w_zlev2=100.0, lsf_th_surf=-100.0, lsf_th_lev1=-50.0, lsf_th_lev2=25.0,
           lsf_th_zlev1=40.0, lsf_th_zlev2=90.0, lsf_qv_surf=-20.0, lsf_qv_lev1=-20.0, lsf_qv_lev2=0.0,
           lsf_qv_zlev1=30.0, lsf_qv_zlev2=70.0)
MOIST_HILL = dict(hill_halfwidth=60.0, hill_height=15.0, qv=(24.0, 8.0, 300.0))
CASES = {
    "cbl_dry": dict(case="cbl_dry", nx=16, ny=12, nz=12, kw={}),
    "moist_hill": dict(case="cbl_moist_hill", nx=16, ny=12, nz=12, kw=MOIST_HILL),
    # the other advection schemes and the explicit filter, by the reference's parameter keys
    "dry_quick_filter": dict(case="cbl_dry", nx=16, ny=12, nz=12,
                             kw=dict(params=dict(advectionSelector=1, TKEAdvSelector=2, TKEAdvSelector_b_hyb=0.5,
                                                 filterSelector=1, filter_6th_coeff=0.12))),
    "moist_weno3_filter": dict(case="cbl_moist_hill", nx=16, ny=12, nz=12,
                               kw=dict(MOIST_HILL, params=dict(advectionSelector=4, TKEAdvSelector=6,
                                                               moistureAdvSelectorQv=0, moistureAdvSelectorQi=1,
                                                               filterSelector=1))),
    "dry_hyb34": dict(case="cbl_dry", nx=16, ny=12, nz=12,
                      kw=dict(params=dict(advectionSelector=2, b_hyb=0.3, TKEAdvSelector=4))),
    "moist_centred_filter": dict(case="cbl_moist_hill", nx=16, ny=12, nz=12,
                                 kw=dict(MOIST_HILL, params=dict(advectionSelector=6, TKEAdvSelector=0,
                                                                 moistureAdvSelectorQv=1, moistureAdvSelectorQi=0,
                                                                 filterSelector=1, filter_6th_coeff=0.12))),
    "dry_upwind_filter": dict(case="cbl_dry", nx=16, ny=12, nz=12,
                              kw=dict(params=dict(advectionSelector=0, TKEAdvSelector=1, filterSelector=1,
                                                  filter_6th_coeff=0.12))),
    # large-scale forcing every 2 steps (BOMEX-type profiles scaled to the 120 m column); the
    # reference's slab-mean reduction tiles the halo-inclusive plane with 2 x 8 blocks, so the
    # plane is 22 x 16 columns here (ny = 10), and its subsidence terms need moisture on
    "moist_lsf": dict(case="cbl_moist_hill", nx=16, ny=10, nz=12,
                      kw=dict(MOIST_HILL, params=dict(LSF, filterSelector=1))),
    "dry_lsf_no_subsidence": dict(case="cbl_dry", nx=16, ny=10, nz=12,
                                  kw=dict(params=dict(LSF, lsf_horMnSubTerms=0, lsf_th_surf=-1000.0,
                                                      lsf_th_lev1=-500.0, lsf_th_lev2=250.0))),
}


def input_digest(inp: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(inp):
        if inp[k] is not None:
            h.update(k.encode())
            h.update(np.ascontiguousarray(inp[k], dtype=np.float32).tobytes())
    return h.hexdigest()


def make_inputs(name: str):
    c = CASES[name]
    host = fe.cases.setup_host(c["case"], c["nx"], c["ny"], c["nz"], **c["kw"])
    return host, host.inputs()


def main(out: str, names=None) -> None:
    os.makedirs(out, exist_ok=True)
    for name in names or list(CASES):
        c = CASES[name]
        host, inp = make_inputs(name)
        ntke, nm = host.nfields()
        text = fe.cases.param_text(c["case"], c["nx"], c["ny"], c["nz"], tb=fe.cases.exact_tb(c["ny"], c["nz"]),
                                   params=c["kw"].get("params"))
        res = {"input_sha256": np.array(input_digest(inp))}
        I = (Ellipsis, slice(3, -3), slice(3, -3), slice(3, -3))
        if not c["kw"].get("params", {}).get("lsfSelector"):
            # one tendency evaluation of every RK stage on the initial state, with the stresses of
            # the physics stage (the reference copies them back when these two switches are set)
            ftext = fe.cases.param_text(c["case"], c["nx"], c["ny"], c["nz"],
                                        tb=fe.cases.exact_tb(c["ny"], c["nz"]),
                                        params=dict(c["kw"].get("params") or {}, hydroForcingWrite=1,
                                                    hydroSubGridWrite=1))
            for stage in (0, 1, 2):
                r = refrun.frhs(ftext, inp, stage, host.shape, ntke, nm)
                res[f"frhs_{stage}"] = r["hydroFrhs"][I]
                if ntke:
                    res[f"tkefrhs_{stage}"] = r["sgstkeFrhs"][I]
                if nm:
                    res[f"moistfrhs_{stage}"] = r["moistFrhs"][I]
                if stage == 2:
                    res["taus_2"] = r["taus"][I]
        for n in (1, 10):
            a = refrun.run(text, inp, n, host.shape, ntke, nm)
            b = refrun.run(text, inp, n, host.shape, ntke, nm)
            res[f"hydro_{n}"] = a["hydroFlds"][I]
            res[f"self_absdiff_{n}"] = np.abs(a["hydroFlds"][I] - b["hydroFlds"][I]).max(axis=(1, 2, 3))
            if ntke:
                res[f"tke_{n}"] = a["sgstke"][I]
            if nm:
                res[f"moist_{n}"] = a["moist"][I]
        np.savez_compressed(os.path.join(out, f"ref_{name}.npz"), **res)
        print(name, {k: (v.shape if hasattr(v, "shape") else v) for k, v in res.items()}, flush=True)
        host.cleanup()


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"), sys.argv[2:] or None)

"""The allocation-free tendency entry point (fe_frhs_noalloc) against the engine's own
tendency evaluation (fe_build_frhs) and the FP64 oracle, through the C ABI.

fe_frhs_noalloc exists for callers that cannot allocate device memory -- allocators that own
all device memory, or embedders whose footprint is fixed after start-up. It keeps its scratch
in one static device array instead of calling cudaMalloc. It is a variant of the engine's
per-cell stage kernel, so it is compared against that kernel (FE_KERNEL_CELL), and against the FP64
oracle. This file is collected last so that a run stopping at the first failure has already run
every other test; it also passes alone.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import interior, rel_l2

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


NOALLOC_CASES = {
    "moist_hill": ("cbl_moist_hill", dict(hill_halfwidth=80.0, hill_height=20.0, qv=(24.0, 8.0, 300.0))),
    "cbl_dry": ("cbl_dry", {}),
}


@pytest.mark.parametrize("name", list(NOALLOC_CASES))
def test_noalloc_tendency_matches_engine_and_oracle_on_calls_in_a_row(fe, name):
    """Three calls in a row (stages 0, 1 and 2; the last runs the SGS and surface physics) on the
    same shared scratch: each equals the engine's tendency of the same stage to 1e-6 and the FP64
    oracle's to the tendency tolerance of the other GPU tests (1e-3; the mass tendency on flat
    terrain is zero up to rounding and is left out of the oracle comparison)."""
    import torch
    from oracle.pyoracle import Oracle

    case, kw = NOALLOC_CASES[name]
    host = fe.cases.setup_host(case, 20, 16, 14, **kw)
    inp, cfg = host.inputs(), host.config()
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    dom.set_stage_kernel("cell")
    st = dom.get_state()  # halo cells filled by the engine
    state = np.concatenate([a for a in (st["hydroFlds"], st["sgstke"], st["moist"]) if a is not None])
    zero2 = np.zeros_like(inp["z0m"])
    surface = np.stack([zero2, zero2, zero2, inp["fricVel"], inp["htFlux"], inp["tskin"], zero2, inp["z0m"],
                        inp["z0t"], inp["qFlux"], inp["qskin"]])
    torch.cuda.init()
    d = {k: _dev(torch, inp[k]) for k in ("zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac")}
    d["baseState"] = _dev(torch, inp["baseState"])
    d["state"] = _dev(torch, state)
    d["surface"] = _dev(torch, surface)
    d["frhs"] = torch.zeros_like(d["state"])
    args = fe.runtime.FeNoallocArgs(**{k: v.data_ptr() for k, v in d.items()})
    eng = fe.load()["engine"]
    assert state[0].size <= eng.fe_noalloc_max_cells()
    o = Oracle(cfg)
    o.set_inputs(inp)
    torch.cuda.synchronize()
    for stage in (0, 1, 2):
        rc = eng.fe_frhs_noalloc(ctypes.byref(cfg), stage, 0.0, 0, ctypes.byref(args), None)
        assert rc == 0, eng.fe_noalloc_last_error().decode()
        got = d["frhs"].cpu().numpy()
        ref = dom.build_frhs(stage)
        want = np.concatenate([a for a in (ref["hydroFrhs"], ref["sgstkeFrhs"], ref["moistFrhs"]) if a is not None])
        r = o.build_frhs(stage)
        exact = np.concatenate([a for a in (r["hydroFrhs"], r["sgstkeFrhs"], r["moistFrhs"]) if a is not None])
        for f in range(want.shape[0]):
            if np.abs(interior(want[f])).max() == 0.0:
                assert np.abs(interior(got[f])).max() == 0.0
            else:
                assert rel_l2(interior(got[f]), interior(want[f])) < 1e-6, (stage, f)
            if np.abs(interior(exact[f])).max() > 0.0 and not (f == 0 and name == "cbl_dry"):
                assert rel_l2(interior(got[f]), interior(exact[f])) < 1e-3, (stage, f)
    o.close()
    dom.close()
    host.cleanup()


def test_noalloc_rejects_domains_beyond_its_scratch(fe):
    import torch

    host = fe.cases.setup_host("cbl_dry", 120, 120, 60)
    cfg = host.config()
    host.cleanup()
    eng = fe.load()["engine"]
    assert 126 * 126 * 66 > eng.fe_noalloc_max_cells()
    t = torch.zeros(8, device="cuda")
    p = t.data_ptr()
    args = fe.runtime.FeNoallocArgs(**{k: p for k in ("zPos", "J31", "J32", "J33", "D_Jac", "invD_Jac", "baseState",
                                                       "state", "surface", "frhs")})
    rc = eng.fe_frhs_noalloc(ctypes.byref(cfg), 0, 0.0, 0, ctypes.byref(args), None)
    assert rc == 3  # FE_ERR_ARG
    assert b"exceeds" in eng.fe_noalloc_last_error()

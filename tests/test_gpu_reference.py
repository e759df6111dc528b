"""Parity with the reference's own CUDA build (oracle/_ref, compiled from the reference sources
for sm_100a) on identical inputs, per prognostic field, on the moist hill at a test size and on
two workloads at their full size: the 128x128x64 dry CBL and the 512x512x128 moist CBL over the
Gaussian hill.

1. One tendency evaluation of every RK stage on the same state (the reference's own
   cuda_hydroCoreDeviceBuildFrhs against fe_build_frhs), per field, and the SGS stresses.
   Momentum and TKE agree to <= 3e-7 (measured); the advected scalars rho, rho theta and rho q_v
   to <= 2e-4: the reference forms every HYB56 face value in double precision (its 37.0, 8.0, ...
   literals promote the stencil sums, cuda_advectionDevice.cu:365-376) and this engine in FP32,
   and the face values' last-bit difference shows in the divergence, a small difference of large
   fluxes. On flat terrain the mass tendency is zero up to rounding in both, and is checked in
   absolute terms.
2. The state after 1 and 100 RK3 steps, per field (rho, rho u, rho v, rho w, rho theta, rho e,
   rho q_v, rho q_l), relative L2 over the interior:
     1 step    <= 1e-5, or, for a field the reference itself moves by more than 4e-5 when its
               inputs change by one ulp (rho v and rho w: 2e-4..4e-4, measured here on every run),
               <= a quarter of that change. rho v and rho w come out 2e-5 from the reference: the
               rho theta tendency's rounding above (1e-4 relative) moves p' by ~1e-3 Pa.
     100 steps <= 1e-3, or 4x the reference's own run-to-run spread where that is larger (the
               reference is not deterministic: its Km reads the length scale of k-1 written by
               another thread, cuda_sgsTurbDevice.cu:236-237; 1.5e-3..2.2e-3 in rho v, rho w on
               the dry CBL).
   At the test size the FP64 oracle runs too: the engine is no farther from the reference
   than the reference is from the FP64 solution.

The reference runs with a thread-block shape that divides the halo-inclusive extents
(cases.exact_tb): with the tutorials' shape, threads past the last level of a column write p'
of the next column's boundary cells (cuda_pressureDevice.cu:70-77 has no upper k guard), a race
that changes rho w by 1e-1 between runs.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import interior, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ["rho", "rho_u", "rho_v", "rho_w", "rho_theta", "rho_e", "rho_qv", "rho_ql"]
CASES = {
    "moist_hill_48": ("cbl_moist_hill", 48, 40, 32, dict(hill_halfwidth=150.0, hill_height=30.0)),
    "dry_cbl_128": ("cbl_dry", 128, 128, 64, {}),
    "moist_hill_512": ("cbl_moist_hill", 512, 512, 128, {}),
}
FORCING = {"hydroForcingWrite": 1, "hydroSubGridWrite": 1}


def _fields(s: dict, tendency: bool = False) -> dict:
    h = s["hydroFrhs" if tendency else "hydroFlds"]
    out = {NAMES[f]: interior(h[f]) for f in range(5)}
    e = s.get("sgstkeFrhs" if tendency else "sgstke")
    if e is not None:
        out["rho_e"] = interior(e[0])
    m = s.get("moistFrhs" if tendency else "moist")
    if m is not None:
        for q in range(m.shape[0]):
            out[NAMES[6 + q]] = interior(m[q])
    return out


def _table(a: dict, b: dict, tendency: bool = False) -> dict:
    fa, fb = _fields(a, tendency), _fields(b, tendency)
    return {k: (0.0 if not np.abs(fb[k]).any() and not np.abs(fa[k]).any() else rel_l2(fa[k], fb[k])) for k in fb}


def _perturb_one_ulp(inp: dict, seed: int = 99) -> dict:
    """Every prognostic value moved by one ulp up or down (seeded)."""
    rng = np.random.default_rng(seed)
    out = dict(inp)
    for key in ("hydroFlds", "sgstke", "moist"):
        v = inp.get(key)
        if v is not None:
            up = rng.integers(0, 2, size=v.shape).astype(bool)
            out[key] = np.where(up, np.nextafter(v, np.float32(np.inf)), np.nextafter(v, np.float32(-np.inf)))
    return out


def _setup(fe, name: str, params: dict | None = None):
    case, nx, ny, nz, kw = CASES[name]
    host = fe.cases.setup_host(case, nx, ny, nz, **kw)
    text = fe.cases.param_text(case, nx, ny, nz, tb=fe.cases.exact_tb(ny, nz), params=params)
    return host, text


@pytest.fixture(scope="module")
def refrun():
    from oracle import refrun as rr

    if not rr.available():
        pytest.skip("reference build not present (python oracle/build_ref.py)")
    return rr


@pytest.mark.parametrize("name", list(CASES))
def test_tendency_of_every_stage_matches_reference_build(fe, refrun, name):
    host, text = _setup(fe, name, FORCING)
    inp, cfg = host.inputs(), host.config()
    ntke, nm = host.nfields()
    flat = "hill" not in name
    for stage in (0, 1, 2):
        d = fe.Domain(cfg)
        d.set_inputs(inp)
        ours = d.build_frhs(stage)
        ours.update(d.sgs_fluxes())
        d.close()
        ref = refrun.frhs(text, inp, stage, host.shape, ntke, nm)
        tab = _table(ours, ref, tendency=True)
        print(name, "stage", stage, {k: f"{v:.1e}" for k, v in tab.items()})
        for k, err in tab.items():
            if k == "rho" and flat:
                # zero up to rounding on flat terrain: absolute, against the theta tendency's scale
                fo, fr = _fields(ours, True), _fields(ref, True)
                scale = np.abs(fr["rho_theta"]).max() / 300.0
                assert np.abs(fo[k].astype(np.float64) - fr[k]).max() <= 1e-5 * scale + 1e-7, (stage, k)
            elif k in ("rho", "rho_theta", "rho_qv", "rho_ql"):
                assert err <= 1e-3, (stage, k, err)
            else:
                assert err <= 1e-5, (stage, k, err)
        if stage == 2:
            sl = (slice(3, -3), slice(3, -3), slice(3, -3))
            for t in range(9):
                assert rel_l2(ours["taus"][t][sl], ref["taus"][t][sl]) <= 1e-5, ("tau", t)
            if nm:
                for t in range(3 * nm):
                    if np.abs(ref["moistTaus"][t][sl]).any():
                        assert rel_l2(ours["moistTaus"][t][sl], ref["moistTaus"][t][sl]) <= 1e-5, ("moist tau", t)
    host.cleanup()


@pytest.mark.parametrize("name", list(CASES))
def test_state_after_1_and_100_steps_matches_reference_build(fe, refrun, name):
    host, text = _setup(fe, name)
    inp, cfg = host.inputs(), host.config()
    ntke, nm = host.nfields()
    pin = _perturb_one_ulp(inp)
    for nsteps in (1, 100):
        d = fe.Domain(cfg)
        d.set_inputs(inp)
        d.advance(nsteps)
        ours = d.get_state()
        assert d.nonfinite() == 0
        d.close()
        r1 = refrun.run(text, inp, nsteps, host.shape, ntke, nm)
        if nsteps == 1:
            spread = _table(refrun.run(text, pin, nsteps, host.shape, ntke, nm), r1)
        else:
            spread = _table(refrun.run(text, inp, nsteps, host.shape, ntke, nm), r1)
        tab = _table(ours, r1)
        print(name, nsteps, "steps: ours-vs-ref", {k: f"{v:.1e}" for k, v in tab.items()},
              "spread", {k: f"{v:.1e}" for k, v in spread.items()})
        for k, err in tab.items():
            if nsteps == 1:
                bound = max(1e-5, 0.25 * spread[k]) if spread[k] > 4e-5 else 1e-5
            else:
                bound = max(1e-3, 4 * spread[k])
            assert err <= bound, (name, nsteps, k, err, bound)
    host.cleanup()


def test_engine_no_farther_from_reference_than_reference_from_fp64(fe, refrun):
    """After one step of the test-size moist hill, per field: |engine - reference| <= max(1e-5,
    |reference - FP64 oracle|), and the engine's own distance from FP64 is within 2x the
    reference's."""
    from oracle.pyoracle import Oracle

    host, text = _setup(fe, "moist_hill_48")
    inp, cfg = host.inputs(), host.config()
    ntke, nm = host.nfields()
    d = fe.Domain(cfg)
    d.set_inputs(inp)
    d.advance(1)
    ours = d.get_state()
    d.close()
    ref = refrun.run(text, inp, 1, host.shape, ntke, nm)
    o = Oracle(cfg)
    o.set_inputs(inp)
    o.step(1)
    exact = o.get_state()
    o.close()
    t_or, t_rx, t_ox = _table(ours, ref), _table(ref, exact), _table(ours, exact)
    print({k: (f"{t_or[k]:.1e}", f"{t_rx[k]:.1e}", f"{t_ox[k]:.1e}") for k in t_or})
    for k in t_or:
        if k == "rho_ql":
            continue  # no condensation in one step of this case: zero in all three
        assert t_or[k] <= max(1e-5, t_rx[k]), k
        assert t_ox[k] <= max(1e-5, 2 * t_rx[k]), k
    host.cleanup()

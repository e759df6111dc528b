"""Parity of the CUDA path (through the C ABI) with the FP64 oracle, plus the engine's
own invariants: graph replay, drop-in entry points, ensembles, reductions, autotuner.

Tolerances. The device path evaluates in FP32 like the reference. The tendency of
momentum is a difference of FP32 perturbation pressures p' = p(rho theta) - p_BS with
|p| ~ 1e5 Pa (ulp 0.008 Pa); the theta tendency a divergence of fluxes of |rho theta|
~ 350. Both carry relative FP32 noise of order 1e-4 against the FP64 oracle on these
perturbation-driven cases, so tendencies are checked at relative L2 <= 1e-3 and
stresses at 2e-3. States after 1 and 10 steps are checked per field against their own
norm: rho, rho theta, rho q_v at 1e-6 (FP32 storage), rho u at 1e-5, and the small
fields rho v, rho w, rho e at 2e-3 (they start at or near zero, so their norm is small).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import interior, rel_l2
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

CASES = {
    "cbl_dry": dict(case="cbl_dry", nx=24, ny=20, nz=16, kw={}),
    "moist_hill": dict(case="cbl_moist_hill", nx=24, ny=20, nz=16,
                       kw=dict(hill_halfwidth=90.0, hill_height=20.0, qv=(24.0, 8.0, 300.0))),
    "hill_dry": dict(case="cbl_hill_dry", nx=20, ny=24, nz=16, kw=dict(hill_halfwidth=80.0, hill_height=25.0)),
}

STATE_TOL = [1e-6, 1e-5, 2e-3, 2e-3, 1e-6]


def _setup(fe, name, nx=None, ny=None, nz=None):
    c = CASES[name]
    host = fe.cases.setup_host(c["case"], nx or c["nx"], ny or c["ny"], nz or c["nz"], **c["kw"])
    return host, host.inputs(), host.config()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("stage", [0, 2])
def test_tendency_matches_oracle(fe, name, stage):
    host, inp, cfg = _setup(fe, name)
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    g = dom.build_frhs(stage)
    o = Oracle(cfg)
    o.set_inputs(inp)
    r = o.build_frhs(stage)
    for f in range(5):
        if np.abs(interior(r["hydroFrhs"][f])).max() == 0.0:
            assert np.abs(interior(g["hydroFrhs"][f])).max() < 1e-6
            continue
        assert rel_l2(interior(g["hydroFrhs"][f]), interior(r["hydroFrhs"][f])) < 1e-3, f
    if r["sgstkeFrhs"] is not None and stage == 2:
        assert rel_l2(interior(g["sgstkeFrhs"][0]), interior(r["sgstkeFrhs"][0])) < 1e-3
    if r["moistFrhs"] is not None:
        for m in range(r["moistFrhs"].shape[0]):
            if np.abs(interior(r["moistFrhs"][m])).max() > 0:
                assert rel_l2(interior(g["moistFrhs"][m]), interior(r["moistFrhs"][m])) < 1e-3, m
    if stage == 2:
        # SGS stresses on the interior + upper ring the divergence reads
        sl = (slice(3, -2), slice(3, -2), slice(3, -2))
        for t in range(9):
            assert rel_l2(g["taus"][t][sl], r["taus"][t][sl]) < 2e-3, t
        sg, so = dom.get_surface(), o.get_surface()
        for k in ("cd", "ch", "fricVel", "invOblen"):
            assert rel_l2(sg[k][3:-3, 3:-3], so[k][3:-3, 3:-3]) < 1e-4, k
    dom.close()
    host.cleanup()


@pytest.mark.parametrize("name", list(CASES))
def test_state_matches_oracle_after_1_and_10_steps(fe, name):
    host, inp, cfg = _setup(fe, name)
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    o = Oracle(cfg)
    o.set_inputs(inp)
    for n in (1, 9):
        dom.advance(n)
        o.step(n)
        g, r = dom.get_state(), o.get_state()
        for f in range(5):
            assert rel_l2(interior(g["hydroFlds"][f]), interior(r["hydroFlds"][f])) < STATE_TOL[f], (n, f)
        if r["sgstke"] is not None:
            assert rel_l2(interior(g["sgstke"][0]), interior(r["sgstke"][0])) < 2e-3
        if r["moist"] is not None:
            assert rel_l2(interior(g["moist"][0]), interior(r["moist"][0])) < 1e-6
            if np.abs(interior(r["moist"][1])).max() > 0:
                assert rel_l2(interior(g["moist"][1]), interior(r["moist"][1])) < 2e-3
        assert dom.nonfinite() == 0
    if name == "moist_hill":
        assert np.abs(interior(r["moist"][1])).max() > 0  # condensation happened
    dom.close()
    host.cleanup()


def test_error_table_against_the_fp64_oracle(fe):
    """Error of the FP32 device path against the FP64 oracle after 1, 10 and 100 steps on the
    moist hill case: relative L2 of every prognostic field and of the perturbations the
    solution is about (theta' = rho theta / rho - theta_BS and p'). Prints the table (pytest -s);
    the bounds are the ones the design states for FP32 storage with the stage sums rounded
    once from double (stages 1-2) or fused (stage 3)."""
    host, inp, cfg = _setup(fe, "moist_hill")
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    o = Oracle(cfg)
    o.set_inputs(inp)
    base = inp["baseState"].astype(np.float64)
    th_bs = interior(base[1] / base[0])
    names = ["rho", "rho u", "rho v", "rho w", "rho theta", "rho e", "rho qv", "rho ql"]
    rows, done = [], 0
    for n in (1, 10, 100):
        dom.advance(n - done)
        o.step(n - done)
        done = n
        g, r = dom.get_state(), o.get_state()
        gf = np.concatenate([g["hydroFlds"], g["sgstke"], g["moist"]])
        rf = np.concatenate([r["hydroFlds"], r["sgstke"], r["moist"]])
        errs = [rel_l2(interior(gf[f]), interior(rf[f])) for f in range(gf.shape[0])]
        thp_g = interior(gf[4].astype(np.float64) / gf[0]) - th_bs
        thp_r = interior(rf[4].astype(np.float64) / rf[0]) - th_bs
        errs.append(rel_l2(thp_g, thp_r))
        errs.append(rel_l2(interior(g["pres"]), interior(r["pres"])))
        rows.append((n, errs))
    print("\nsteps  " + "  ".join(f"{h:>9s}" for h in names + ["theta'", "p'"]))
    for n, e in rows:
        print(f"{n:5d}  " + "  ".join(f"{v:9.2e}" for v in e))
    e1, e10, e100 = (r[1] for r in rows)
    assert e100[0] < 1e-5 and e100[4] < 1e-5        # rho, rho theta
    assert e100[8] < 2e-2                           # theta' (perturbation of ~0.25 K)
    assert e10[9] < 2e-2 and e100[9] < 5e-2          # p'
    dom.close()
    o.close()
    host.cleanup()


def test_graph_replay_equals_step_by_step(fe):
    host, inp, cfg = _setup(fe, "moist_hill")
    a = fe.Domain(cfg)
    a.set_inputs(inp)
    a.advance(8)  # one captured 8-step graph
    b = fe.Domain(cfg)
    b.set_inputs(inp)
    for _ in range(8):
        b.advance(1)  # eager launches
    sa, sb = a.get_state(), b.get_state()
    for k in ("hydroFlds", "sgstke", "moist"):
        np.testing.assert_array_equal(interior(sa[k]), interior(sb[k]))
    a.close()
    b.close()
    host.cleanup()


def test_tiling_and_autotune_do_not_change_results(fe):
    """March shapes give identical bits (every inlined copy of the flux arithmetic rounds
    explicitly); the cell kernel agrees to FP32 rounding (per-field state tolerances)."""
    host, inp, cfg = _setup(fe, "cbl_dry")
    a = fe.Domain(cfg)
    a.set_inputs(inp)
    kind, tj, ni = a.stage_kernel()  # default: tiles of 8 rows, planes per block chosen for the size
    assert (kind, tj) == ("march", 8) and ni in (8, 16, 32, 64)
    a.advance(3)
    b = fe.Domain(cfg)
    b.set_inputs(inp)
    kind, tj, ni = b.autotune()
    assert kind in ("march", "cell")
    b.set_inputs(inp)
    b.set_stage_kernel("march", 4, 5)
    b.advance(3)
    np.testing.assert_array_equal(interior(a.get_state()["hydroFlds"]), interior(b.get_state()["hydroFlds"]))
    c = fe.Domain(cfg)
    c.set_inputs(inp)
    c.set_stage_kernel("cell")
    c.set_tiling(32, 8, 1)
    c.advance(3)
    sa, sc = a.get_state(), c.get_state()
    for f in range(5):
        assert rel_l2(interior(sc["hydroFlds"][f]), interior(sa["hydroFlds"][f])) < STATE_TOL[f]
    for d in (a, b, c):
        d.close()
    host.cleanup()


@pytest.mark.parametrize("case", ["cbl_dry", "moist_hill", "hill_dry"])
def test_march_matches_cell_kernel_on_ragged_tiles(fe, case):
    """Domain extents that are not multiples of the tile (k: 32, j: 8 or 4, i: ni) -- the
    ring, halo and partial-tile paths of the march kernel -- against the cell kernel.

    The two kernels sum the same flux differences in different orders, so they agree to FP32
    rounding of the fluxes, not of the (often much smaller) tendency: each tendency field is
    checked to 1e-4 of its own maximum plus 1e-6 of the largest tendency of its block; states
    and halos after 4 steps to the per-field tolerances used against the FP64 oracle."""
    host, inp, cfg = _setup(fe, case, nx=37, ny=13, nz=45)
    ref = fe.Domain(cfg)
    ref.set_inputs(inp)
    ref.set_stage_kernel("cell")
    ref2 = fe.Domain(cfg)
    ref2.set_inputs(inp)
    ref2.set_stage_kernel("cell")
    ref2.advance(4)
    s2 = ref2.get_state()
    for tj, ni in ((8, 16), (4, 7)):
        d = fe.Domain(cfg)
        d.set_inputs(inp)
        d.set_stage_kernel("march", tj, ni)
        for stage in (0, 2):
            fr, fd = ref.build_frhs(stage), d.build_frhs(stage)
            for key in ("hydroFrhs", "sgstkeFrhs", "moistFrhs"):
                if fr.get(key) is None:
                    continue
                big = max(float(np.abs(interior(fr[key][f])).max()) for f in range(fr[key].shape[0]))
                for f in range(fr[key].shape[0]):
                    a_, b_ = interior(fd[key][f]), interior(fr[key][f])
                    tol = 1e-4 * float(np.abs(b_).max()) + 1e-6 * big
                    assert np.abs(a_ - b_).max() <= tol, (key, f, stage, tj, ni)
        d.advance(4)
        s1 = d.get_state()
        for f in range(5):
            assert rel_l2(s1["hydroFlds"][f], s2["hydroFlds"][f]) < STATE_TOL[f], ("hydro", f, tj, ni)
        for key in ("sgstke", "moist"):
            if s1.get(key) is not None:
                for f in range(s1[key].shape[0]):
                    assert rel_l2(s1[key][f], s2[key][f]) < 2e-3, (key, f, tj, ni)
        # p' = (c rho theta)^(cp/cv) - p_BS: a few ulps of rho theta move it by ~0.01 Pa
        np.testing.assert_allclose(s1["pres"], s2["pres"], rtol=0, atol=0.1)
        d.close()
    ref.close()
    ref2.close()
    host.cleanup()


@pytest.mark.parametrize("name", ["moist_hill", "cbl_dry", "moist_hill_lsf"])
def test_checkpoint_resume_is_bit_identical(fe, name):
    """16 steps in one go against 8 steps, checkpoint, a fresh domain, resume, 8 steps: state,
    pressure, surface planes and clock agree bit for bit (the graph path on both sides). With
    large-scale forcing every 2 steps the checkpoint also carries the buffer whose halo cells the
    next step's slab means read."""
    if name == "moist_hill_lsf":
        c = CASES["moist_hill"]
        host = fe.cases.setup_host(c["case"], c["nx"], c["ny"], c["nz"], params=LSF, **c["kw"])
        inp, cfg = host.inputs(), host.config()
    else:
        host, inp, cfg = _setup(fe, name)
    a = fe.Domain(cfg)
    a.set_inputs(inp)
    a.advance(16)
    b = fe.Domain(cfg)
    b.set_inputs(inp)
    b.advance(8)
    blob = b.checkpoint()
    b.close()
    c = fe.Domain(cfg)
    c.set_inputs(inp)  # grid, base state (the state is replaced by the checkpoint)
    c.restore(blob)
    c.advance(8)
    sa, sc = a.get_state(), c.get_state()
    for k in ("hydroFlds", "sgstke", "moist", "pres"):
        if sa[k] is not None:
            np.testing.assert_array_equal(sa[k], sc[k])
    for k, v in a.get_surface().items():
        np.testing.assert_array_equal(v, c.get_surface()[k])
    assert a.clock() == c.clock()
    bad = bytearray(blob)
    bad[0:8] = b"XXXXXXXX"
    with pytest.raises(fe.FeError):
        c.restore(bytes(bad))
    if name == "moist_hill_lsf":
        # a checkpoint with the subsidence buffer does not load into a domain without subsidence
        cfg.lsf_horMnSubTerms = 0
        e = fe.Domain(cfg)
        e.set_inputs(inp)
        with pytest.raises(fe.FeError, match="subsidence"):
            e.restore(blob)
        e.close()
    a.close()
    c.close()
    host.cleanup()


def test_dropin_entry_points_match_engine(fe):
    """cuda_gridInit/..../cuda_timeIntCommence on the host globals == engine API."""
    host, inp, cfg = _setup(fe, "moist_hill")
    libs = fe.load()
    ra = libs["refabi"]
    host.set_gi("NtBatch", 5)
    for fn in ("fecuda_Init", "cuda_gridInit", "cuda_hydroCoreInit", "cuda_timeIntInit"):
        assert getattr(ra, fn)() == 0, fn
    assert ra.fecuda_SetBlocksPerGrid(*host.shape) == 0
    assert ra.cuda_timeIntCommence(0) == 0
    assert host.gi("simTime_it") == 5
    ref_h = host.array("hydroFlds", 5).copy()
    ref_m = host.array("moistScalars", 2).copy()
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    dom.advance(5)
    s = dom.get_state()
    np.testing.assert_array_equal(interior(ref_h), interior(s["hydroFlds"]))
    np.testing.assert_array_equal(interior(ref_m), interior(s["moist"]))
    # a second batch continues from the device state (no re-upload when it != restart step)
    assert ra.cuda_timeIntCommence(5) == 0
    dom.advance(5)
    np.testing.assert_array_equal(interior(host.array("hydroFlds", 5)), interior(dom.get_state()["hydroFlds"]))
    # the device-level tendency twin fills the host Frhs arrays
    assert ra.cuda_hydroCoreDeviceBuildFrhs(0.0, 0, 0, host.gf("dt"), 0, 2) == 0
    assert np.abs(interior(host.array("hydroFldsFrhs", 5)[3])).max() > 0
    for fn in ("cuda_timeIntCleanup", "cuda_hydroCoreCleanup", "cuda_gridCleanup", "fecuda_Cleanup"):
        assert getattr(ra, fn)() == 0
    dom.close()
    host.cleanup()


@pytest.mark.parametrize("name", ["moist_hill", "cbl_dry"])
def test_kept_last_stage_tendencies_match_oracle(fe, name):
    """With tendency capture on, an advance keeps the last RK stage's tendencies of its last step
    (what the reference holds in its Frhs arrays after a batch, cuda_timeIntDevice.cu:210-224):
    after 1 and 3 steps they match the FP64 oracle's last-stage tendencies after the same steps;
    the state is the same as without capture, bit for bit."""
    from oracle.pyoracle import Oracle

    host, inp, cfg = _setup(fe, name)
    d = fe.Domain(cfg)
    d.set_inputs(inp)
    d.set_forcing_capture(True)
    plain = fe.Domain(cfg)
    plain.set_inputs(inp)
    o = Oracle(cfg)
    o.set_inputs(inp)
    for n in (1, 2):
        d.advance(n)
        plain.advance(n)
        o.step(n)
        g, r = d.last_forcing(), o.last_frhs()
        for f in range(5):
            if f == 0 and name == "cbl_dry":
                continue  # the mass tendency on flat terrain: zero up to rounding in FP32
            assert rel_l2(interior(g["hydroFrhs"][f]), interior(r["hydroFrhs"][f])) < 2e-3, (n, f)
        assert rel_l2(interior(g["sgstkeFrhs"][0]), interior(r["sgstkeFrhs"][0])) < 2e-3
        if r["moistFrhs"] is not None:
            assert rel_l2(interior(g["moistFrhs"][0]), interior(r["moistFrhs"][0])) < 2e-3
        for k in ("hydroFlds", "sgstke", "moist"):
            if plain.get_state()[k] is not None:
                np.testing.assert_array_equal(d.get_state()[k], plain.get_state()[k])
    d.close()
    plain.close()
    host.cleanup()


def test_dropin_batch_copies_back_tendencies_and_sgs_fluxes(fe):
    """With hydroForcingWrite and hydroSubGridWrite set, cuda_timeIntCommence copies back the last
    stage's tendencies (hydroFldsFrhs, sgstkeScalarsFrhs, moistScalarsFrhs) and the SGS stresses and
    moisture fluxes (hydroTauFlds, moistTauFlds), as cuda_timeIntDevice.cu:210-251 does: they equal
    the engine's own after the same steps."""
    host, inp, cfg = _setup(fe, "moist_hill")
    libs = fe.load()
    ra = libs["refabi"]
    host.set_gi("NtBatch", 3)
    host.set_gi("hydroForcingWrite", 1)
    host.set_gi("hydroSubGridWrite", 1)
    for fn in ("fecuda_Init", "cuda_gridInit", "cuda_hydroCoreInit", "cuda_timeIntInit"):
        assert getattr(ra, fn)() == 0, fn
    assert ra.cuda_timeIntCommence(0) == 0
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    dom.set_forcing_capture(True)
    dom.advance(3)
    lf = dom.last_forcing()
    np.testing.assert_array_equal(interior(host.array("hydroFldsFrhs", 5)), interior(lf["hydroFrhs"]))
    np.testing.assert_array_equal(interior(host.array("sgstkeScalarsFrhs", 1)), interior(lf["sgstkeFrhs"]))
    np.testing.assert_array_equal(interior(host.array("moistScalarsFrhs", 2)), interior(lf["moistFrhs"]))
    np.testing.assert_array_equal(interior(host.array("hydroTauFlds", 9)), interior(lf["taus"]))
    np.testing.assert_array_equal(interior(host.array("moistTauFlds", 6)), interior(lf["moistTaus"]))
    assert np.abs(interior(lf["hydroFrhs"][3])).max() > 0 and np.abs(interior(lf["taus"][0])).max() > 0
    assert ra.cuda_hydroCoreCleanup() == 0
    dom.close()
    host.cleanup()


@pytest.mark.parametrize("name", list(CASES) + ["bomex"])
def test_fused_sgs_kernel_equals_kernel_chain(fe, name):
    """The last stage's SGS physics as one fused kernel (the default with the march stage kernel)
    and as the kernel chain (closure into scratch fields, then the tendencies): the same state after
    10 steps bit for bit, and the same tendencies and stresses of a physics stage."""
    if name == "bomex":
        host = fe.cases.setup_host("bomex", 24, 20, 16)
        inp, cfg = host.inputs(), host.config()
    else:
        host, inp, cfg = _setup(fe, name, nx=37, ny=13, nz=45)  # ragged tiles
    a = fe.Domain(cfg)
    a.set_inputs(inp)
    b = fe.Domain(cfg)
    b.set_inputs(inp)
    b.set_sgs_kernel(0)
    c = fe.Domain(cfg)
    c.set_inputs(inp)
    c.set_sgs_kernel(16)
    fa, fb, fc = a.build_frhs(2), b.build_frhs(2), c.build_frhs(2)
    for key in ("hydroFrhs", "sgstkeFrhs", "moistFrhs", "taus"):
        if fa.get(key) is not None:
            np.testing.assert_array_equal(interior(fa[key]), interior(fb[key]), err_msg=key)
            np.testing.assert_array_equal(interior(fc[key]), interior(fb[key]), err_msg=key)
    for dom in (a, b, c):
        dom.advance(10)
    sa, sb, sc = a.get_state(), b.get_state(), c.get_state()
    for key in ("hydroFlds", "sgstke", "moist"):
        if sa.get(key) is not None:
            np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
            np.testing.assert_array_equal(sc[key], sb[key], err_msg=key)
    for dom in (a, b, c):
        dom.close()
    host.cleanup()


def test_nonfinite_state_is_reported(fe):
    host, inp, cfg = _setup(fe, "cbl_dry")
    libs = fe.load()
    ra = libs["refabi"]
    host.array("hydroFlds", 5)[4, 10, 10, 8] = np.nan
    host.set_gi("NtBatch", 1)
    assert ra.fecuda_Init() == 0 and ra.cuda_gridInit() == 0 and ra.cuda_hydroCoreInit() == 0
    assert ra.cuda_timeIntInit() == 0
    assert ra.cuda_timeIntCommence(0) == 6  # FE_ERR_NONFINITE
    ra.cuda_hydroCoreCleanup()
    host.cleanup()


def test_fp64_domain_means(fe):
    host, inp, cfg = _setup(fe, "moist_hill")
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    dom.advance(2)
    s = dom.get_state()
    m = dom.means()
    fields = [s["hydroFlds"][f] for f in range(5)] + [s["sgstke"][0]] + [s["moist"][k] for k in range(2)]
    for f, a in enumerate(fields):
        np.testing.assert_allclose(m[f], interior(a).astype(np.float64).mean(), rtol=1e-12, atol=1e-300)
    dom.close()
    host.cleanup()


@pytest.mark.parametrize("batched", [True, False])
def test_ensemble_of_uneven_domains_matches_members(fe, batched):
    """Uneven neutral-ABL members advanced together -- as work-list launches over all members'
    tiles, or as one graph branch per member -- equal the members advanced alone, bit for bit."""
    shapes = [(16, 12, 10), (20, 16, 12), (12, 20, 14), (37, 13, 45)]
    hosts, inps, cfgs = [], [], []
    for i, (nx, ny, nz) in enumerate(shapes):
        h = fe.cases.setup_host("abl_neutral", nx, ny, nz, seed=100 + i, ug=5.0 + 2 * i)
        inps.append(h.inputs())
        cfgs.append(h.config())
        h.cleanup()
    members = []
    for cfg, inp in zip(cfgs, inps):
        d = fe.Domain(cfg)
        d.set_inputs(inp)
        members.append(d)
    members[1].set_stage_kernel("march", 8, 5)  # a member with its own march shape (same bits)
    ens = fe.Ensemble(members)
    ens.set_batched(batched)
    ens.advance(11)  # one 8-step graph + 3 eager steps
    assert ens.batched() == batched
    for cfg, inp, d in zip(cfgs, inps, members):
        solo = fe.Domain(cfg)
        solo.set_inputs(inp)
        solo.advance(11)
        np.testing.assert_array_equal(interior(d.get_state()["hydroFlds"]), interior(solo.get_state()["hydroFlds"]))
        solo.close()
    # without a host synchronisation, a member's own stream (its state copy) waits for the ensemble
    ens.advance(16, sync=False)
    for cfg, inp, d in zip(cfgs, inps, members):
        solo = fe.Domain(cfg)
        solo.set_inputs(inp)
        solo.advance(27)
        np.testing.assert_array_equal(interior(d.get_state()["hydroFlds"]), interior(solo.get_state()["hydroFlds"]))
        solo.close()
    ens.close()
    for d in members:
        d.close()


def test_unsupported_configuration_is_rejected(fe):
    host, inp, cfg = _setup(fe, "cbl_dry")
    for key, value, msg in (("advectionSelector", 7, "advectionSelector"), ("diffusionSelector", 1, "diffusion"),
                            ("lsfSelector", 2, "lsfSelector"), ("filterSelector", 2, "filterSelector")):
        bad = type(cfg).from_buffer_copy(cfg)
        setattr(bad, key, value)
        with pytest.raises(fe.FeError, match=msg):
            fe.Domain(bad)
    host.cleanup()


# The other advection schemes (upwind, QUICK, HYB34, WENO3, centred 2nd) on every advected field
# and the explicit 6th-order filter of rho w, by the reference's own parameter keys. The last two
# cases keep the default schemes (but q_v's, in the last) and add the filter, so the compile-time
# moist forms of the march kernel carry it.
SCHEME_CASES = {
    "dry_quick_upwind_filter": ("cbl_dry", dict(advectionSelector=1, TKEAdvSelector=0, filterSelector=1)),
    "dry_hyb34_centred_filter": ("cbl_dry", dict(advectionSelector=2, b_hyb=0.4, TKEAdvSelector=6, filterSelector=1,
                                                 filter_6th_coeff=0.12)),
    "hill_weno3_quick": ("hill_dry", dict(advectionSelector=4, TKEAdvSelector=1, filterSelector=1)),
    "moist_centred_weno3": ("moist_hill", dict(advectionSelector=6, TKEAdvSelector=4, moistureAdvSelectorQv=2,
                                               moistureAdvSelectorQv_b=0.3, moistureAdvSelectorQi=1, filterSelector=1)),
    "moist_upwind_quick": ("moist_hill", dict(advectionSelector=0, TKEAdvSelector=2, TKEAdvSelector_b_hyb=0.5,
                                              moistureAdvSelectorQv=1, moistureAdvSelectorQi=0)),
    "moist_default_filter": ("moist_hill", dict(filterSelector=1, filter_6th_coeff=0.12)),
    # HYB34 for q_v with the other schemes at their defaults: the compile-time moist form with
    # q_v's scheme fixed to HYB34 (the BOMEX tutorial's selectors)
    "moist_hyb34_qv_filter": ("moist_hill", dict(moistureAdvSelectorQv=2, moistureAdvSelectorQv_b=0.2, filterSelector=1)),
}


def _scheme_setup(fe, name):
    base, params = SCHEME_CASES[name]
    c = CASES[base]
    host = fe.cases.setup_host(c["case"], c["nx"], c["ny"], c["nz"], params=params, **c["kw"])
    return host, host.inputs(), host.config()


@pytest.mark.parametrize("name", list(SCHEME_CASES))
def test_advection_schemes_and_filter_match_oracle(fe, name):
    """Stage tendencies of both kernel forms (stages 1 and 3) and the state after 4 steps
    against the FP64 oracle, at the tolerances of the default schemes."""
    host, inp, cfg = _scheme_setup(fe, name)
    o = Oracle(cfg)
    o.set_inputs(inp)
    ref = {stage: o.build_frhs(stage) for stage in (0, 2)}
    for kind in ("march", "cell"):
        dom = fe.Domain(cfg)
        dom.set_inputs(inp)
        dom.set_stage_kernel(kind, 8 if kind == "march" else 0, 0)
        for stage in (0, 2):
            g, r = dom.build_frhs(stage), ref[stage]
            for f in range(5):
                if np.abs(interior(r["hydroFrhs"][f])).max() == 0.0:
                    assert np.abs(interior(g["hydroFrhs"][f])).max() < 1e-6
                    continue
                assert rel_l2(interior(g["hydroFrhs"][f]), interior(r["hydroFrhs"][f])) < 1e-3, (kind, stage, f)
            if r["sgstkeFrhs"] is not None and stage == 2:
                assert rel_l2(interior(g["sgstkeFrhs"][0]), interior(r["sgstkeFrhs"][0])) < 1e-3, kind
            if r["moistFrhs"] is not None:
                for m in range(r["moistFrhs"].shape[0]):
                    if np.abs(interior(r["moistFrhs"][m])).max() > 0:
                        assert rel_l2(interior(g["moistFrhs"][m]), interior(r["moistFrhs"][m])) < 1e-3, (kind, stage, m)
        dom.close()
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    dom.advance(4)
    o.step(4)
    g, r = dom.get_state(), o.get_state()
    for f in range(5):
        assert rel_l2(interior(g["hydroFlds"][f]), interior(r["hydroFlds"][f])) < STATE_TOL[f], f
    if r["sgstke"] is not None:
        assert rel_l2(interior(g["sgstke"][0]), interior(r["sgstke"][0])) < 2e-3
    if r["moist"] is not None:
        assert rel_l2(interior(g["moist"][0]), interior(r["moist"][0])) < 1e-6
        if np.abs(interior(r["moist"][1])).max() > 0:
            assert rel_l2(interior(g["moist"][1]), interior(r["moist"][1])) < 2e-3
    assert dom.nonfinite() == 0
    dom.close()
    host.cleanup()


def test_filter_changes_only_rho_w(fe):
    """With the filter on, the engine's tendency differs from the unfiltered one in rho w only,
    by the oracle's filter term. The initial state is at rest in w, so the comparison starts from
    the state after 20 steps."""
    host, inp, cfg = _scheme_setup(fe, "moist_default_filter")
    d = fe.Domain(cfg)
    d.set_inputs(inp)
    d.advance(20)
    st = d.get_state()
    d.close()
    inp = dict(inp, hydroFlds=st["hydroFlds"], sgstke=st["sgstke"], moist=st["moist"])
    out = {}
    for filt in (0, 1):
        cfg.filterSelector = filt
        d = fe.Domain(cfg)
        d.set_inputs(inp)
        o = Oracle(cfg)
        o.set_inputs(inp)
        out[filt] = (d.build_frhs(0)["hydroFrhs"], o.build_frhs(0)["hydroFrhs"])
        d.close()
    for f in (0, 1, 2, 4):
        np.testing.assert_array_equal(interior(out[1][0][f]), interior(out[0][0][f]))
    dg = interior(out[1][0][3]).astype(np.float64) - interior(out[0][0][3])
    dr = interior(out[1][1][3]) - interior(out[0][1][3])
    assert np.abs(dr).max() > 0
    assert rel_l2(dg, dr) < 1e-3
    host.cleanup()


# Large-scale forcing as in the BOMEX tutorial (theta and q_v forcing, subsidence of the slab-mean
# u, v, theta, q_v), heights scaled to the 160 m test column, applied every 2 steps. The subsidence
# rate is 200 times BOMEX's so that its term on rho u (otherwise ~1e-5 against O(1) tendencies)
# is resolved by the difference of two FP32 tendencies.
LSF = dict(lsfSelector=1, lsf_horMnSubTerms=1, lsf_freq=0.05, lsf_w_surf=0.0, lsf_w_lev1=-8000.0, lsf_w_lev2=0.0,
           lsf_w_zlev1=60.0, lsf_w_zlev2=120.0, lsf_th_surf=-2.0, lsf_th_lev1=-1.0, lsf_th_lev2=0.5,
           lsf_th_zlev1=50.0, lsf_th_zlev2=110.0, lsf_qv_surf=-0.5, lsf_qv_lev1=-0.5, lsf_qv_lev2=0.0,
           lsf_qv_zlev1=40.0, lsf_qv_zlev2=90.0)


@pytest.mark.parametrize("kind", ["march", "cell"])
def test_large_scale_forcing_matches_oracle(fe, kind):
    """The forcing's own tendency (last stage on a forcing step, with minus without) from the
    state after 8 steps, and the state after 6 forced steps (forcing at steps 2 and 4; the slab
    means taken at their start from phi^n inside and the previous phi** in the halo cells).

    The forcing is small against the O(1) tendencies it is added to, so the engine's value of it
    (the difference of two FP32 tendencies that share every other term) is known to a few ulps of
    those tendencies: each cell is checked to 4 ulps of the larger tendency plus 1e-4 of the
    largest forcing term. The subsidence terms are checked on u and v. On theta (and q_v) the
    reference's formula differences two FP32 slab-mean ratios <rho theta>/<rho> ~ 300 across two
    levels, which carries ~1e-7 relative noise of theta itself; there the theta and q_v forcing is
    checked without subsidence, and the subsidence through the forced state below."""
    c = CASES["moist_hill"]
    host = fe.cases.setup_host(c["case"], c["nx"], c["ny"], c["nz"], params=LSF, **c["kw"])
    inp, cfg = host.inputs(), host.config()
    d = fe.Domain(cfg)
    d.set_inputs(inp)
    d.advance(8)
    st = d.get_state()
    d.close()
    moved = dict(inp, hydroFlds=st["hydroFlds"], sgstke=st["sgstke"], moist=st["moist"])
    for sub, checks in ((1, (("hydroFrhs", 1), ("hydroFrhs", 2))), (0, (("hydroFrhs", 4), ("moistFrhs", 0)))):
        cfg.lsf_horMnSubTerms = sub
        diff = {}
        for on in (0, 1):
            cfg.lsfSelector = on
            dom = fe.Domain(cfg)
            dom.set_inputs(moved, 0.2, 8)
            dom.set_stage_kernel(kind, 8 if kind == "march" else 0, 0)
            o = Oracle(cfg)
            o.set_inputs(moved, 0.2, 8)
            diff[on] = (dom.build_frhs(2), o.build_frhs(2))
            dom.close()
        for key, f in checks:
            on, off = interior(diff[1][0][key][f]), interior(diff[0][0][key][f])
            dg = on.astype(np.float64) - off
            dr = interior(diff[1][1][key][f]) - interior(diff[0][1][key][f])
            assert np.abs(dr).max() > 0, (key, f)
            tol = 4 * np.spacing(np.maximum(np.abs(on), np.abs(off))) + 1e-4 * np.abs(dr).max()
            assert (np.abs(dg - dr) <= tol).all(), (kind, sub, key, f, float((np.abs(dg - dr) / tol).max()))
    cfg.lsf_horMnSubTerms = 1
    cfg.lsfSelector = 1
    dom = fe.Domain(cfg)
    dom.set_inputs(inp)
    dom.set_stage_kernel(kind, 8 if kind == "march" else 0, 0)
    o = Oracle(cfg)
    o.set_inputs(inp)
    dom.advance(6)
    o.step(6)
    g, r = dom.get_state(), o.get_state()
    for f in range(5):
        assert rel_l2(interior(g["hydroFlds"][f]), interior(r["hydroFlds"][f])) < STATE_TOL[f], f
    assert rel_l2(interior(g["moist"][0]), interior(r["moist"][0])) < 1e-6
    assert dom.nonfinite() == 0
    dom.close()
    host.cleanup()

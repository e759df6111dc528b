"""Known-answer tests of the FP64 oracle (the checker of the CUDA path).

The reference ships no tests or golden vectors for this path; the oracle is pinned by
analytic properties here and by the reference build's own outputs in
tests/test_golden_reference.py."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import interior
from oracle.pyoracle import Oracle


def _host(fe, case, nx, ny, nz, edits=(), **kw):
    host = fe.Host()
    text = fe.cases.param_text(case, nx, ny, nz, **kw)
    for a, b in edits:
        assert a in text
        text = text.replace(a, b)
    host.load_params_text(text)
    if kw.get("hill"):
        pass
    return host


REST = (("thetaPerturbationSwitch = 1", "thetaPerturbationSwitch = 0"), ("U_g = 10.0", "U_g = 0.0"),
        ("surflayerSelector = 1", "surflayerSelector = 0"))


@pytest.mark.parametrize("hill", [False, True])
def test_rest_state_has_zero_tendency(fe, hill):
    case = "cbl_hill_dry" if hill else "cbl_dry"
    host = _host(fe, case, 12, 10, 16, REST)
    if hill:
        host.gaussian_hill(20.0, 60.0)
    host.init(1)
    o = Oracle(host.config())
    o.set_inputs(host.inputs())
    for stage in (0, 2):
        F = o.build_frhs(stage)
        for f in range(5):
            assert np.abs(interior(F["hydroFrhs"][f])).max() == 0.0, (stage, f)
        assert np.abs(interior(F["sgstkeFrhs"][0])).max() == 0.0
    host.cleanup()


def test_uniform_geostrophic_flow_is_steady(fe):
    edits = REST[:1] + REST[2:]  # keep U_g = 10 m/s, no perturbations, no surface layer
    host = _host(fe, "cbl_dry", 12, 10, 16, edits)
    host.init(1)
    o = Oracle(host.config())
    o.set_inputs(host.inputs())
    F = o.build_frhs(2)["hydroFrhs"]
    for f in range(5):
        assert np.abs(interior(F[f])).max() < 1e-9, f
    host.cleanup()


def test_mass_is_conserved(fe):
    host = fe.cases.setup_host("cbl_dry", 12, 10, 16)
    inp = host.inputs()
    o = Oracle(host.config())
    o.set_inputs(inp)
    D = interior(inp["D_Jac"].astype(np.float64))
    m0 = (interior(inp["hydroFlds"][0].astype(np.float64)) * D).sum()
    o.step(5)
    m1 = (interior(o.get_state()["hydroFlds"][0]) * D).sum()
    assert abs(m1 - m0) / m0 < 1e-13
    host.cleanup()


ADVECTION_ONLY = (("stabilityScheme = 1", "stabilityScheme = 0"), ("thetaPerturbationSwitch = 1", "thetaPerturbationSwitch = 0"),
                  ("surflayerSelector = 1", "surflayerSelector = 0"), ("turbulenceSelector = 1", "turbulenceSelector = 0"),
                  ("TKESelector = 1", "TKESelector = 0"), ("coriolisSelector = 1", "coriolisSelector = 0"),
                  ("U_g = 10.0", "U_g = 5.0"))


def _theta_advection(fe, n, profile, sel=3, b=0.0):
    """rho*theta tendency and its exact value -u d(rho theta)/dx for theta = 300 + profile(x/L)
    on one periodic wavelength of n cells, advected by a uniform 5 m/s wind with scheme `sel`.
    profile returns (value, derivative in x/L)."""
    edits = ADVECTION_ONLY + (("advectionSelector = 3", f"advectionSelector = {sel}"), ("b_hyb = 0.0", f"b_hyb = {b}"))
    host = _host(fe, "cbl_dry", n, 4, 4, edits)
    host.init(1)
    inp = host.inputs()
    H = inp["hydroFlds"].astype(np.float64)
    dx = 20.0
    L = n * dx
    x = ((np.arange(n + 6) - 3 + 0.5) * dx) / L
    val, der = profile(x)
    rho = H[0]
    H[4] = rho * (300.0 + val)[:, None, None]
    o = Oracle(host.config())
    o.set_inputs(inp)
    o.lib.ora_set_state_f64(o.h, np.ascontiguousarray(H).ctypes.data_as(o.lib.ora_set_state_f64.argtypes[1]), None, None)
    F = o.build_frhs(0)["hydroFrhs"][4]
    exact = -5.0 * rho * (der / L)[:, None, None]
    host.cleanup()
    return interior(F), interior(exact)


def _sine(x):
    return np.sin(2 * np.pi * x), 2 * np.pi * np.cos(2 * np.pi * x)


def _advective_tendency_error(fe, n, sel=3, b=0.0):
    """Relative max error of the rho*theta advective tendency of one sine wave per domain
    (n cells per wavelength) advected by a uniform wind."""
    F, exact = _theta_advection(fe, n, _sine, sel, b)
    # relative to the exact tendency: the grid spacing is fixed, so kh = 2 pi / n
    return np.abs(F - exact).max() / np.abs(exact).max()


def test_hyb56_advection_is_fifth_order(fe):
    e1 = _advective_tendency_error(fe, 16)
    e2 = _advective_tendency_error(fe, 32)
    order = np.log2(e1 / e2)
    assert 4.6 < order < 5.4, order


# Orders of the other schemes' tendency in the max norm on point values: upwind 1; QUICK 2
# (its face value is third-order, but the difference of two face values of point data leaves a
# (kh)^2/24 term); HYB34 3 with full upwinding (b = 0) and 4 centred (b = 1); centred 2nd 2.
@pytest.mark.parametrize("sel,b,order", [(0, 0.0, 1.0), (1, 0.0, 2.0), (2, 0.0, 3.0), (2, 1.0, 4.0), (6, 0.0, 2.0)])
def test_advection_scheme_orders(fe, sel, b, order):
    e1 = _advective_tendency_error(fe, 32, sel, b)
    e2 = _advective_tendency_error(fe, 64, sel, b)
    assert abs(np.log2(e1 / e2) - order) < 0.3, (sel, b, np.log2(e1 / e2))


@pytest.mark.parametrize("sel", range(7))
def test_every_scheme_is_exact_on_linear_data(fe, sel):
    """theta = 300 + |x/L - 1/2|: away from the two kinks every stencil sees linear data, where
    each scheme's face value is exact (WENO3/WENO5: the smoothness indicators are equal, so the
    weights reduce to the linear ones) and the tendency is -u rho dtheta/dx."""
    n = 32
    F, exact = _theta_advection(fe, n, lambda x: (np.abs(x - 0.5), np.sign(x - 0.5)), sel, 0.5)
    away = np.r_[3:13, 19:29]  # cells whose +-3 stencil lies on one linear segment
    np.testing.assert_allclose(F[away], exact[away], rtol=1e-9)


def test_filter_damps_the_two_grid_mode_at_coeff_over_dt(fe):
    """The 6th-order filter on rho w (cuda_filtersDevice.cu:73-122): for w = a(-1)^k both face
    fluxes are +-32 a and pass the limiter, so the tendency is -64 a (0.015625 c/dt) = -(c/dt) a;
    a profile linear in z has zero filtered flux. Checked on levels whose +-3 stencil is interior."""
    coeff = 0.03
    edits = REST + (("filterSelector = 0", "filterSelector = 1"), ("filter_6th_coeff = 0.03", f"filter_6th_coeff = {coeff}"))
    host = _host(fe, "cbl_dry", 8, 8, 24, edits)
    host.init(1)
    inp = host.inputs()
    cfg = host.config()
    dt = float(np.float32(cfg.dt))
    H = inp["hydroFlds"].astype(np.float64)
    k = np.arange(H.shape[3])
    lv = slice(6, H.shape[3] - 6)
    rate = float(np.float32(coeff)) / dt  # filter_6th_coeff and dt are float parameters
    for w, expect in ((0.01 * (-1.0) ** k, -rate * 0.01 * (-1.0) ** k), (1e-3 * k, 0.0 * k)):
        H[3] = w[None, None, :] * np.ones(H.shape[1:3])[:, :, None]
        tend = []
        for filt in (0, 1):
            cfg.filterSelector = filt
            o = Oracle(cfg)
            o.set_inputs(inp)
            o.lib.ora_set_state_f64(o.h, np.ascontiguousarray(H).ctypes.data_as(o.lib.ora_set_state_f64.argtypes[1]),
                                    None, None)
            tend.append(o.build_frhs(0)["hydroFrhs"][3])
        diff = (tend[1] - tend[0])[3:-3, 3:-3, lv]
        np.testing.assert_allclose(diff, np.broadcast_to(expect[lv], diff.shape), rtol=1e-9, atol=1e-12)
    host.cleanup()


def test_neutral_surface_layer_log_law(fe):
    edits = (("surflayer_wth = 0.35", "surflayer_wth = 0.0"), ("thetaPerturbationSwitch = 1", "thetaPerturbationSwitch = 0"))
    host = _host(fe, "cbl_dry", 8, 8, 8, edits)
    host.init(1)
    inp = host.inputs()
    o = Oracle(host.config())
    o.set_inputs(inp)
    F = o.build_frhs(2)
    s = o.get_surface()
    z1, z0, kap = 5.0, 0.05, 0.4
    cd = kap ** 2 / np.log((z1 + z0) / z0) ** 2
    rho = inp["hydroFlds"][0][5, 5, 3]
    U = inp["hydroFlds"][1][5, 5, 3] / rho
    np.testing.assert_allclose(s["cd"][5, 5], cd, rtol=1e-6)  # z0 and dZi are float inputs
    np.testing.assert_allclose(F["taus"][2][5, 5, 3], -cd * U * (U * rho), rtol=1e-6)
    # the final u* is taken from the flux-form stress -cd|U|(rho u), so it carries sqrt(rho)
    # (cuda_surfaceLayerDevice.cu:402-406)
    np.testing.assert_allclose(s["fricVel"][5, 5], np.sqrt(cd * rho) * U, rtol=1e-6)
    host.cleanup()


def test_rk3_stage_weights(fe):
    """phi* = phi + dt/3 F, phi** = phi + dt/2 F*, phi^{n+1} = phi + dt F** (WS2002)."""
    host = fe.cases.setup_host("cbl_dry", 8, 8, 8)
    inp = host.inputs()
    o = Oracle(host.config())
    o.set_inputs(inp)
    phi0 = o.get_state()["hydroFlds"].copy()
    F0 = o.build_frhs(0)["hydroFrhs"].copy()
    o.rk_stage(0)
    phi1 = o.get_state()["hydroFlds"]
    dt = float(np.float32(0.025))  # dt is a float parameter (time_integration.h:26)
    np.testing.assert_allclose(interior(phi1), interior(phi0 + dt / 3.0 * F0), rtol=0, atol=1e-12)
    host.cleanup()


LSF = dict(lsfSelector=1, lsf_freq=0.05, lsf_w_surf=0.0, lsf_w_lev1=-40.0, lsf_w_lev2=0.0, lsf_w_zlev1=60.0,
           lsf_w_zlev2=120.0, lsf_th_surf=-2.0, lsf_th_lev1=-1.0, lsf_th_lev2=0.5, lsf_th_zlev1=50.0,
           lsf_th_zlev2=110.0, lsf_qv_surf=-0.5, lsf_qv_lev1=-0.5, lsf_qv_lev2=0.0, lsf_qv_zlev1=40.0, lsf_qv_zlev2=90.0)


def _lsf_profile(p, z):
    s_, l1, l2, z1, z2 = [float(np.float32(x)) for x in p]  # the parameters are floats
    return np.where(z <= z1, s_ + (l1 - s_) / z1 * z, np.where(z <= z2, l1 + (l2 - l1) / (z2 - z1) * (z - z1), l2))


def _lsf_tendency_difference(fe, params, state_edit=None):
    """Last-stage tendency with the forcing minus without it, at a forcing step (it = 2 with
    lsf_freq = 2 dt), from the same state."""
    host = fe.Host()
    host.load_params_text(fe.cases.param_text("cbl_moist_hill", 10, 8, 16, params=params))
    host.init(3)
    host.set_qv_profile(14.0, 4.0, 1500.0)
    inp = host.inputs()
    cfg = host.config()
    out = []
    for on in (0, 1):
        cfg.lsfSelector = on
        o = Oracle(cfg)
        o.set_inputs(inp, 0.05, 2)
        if state_edit is not None:
            state_edit(o, inp)
        r = o.build_frhs(2)
        out.append((r["hydroFrhs"], r["moistFrhs"]))
    host.cleanup()
    return inp, (out[1][0] - out[0][0]), (out[1][1] - out[0][1])


def test_lsf_forcing_follows_the_piecewise_linear_profiles(fe):
    """theta and q_v forcing (cuda_largeScaleForcingsDevice.cu:177-230): rate(z) rho n / 3600
    with n = lsf_freq/dt steps per application; no subsidence terms without lsf_horMnSubTerms."""
    inp, dH, dM = _lsf_tendency_difference(fe, dict(LSF, lsf_horMnSubTerms=0))
    z = inp["zPos"].astype(np.float64)
    rho = inp["hydroFlds"][0].astype(np.float64)
    th = _lsf_profile((-2.0, -1.0, 0.5, 50.0, 110.0), z) * rho * 2 / 3600.0
    qv = _lsf_profile((-0.5, -0.5, 0.0, 40.0, 90.0), z) * rho * 2 / 3600.0
    np.testing.assert_allclose(interior(dH[4]), interior(th), rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(interior(dM[0]), interior(qv), rtol=1e-9, atol=1e-15)
    for f in (0, 1, 2, 3):
        assert np.abs(interior(dH[f])).max() == 0.0


def test_lsf_subsidence_of_a_linear_wind_profile(fe):
    """With a horizontally uniform state the slab means are the profiles themselves, so the
    subsidence term of u = a z on the uniform grid is -w_ls rho rho a (the reference multiplies
    the rho-weighted w_ls by rho once more) on levels whose k+-1 neighbours are interior."""
    a = 0.02

    def edit(o, inp):
        H = inp["hydroFlds"].astype(np.float64).copy()
        rho = H[0].mean(axis=(0, 1), keepdims=True) * np.ones_like(H[0])
        H[0] = rho
        H[1] = rho * a * inp["zPos"].astype(np.float64)
        H[2] = 0.0
        H[3] = 0.0
        H[4] = rho * 300.0
        M = inp["moist"].astype(np.float64).copy()
        M[0] = rho * 10.0
        M[1] = 0.0
        o.lib.ora_set_state_f64(o.h, *(np.ascontiguousarray(x).ctypes.data_as(o.lib.ora_set_state_f64.argtypes[1])
                                       for x in (H, inp["sgstke"].astype(np.float64), M)))

    inp, dH, dM = _lsf_tendency_difference(fe, dict(LSF, lsf_horMnSubTerms=1), edit)
    z = inp["zPos"].astype(np.float64)
    rho = inp["hydroFlds"][0].astype(np.float64).mean(axis=(0, 1), keepdims=True) * np.ones_like(z)
    fw = _lsf_profile((0.0, -40.0, 0.0, 60.0, 120.0), z) * rho * 2 / 3600.0
    lv = slice(4, -4)
    np.testing.assert_allclose(interior(dH[1])[..., lv], interior(-fw * rho * a)[..., lv], rtol=1e-7)
    # v = 0, theta and q_v/rho uniform: only the large-scale forcing of theta and q_v remains
    assert np.abs(interior(dH[2])).max() == 0.0
    th = _lsf_profile((-2.0, -1.0, 0.5, 50.0, 110.0), z) * rho * 2 / 3600.0
    np.testing.assert_allclose(interior(dH[4])[..., lv], interior(th)[..., lv], rtol=1e-7, atol=1e-12)

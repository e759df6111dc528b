"""Host C layer: grid coordinates and metrics (reference SRC/GRID/grid.c:263-803), FP64
hydrostatic base state (SRC/HYDRO_CORE/hydro_core.c:1053-1190), initial state (:1193-1250)."""
from __future__ import annotations

import numpy as np

from conftest import interior


def test_flat_grid_and_metrics(fe):
    host = fe.cases.setup_host("cbl_dry", 8, 6, 10)
    z = host.array("zPos")[0]
    dz = host.gf("dZ")
    k = np.arange(z.shape[2])
    np.testing.assert_allclose(z[5, 4, :], (k - 3 + 0.5) * dz, rtol=0, atol=1e-4)
    for name, val in (("D_Jac", 1.0), ("invD_Jac", 1.0), ("J33", 1.0), ("J31", 0.0), ("J32", 0.0)):
        np.testing.assert_array_equal(host.array(name)[0], np.float32(val))
    host.cleanup()


def test_hill_terrain_following_metrics(fe):
    host = fe.cases.setup_host("cbl_hill_dry", 24, 20, 12, hill_halfwidth=120.0, hill_height=30.0)
    z, D, J31, J32, J33 = (host.array(n)[0].astype(np.float64) for n in ("zPos", "D_Jac", "J31", "J32", "J33"))
    ztop = 12 * 10.0 - 5.0
    h = host.array("topoPos", 1, two_d=True)[0].astype(np.float64)
    # surface cell centre lifted by the terrain and compressed (grid.c:407)
    np.testing.assert_allclose(z[3:-3, 3:-3, 3], 5.0 * (ztop - h[3:-3, 3:-3]) / ztop + h[3:-3, 3:-3], rtol=1e-6)
    # D = dz/dzeta = (ztop - h)/ztop in the interior; J33 = 1/D
    np.testing.assert_allclose(interior(D), np.broadcast_to(((ztop - h) / ztop)[3:-3, 3:-3, None], interior(D).shape),
                               rtol=2e-6)
    np.testing.assert_allclose(interior(J33) * interior(D), 1.0, rtol=2e-6)
    # the reference's cofactor choice gives exactly zero horizontal metric terms
    assert np.all(J31 == 0.0) and np.all(J32 == 0.0)
    assert D.min() < 0.99  # the hill is resolved
    # metric halos copy the nearest interior value (grid.c:663-742)
    np.testing.assert_array_equal(D[0:3, 5, 5], D[3, 5, 5])
    np.testing.assert_array_equal(D[5, 5, -3:], D[5, 5, -4])
    host.cleanup()


def test_topofile_round_trip(fe, tmp_path):
    host = fe.cases.setup_host("cbl_hill_dry", 16, 12, 8, hill_halfwidth=80.0, hill_height=20.0)
    z1 = host.array("zPos")[0].copy()
    path = str(tmp_path / "topo.bin")
    host.write_topofile(path)
    raw = np.fromfile(path, dtype=np.int32, count=2)
    assert tuple(raw) == (16, 12)
    host2 = fe.Host()
    host2.load_params_text(fe.cases.param_text("cbl_hill_dry", 16, 12, 8, topo=path))
    host2.init(12345)
    np.testing.assert_array_equal(host2.array("zPos")[0], z1)
    host2.cleanup()


def test_base_state_hydrostatic_fp64(fe):
    host = fe.cases.setup_host("cbl_dry", 8, 8, 80)
    z = host.array("zPos")[0][5, 5, :].astype(np.float64)
    bs = host.array("hydroBaseStateFlds", 2)[:, 5, 5, :].astype(np.float64)
    rho, rth = bs
    th = rth / rho
    R, cv, g, p0 = 287.04, 718.0, 9.81, 1e5
    cp = R + cv
    p = (rth * R / p0 ** (R / cp)) ** (cp / cv)
    # theta: neutral to zStableBottom = 600 m, +8 K/km above
    below = z <= 600.0
    np.testing.assert_allclose(th[below], 300.0, rtol=2e-7)
    np.testing.assert_allclose(th[~below], 300.0 + 0.008 * (z[~below] - 600.0), rtol=2e-7)
    # hydrostatic balance dp/dz = -rho g (centred differences, O(dz^2))
    dpdz = (p[2:] - p[:-2]) / (z[2:] - z[:-2])
    np.testing.assert_allclose(dpdz, -rho[1:-1] * g, rtol=2e-4)
    host.cleanup()


def test_initial_state_and_seed(fe):
    host = fe.cases.setup_host("cbl_dry", 12, 10, 50, seed=7)
    H = host.array("hydroFlds", 5).astype(np.float64)
    bs = host.array("hydroBaseStateFlds", 2).astype(np.float64)
    z = host.array("zPos")[0]
    th = interior(H[4] / H[0])
    thbs = interior(bs[1] / bs[0])
    d = th - thbs
    low = interior(z) <= 400.0
    assert np.abs(d[low]).max() <= 0.25 + 1e-4 and np.abs(d[low]).max() > 0.2
    assert np.all(d[~low] == 0.0)
    np.testing.assert_allclose(interior(H[1]), 10.0 * interior(bs[0]), rtol=1e-6)
    assert np.all(H[3] == 0.0) and np.all(H[2] == 0.0)
    first = H[4].copy()
    host.init(7)
    np.testing.assert_array_equal(host.array("hydroFlds", 5)[4], first)
    host.init(8)
    assert not np.array_equal(host.array("hydroFlds", 5)[4], first)
    host.cleanup()


def test_moisture_profile(fe):
    host = fe.cases.setup_host("cbl_moist_hill", 8, 8, 20, hill_halfwidth=50.0, hill_height=10.0)
    q = host.array("moistScalars", 2)
    rho = host.array("hydroFlds", 1)[0]
    z = host.array("zPos")[0]
    qv = interior(q[0] / rho)
    expect = 14.0 + (4.0 - 14.0) * np.clip(interior(z), 0, 1500.0) / 1500.0
    np.testing.assert_allclose(qv, expect, rtol=1e-5)
    assert np.all(q[1] == 0.0)
    host.cleanup()



def test_configuration_checks_of_the_optional_physics(fe):
    """fe_create validates a configuration before it looks for a device, so on a machine without
    one an accepted configuration fails only with FE_ERR_NO_DEVICE (7). Every advection selector,
    the explicit filter and the large-scale forcing are accepted; out-of-range selectors, an
    interval below half a step and molecular diffusion are refused (FE_ERR_CONFIG, 2) by name."""
    import ctypes

    eng = fe.load(rebuild=False)["engine"]
    host = fe.cases.setup_host("cbl_moist_hill", 8, 6, 6)
    base = host.config()
    host.cleanup()

    def create(**kw):
        cfg = type(base).from_buffer_copy(base)
        for k, v in kw.items():
            setattr(cfg, k, v)
        h = ctypes.c_void_p()
        rc = eng.fe_create(ctypes.byref(cfg), 0, ctypes.byref(h))
        msg = eng.fe_last_error().decode()
        if rc == 0:
            eng.fe_destroy(h)
        return rc, msg

    accepted = [dict(advectionSelector=s) for s in range(7)] + [dict(TKEAdvSelector=s) for s in range(7)]
    accepted += [dict(moistureAdvSelectorQv=s) for s in range(7)] + [dict(moistureAdvSelectorQi=s) for s in range(3)]
    accepted += [dict(filterSelector=1, filter_6th_coeff=0.12), dict(lsfSelector=1, lsf_horMnSubTerms=1, lsf_freq=1.0)]
    for kw in accepted:
        rc, msg = create(**kw)
        assert rc in (0, 7), (kw, rc, msg)
    refused = [(dict(advectionSelector=7), "advectionSelector"), (dict(moistureAdvSelectorQi=3), "moistureAdvSelectorQi"),
               (dict(filterSelector=2), "filterSelector"), (dict(filterSelector=1, filter_6th_coeff=1.5), "filter_6th_coeff"),
               (dict(lsfSelector=1, lsf_freq=0.01), "lsf_freq"), (dict(diffusionSelector=1), "diffusion"),
               (dict(b_hyb=1.5), "b_hyb")]
    for kw, name in refused:
        rc, msg = create(**kw)
        assert rc == 2 and name in msg, (kw, rc, msg)

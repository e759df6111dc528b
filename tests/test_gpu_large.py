"""The large dry CBL over terrain at its full size, 1024 x 1024 x 256 cells (about 46 GB of device
memory), checked without an FP64 run of that size (which would need ~100 GB of host memory and
hours of one core): the domain is built as 8 x 8 periodic copies of a 128 x 128 x 256 domain with
the same physics and a Gaussian hill centred in each copy.

The hill is symmetric about the copy's centre, so its edge columns carry equal metrics; every
input is given periodic horizontal halos in both domains. Every cell of the large domain then
sees exactly the inputs of the corresponding cell of the small one, and the arithmetic does not
depend on where a cell lies, so the large domain's tendencies of every RK stage and its state
after 2 RK3 steps must equal the tiled small domain's bit for bit: this checks the 64-bit
offsets, the launch geometry and the march shape chosen at the full size (64 planes per thread
block there). The small domain's tendencies are checked against the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import interior, rel_l2

pytestmark = pytest.mark.gpu

REPS = 8
TWO_D = ("z0m", "z0t", "htFlux", "tskin", "fricVel", "qFlux", "qskin")


def _tile_wrap(a: np.ndarray, reps: int, two_d: bool) -> np.ndarray:
    """Interior columns of a halo-inclusive field tiled reps x reps times, with periodic halos."""
    ax = (a.ndim - 2, a.ndim - 1) if two_d else (a.ndim - 3, a.ndim - 2)
    sl = [slice(None)] * a.ndim
    sl[ax[0]] = slice(3, -3)
    sl[ax[1]] = slice(3, -3)
    core = np.ascontiguousarray(a[tuple(sl)])
    r = [1] * a.ndim
    r[ax[0]] = reps
    r[ax[1]] = reps
    pad = [(0, 0)] * a.ndim
    pad[ax[0]] = (3, 3)
    pad[ax[1]] = (3, 3)
    return np.pad(np.tile(core, r), pad, mode="wrap")


def _inputs(inp: dict, reps: int) -> dict:
    return {k: (None if v is None else _tile_wrap(v, reps, k in TWO_D)) for k, v in inp.items()}


def _tiled_interior(a: np.ndarray) -> np.ndarray:
    """Interior cells of a small-domain field, tiled to the large domain's interior."""
    return np.tile(interior(a), (REPS, REPS, 1))


def test_full_size_domain_equals_tiled_copies(fe):
    from oracle.pyoracle import Oracle

    host = fe.cases.setup_host("cbl_hill_dry", 128, 128, 256)
    small_cfg = host.config()
    raw = host.inputs()
    host.cleanup()
    small_inp = _inputs(raw, 1)
    big_cfg = fe.FeConfig.from_buffer_copy(small_cfg)
    big_cfg.Nx = big_cfg.Ny = 128 * REPS
    big_inp = _inputs(raw, REPS)
    del raw

    small = fe.Domain(small_cfg)
    small.set_inputs(small_inp)
    big = fe.Domain(big_cfg)
    big.set_inputs(big_inp)
    del big_inp
    assert big.stage_kernel()[0] == "march"
    o = Oracle(small_cfg)
    o.set_inputs(small_inp)
    for stage in (0, 1, 2):
        fs = small.build_frhs(stage, taus=False)
        fb = big.build_frhs(stage, taus=False)
        fo = o.build_frhs(stage)
        for key, nf in (("hydroFrhs", 5), ("sgstkeFrhs", 1)):
            for f in range(nf):
                np.testing.assert_array_equal(interior(fb[key][f]), _tiled_interior(fs[key][f]),
                                              err_msg=f"{stage} {key} {f}")
                if np.abs(interior(fo[key][f])).max() > 0:
                    assert rel_l2(interior(fs[key][f]), interior(fo[key][f])) < 1e-3, (stage, key, f)
        del fb
    o.close()
    small.advance(2)
    big.advance(2)
    ss, sb = small.get_state(), big.get_state()
    for f in range(5):
        np.testing.assert_array_equal(interior(sb["hydroFlds"][f]), _tiled_interior(ss["hydroFlds"][f]),
                                      err_msg=str(f))
    np.testing.assert_array_equal(interior(sb["sgstke"][0]), _tiled_interior(ss["sgstke"][0]))
    assert big.nonfinite() == 0
    big.close()
    small.close()

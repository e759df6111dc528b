"""Domain decomposition on the device: px x py slabs of one domain on one B200, each RK
stage's commit writing the neighbouring slabs' halos (the per-stage exchange of
cuda_hydroCoreDevice.cu:276-314 fused into the commit), give the undecomposed domain's state bit
for bit -- through graph replay (8-step batches) and eager steps, with the autotuner's timing
launches in between (which must not write into a neighbour)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "moist_hill": ("cbl_moist_hill", 24, 20, 16, dict(hill_halfwidth=90.0, hill_height=20.0, qv=(24.0, 8.0, 300.0))),
    "hill_dry": ("cbl_hill_dry", 24, 24, 16, dict(hill_halfwidth=80.0, hill_height=25.0)),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("px,py", [(2, 1), (1, 2), (2, 2), (3, 2)])
def test_slab_group_equals_whole_domain(fe, name, px, py):
    case, nx, ny, nz, kw = CASES[name]
    host = fe.cases.setup_host(case, nx, ny, nz, **kw)
    cfg, inp = host.config(), host.inputs()
    whole = fe.Domain(cfg)
    whole.set_inputs(inp)
    group = fe.halo.SlabGroup(cfg, inp, px, py)
    for s in group.slabs:
        s.autotune()  # its timing commits keep their images local
        s.set_stage_kernel("march", 8, 8)  # the cell kernel agrees to FP32 rounding only
    whole.advance(11)
    group.advance(11)  # one 8-step graph + 3 eager steps
    a, b = whole.get_state(), group.get_state()
    for key in ("hydroFlds", "sgstke", "moist", "pres"):
        if a.get(key) is not None:
            np.testing.assert_array_equal(b[key][..., 3:-3, 3:-3, 3:-3], a[key][..., 3:-3, 3:-3, 3:-3], err_msg=key)
    # the slab halos hold the neighbours' cells: the reassembled array, halos included, is the whole one
    np.testing.assert_array_equal(b["hydroFlds"][:, :, :, 3:-3], a["hydroFlds"][:, :, :, 3:-3])
    group.close()
    whole.close()
    host.cleanup()


def test_decomposition_refuses_subsidence_means(fe):
    host = fe.cases.setup_host("cbl_dry", 16, 12, 8)
    cfg = host.config()
    cfg.lsfSelector, cfg.lsf_horMnSubTerms = 1, 1
    with pytest.raises(fe.FeError, match="whole domain"):
        fe.halo.SlabGroup(cfg, host.inputs(), 2, 1)
    host.cleanup()

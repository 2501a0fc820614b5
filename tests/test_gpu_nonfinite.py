"""Non-finite detection (CF_ENONFINITE).

The reference has no NaN check: its check() (check.h:8-12) aborts only on
allocation, order and pivot failures, and a blown-up run writes NaN fields.
Here the mass-control kernel of every substep sums each interior point of u
and c into a bulk mean; a NaN or Inf anywhere in them sets a device flag that
cf_sync and cf_get_log report, and that cf_serve turns into a per-request
status.  The failures are made on the host: a NaN written into a field with
cf_set_field, or a request whose seeded amplitude is NaN.  No GPU fault is
involved -- NaN arithmetic is ordinary floating point."""
import math

import numpy as np
import pytest

import chanfast_np as cn

pytestmark = pytest.mark.gpu


def make_cfg(cf, order, scheme="chanfast", nx=64, ny=24, nz=16):
    prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1 / 2800.0, prandtl=0.71)
    return cf.Config.from_params(prm, scheme=scheme)


def expect_nonfinite(cf, fn):
    with pytest.raises(cf.ChanfastError) as e:
        fn()
    assert e.value.status == cf.CF_ENONFINITE


@pytest.mark.parametrize("scheme,order", [("chanfast", 2), ("chanfast", 4), ("channel", 4)])
@pytest.mark.parametrize("field,value", [("v", math.nan), ("w", math.nan), ("c", math.inf)])
def test_nonfinite_field_is_reported(cf, gpu, scheme, order, field, value):
    with cf.Instance(make_cfg(cf, order, scheme)) as inst:
        inst.init_fields(1, 0.1, 0.01)
        inst.step(3)
        inst.sync()                      # a clean state reports nothing
        assert inst.log().shape[0] == 3
        a = inst.get_field(field)
        a[5, 6, 7] = value
        inst.set_field(field, a)
        inst.sync()                      # setting a field alone is not a substep
        inst.step(2)
        expect_nonfinite(cf, inst.sync)
        expect_nonfinite(cf, inst.log)
        inst.step(1)                     # the flag is sticky
        expect_nonfinite(cf, inst.sync)
        inst.init_fields(1, 0.1, 0.01)   # new fields clear it
        inst.sync()
        assert np.isfinite(inst.get_field("u")).all()


def test_graph_path_reports_nonfinite(cf, gpu):
    with cf.Instance(make_cfg(cf, 4)) as inst:
        inst.init_fields(2, 0.1, 0.01)
        a = inst.get_field("u")
        a[3, 3, 3] = math.nan
        inst.set_field("u", a)
        inst.step_graph(4)
        expect_nonfinite(cf, inst.sync)


def test_serve_retires_nonfinite_request_alone(cf, gpu):
    cfg = make_cfg(cf, 2, nx=32, ny=32, nz=16)
    reqs = [dict(cfg=cfg, seed=q, amp=(math.nan if q == 1 else 0.1), c_amp=0.01, nsteps=4, arrival_s=0.0)
            for q in range(3)]
    res = cf.serve(reqs, hbm_budget_bytes=8e9, max_active=4, quantum=1)
    assert res[1]["status"] == cf.CF_ENONFINITE
    assert res[1]["steps_done"] == 1      # retired after its first round
    for q in (0, 2):
        assert res[q]["status"] == cf.CF_OK and res[q]["steps_done"] == 4

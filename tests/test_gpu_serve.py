"""The serving loop (cf_serve): requests of different grids, orders,
Reynolds numbers and step counts arriving over time, admitted by a device-
memory budget, stepped together by batched launches, retired one by one.

Each served result must equal, bit for bit, the same request run alone
(cf_batch_step on that instance only): in the mix, neighbours share launches
but never data.  Admission must keep the resident instances within the
budget, and a request larger than the budget fails alone."""
import numpy as np
import pytest

import chanfast_np as cn

pytestmark = pytest.mark.gpu


def cfg_of(cf, order, nx, ny, nz, re):
    prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1.0 / re, prandtl=0.71)
    return cf.Config.from_params(prm)


TRACE = [  # order, nx, ny, nz, Re_b, steps, arrival (s)
    (2, 64, 64, 32, 2800.0, 7, 0.0), (2, 96, 96, 24, 5000.0, 4, 0.0), (4, 128, 64, 32, 8000.0, 9, 0.05),
    (4, 48, 40, 16, 3000.0, 3, 0.1), (2, 64, 48, 20, 10000.0, 6, 0.1), (4, 64, 64, 24, 4000.0, 5, 0.3),
]


def snapshot(view):
    return {nm: view.get_field(nm) for nm in "uvwcp"} | {"log": view.log()}


def test_served_results_equal_alone(cf, gpu):
    reqs = [dict(cfg=cfg_of(cf, o, nx, ny, nz, re), seed=20 + q, amp=0.1, c_amp=0.01, nsteps=st, arrival_s=t)
            for q, (o, nx, ny, nz, re, st, t) in enumerate(TRACE)]
    got = {}
    res = cf.serve(reqs, hbm_budget_bytes=40e9, max_active=8, quantum=2,
                   on_done=lambda i, v: got.__setitem__(i, snapshot(v)))
    for q, r in enumerate(res):
        assert r["status"] == 0, q
        assert r["steps_done"] == reqs[q]["nsteps"]
        assert reqs[q]["arrival_s"] <= r["admit_s"] <= r["finish_s"]
    for q, r in enumerate(reqs):
        with cf.Instance(r["cfg"]) as inst:
            inst.init_fields(r["seed"], r["amp"], r["c_amp"])
            cf.batch_step([inst], 3 * r["nsteps"])
            inst.sync()
            for nm in "uvwcp":
                assert np.array_equal(inst.get_field(nm), got[q][nm]), (q, nm)
            assert np.array_equal(inst.log(), got[q]["log"]), q


def test_admission_respects_budget(cf, gpu):
    cfgs = [cfg_of(cf, 2, 128, 128, 64, 3000.0) for _ in range(6)]
    one = cf.instance_bytes(cfgs[0])
    budget = 2.5 * one   # two resident at a time
    reqs = [dict(cfg=c, seed=q, nsteps=4, arrival_s=0.0) for q, c in enumerate(cfgs)]
    reqs.append(dict(cfg=cfg_of(cf, 2, 512, 512, 128, 3000.0), seed=9, nsteps=1, arrival_s=0.0))   # too large
    res = cf.serve(reqs, hbm_budget_bytes=budget, max_active=8, quantum=1)
    assert res[-1]["status"] == cf.CF_ENOMEM and res[-1]["steps_done"] == 0
    spans = [(r["admit_s"], r["finish_s"]) for r in res[:-1]]
    assert all(r["status"] == 0 for r in res[:-1])
    events = sorted([(a, 1) for a, _ in spans] + [(b, -1) for _, b in spans], key=lambda e: (e[0], e[1]))
    live = peak = 0
    for _, d in events:
        live += d
        peak = max(peak, live)
    assert peak <= 2

"""Batched stepping: one launch per stage of the substep covering many
instances of different sizes, orders and parameters (cf_batch_step,
cf_batch_create / cf_batch_run).

Alone and in the mix: each member's fields, pressure and log equal, bit for
bit, the same instance stepped alone in a batch of one (the same kernels on
the same arguments; neighbours in a launch do not interact).  Against the
plain single-instance path (cf_step), whose kernels are separate
instantiations of the same bodies and may contract a few multiply-adds
differently, they agree to relative L2 <= 1e-13 (the engine's own bar against
the reference is 1e-13 on u, v, w, c)."""
import numpy as np
import pytest

import chanfast_np as cn

pytestmark = pytest.mark.gpu

# order, nx, ny, nz, Re_b: power-of-two and generic transform sizes in x and y
MEMBERS = [(2, 64, 64, 32, 2800.0), (2, 96, 96, 24, 5000.0), (4, 128, 64, 32, 8000.0),
           (4, 48, 40, 16, 3000.0), (2, 64, 48, 20, 10000.0), (4, 64, 64, 24, 4000.0)]


def make(cf, order, nx, ny, nz, re, seed):
    prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1.0 / re, prandtl=0.71)
    inst = cf.Instance(cf.Config.from_params(prm))
    inst.init_fields(seed, 0.1, 0.01)
    return inst


def assert_same(a, b):
    for nm in "uvwcp":
        assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
    assert np.array_equal(a.log(), b.log())
    assert a.substeps_done() == b.substeps_done()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def assert_close(a, b):
    for nm in "uvwc":
        assert rel(a.get_field(nm), b.get_field(nm)) <= 1e-13, nm
    assert rel(a.get_field("p"), b.get_field("p")) <= 1e-10
    la, lb = a.log(), b.log()
    assert la.shape == lb.shape
    assert np.all(np.abs(la - lb) <= 1e-9 * np.maximum(np.abs(lb).max(axis=0), 1e-3))
    assert a.substeps_done() == b.substeps_done()


def test_batch_run_equals_alone(cf, gpu):
    alone = [make(cf, *m, seed=q) for q, m in enumerate(MEMBERS)]
    mixed = [make(cf, *m, seed=q) for q, m in enumerate(MEMBERS)]
    plain = [make(cf, *m, seed=q) for q, m in enumerate(MEMBERS)]
    # one member starts mid-step (another phase of the RK3 cycle)
    for group in (alone, mixed, plain):
        group[2].step(1)
    with cf.Batch(mixed) as B:
        assert B.launches_per_substep() < 11 * len(MEMBERS)
        B.run(1)   # odd step: first half of the cycle, eager
        B.run(4)   # second half, one graph replay, first half
        B.sync()
    for inst in alone:
        with cf.Batch([inst]) as B1:
            B1.run(1)
            B1.run(4)
            B1.sync()
    for inst in plain:
        inst.step(15)
    for a, b, c in zip(alone, mixed, plain):
        assert_same(a, b)
        assert_close(b, c)
        assert b.max_divergence() < 1e-12
    for inst in alone + mixed + plain:
        inst.close()


def test_batch_step_equals_alone(cf, gpu):
    alone = [make(cf, *m, seed=10 + q) for q, m in enumerate(MEMBERS)]
    mixed = [make(cf, *m, seed=10 + q) for q, m in enumerate(MEMBERS)]
    plain = [make(cf, *m, seed=10 + q) for q, m in enumerate(MEMBERS)]
    cf.batch_step(mixed, 7)
    for inst in alone:
        cf.batch_step([inst], 7)
    for inst in plain:
        inst.step(7)
    for inst in alone + mixed + plain:
        inst.sync()
    for a, b, c in zip(alone, mixed, plain):
        assert_same(a, b)
        assert_close(b, c)
    for inst in alone + mixed + plain:
        inst.close()


def test_batch_rejects_foreign_steps_and_schemes(cf, gpu):
    a = make(cf, 2, 64, 64, 16, 2800.0, 1)
    b = make(cf, 2, 64, 64, 16, 2800.0, 2)
    with cf.Batch([a, b]) as B:
        a.step(1)   # stepped outside the batch: its recorded cycle no longer applies
        with pytest.raises(cf.ChanfastError):
            B.run(2)
    prm = cn.Params(order=2, nx=64, ny=16, nz=16, lx=1.0, ly=1.0, lz=2.0, dt=1e-3, nu=1e-3)
    ch = cf.Instance(cf.Config.from_params(prm, scheme="channel"))
    with pytest.raises(cf.ChanfastError):
        cf.Batch([a, ch])
    with pytest.raises(cf.ChanfastError):
        cf.Batch([a, a])
    for inst in (a, b, ch):
        inst.close()

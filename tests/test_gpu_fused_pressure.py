"""The y transforms fused with the Poisson solve (k_poisson_fft, one block per
kx, for ny = 256 and 512) against the three separate launches (k_ffty_p2,
k_poisson, k_ffty_p2) that CF_FUSE_PRESSURE=0 selects at creation.

Both run the same elimination code (PairRows, HeptSweep) and the same
radix-8 transform (fft_p2_line), the fused one with its twiddles read from a
per-stage table instead of formed as products, and both kernels are compiled
with FMA contraction, which may pair a few multiply-adds differently; so the
states agree to rounding, not bit for bit (measured at most 1.3e-14 on u,
v, w, c and 4.5e-12 on p): relative L2 <= 1e-13 on u, v, w, c and <= 1e-10
on p, the engine's bars against the reference, after 3 eager
substeps and two graph-replayed RK3 steps.  The grids reach every path of
the kernel: both sizes (groups of 4 rows of 512 and of 8 rows of 256); the
last solver warp, whose one thread solves the ky = ny/2 pair; a last row
group shorter than the others; the smallest nz of each order; orders 2
and 4 (order 4 with its back-sweep inputs in shared memory); and
non-power-of-two nx.  Other ny keep the separate launches, and by default
the fused launch is taken only where its blocks fill the GPU.  A batch
mixing fused and separate members gives each member the result it has
alone.  The fully implicit scheme's four spectral Helmholtz solves take the
same kernel without the ghost fill."""
import os

import numpy as np
import pytest

import chanfast_np as cn

pytestmark = pytest.mark.gpu

# order, nx, ny, nz
CASES = [(4, 32, 512, 22), (2, 16, 512, 9), (4, 64, 512, 37), (4, 48, 512, 20), (2, 32, 512, 4),
         (4, 16, 512, 6), (2, 24, 512, 14), (4, 32, 256, 20), (2, 16, 256, 9), (4, 48, 256, 13),
         (4, 64, 256, 6)]


def make(cf, order, nx, ny, nz, fused, seed=3, re=4000.0, scheme="chanfast", dt=1e-3):
    """fused: True forces the fused launch where supported, False the
    separate ones, None leaves the choice to the default rule."""
    prm = cn.Params(order=order, nx=nx, ny=ny, nz=nz, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=dt,
                    nu=1.0 / re, prandtl=0.71)
    if fused is not None:
        os.environ["CF_FUSE_PRESSURE"] = "1" if fused else "0"
    try:
        inst = cf.Instance(cf.Config.from_params(prm, scheme=scheme))
    finally:
        os.environ.pop("CF_FUSE_PRESSURE", None)
    inst.init_fields(seed, 0.1, 0.01)
    return inst


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def compare(a, b, what):
    err = {nm: rel(a.get_field(nm), b.get_field(nm)) for nm in "uvwcp"}
    same = all(np.array_equal(a.get_field(nm), b.get_field(nm)) for nm in "uvwcp")
    print(what, "bitwise" if same else {k: "%.1e" % v for k, v in err.items()})
    assert all(err[nm] <= 1e-13 for nm in "uvwc"), (what, err)
    assert err["p"] <= 1e-10, (what, err)
    la, lb = a.log(), b.log()
    assert la.shape == lb.shape
    assert np.all(np.abs(la - lb) <= 1e-9 * np.maximum(np.abs(lb).max(axis=0), 1e-3)), what


@pytest.mark.parametrize("order,nx,ny,nz", CASES)
def test_fused_equals_separate(cf, gpu, order, nx, ny, nz):
    fused = make(cf, order, nx, ny, nz, True)
    sep = make(cf, order, nx, ny, nz, False)
    assert fused.launches_per_substep() == sep.launches_per_substep() - 2
    assert fused.pressure_fused() and not sep.pressure_fused()
    fused.step(3)
    sep.step(3)
    compare(fused, sep, f"o{order} {nx}x{ny}x{nz} 3 substeps")
    fused.step_graph(2)
    sep.step_graph(2)
    compare(fused, sep, f"o{order} {nx}x{ny}x{nz} +2 steps")
    fused.sync()
    assert fused.max_divergence() < 1e-12
    fused.close()
    sep.close()


@pytest.mark.parametrize("order,nx,ny,nz", [(4, 64, 256, 12), (2, 64, 512, 9), (4, 64, 512, 10)])
def test_channel_fused_equals_separate(cf, gpu, order, nx, ny, nz):
    """The fully implicit scheme: its four spectral Helmholtz solves with
    their y transforms in one launch (k_poisson_fft_batch without the ghost
    fill; w over nz - 1 faces; the xy-average profiles of u and c from the
    (0, 0) column), and the pressure solve fused as above."""
    fused = make(cf, order, nx, ny, nz, True, scheme="channel")
    sep = make(cf, order, nx, ny, nz, False, scheme="channel")
    assert fused.launches_per_substep() == sep.launches_per_substep() - 7
    fused.step(3)
    sep.step(3)
    compare(fused, sep, f"channel o{order} {nx}x{ny}x{nz} 3 substeps")
    fused.step_graph(2)
    sep.step_graph(2)
    compare(fused, sep, f"channel o{order} {nx}x{ny}x{nz} +2 steps")
    assert fused.max_divergence() < 1e-12
    fused.close()
    sep.close()


def test_copy_wait_timeout(cf, gpu):
    """A bounded wait that runs out, with nothing faulted: with
    cf_debug_stall_copies the fused launch leaves its row copies unissued (an
    mbarrier phase that nothing completes).  Every block's wait gives up after
    about a second, the kernel finishes without data, and cf_sync reports
    CF_ETIMEOUT.  Reloading the fields clears the status, and the GPU goes on
    working: two fresh instances step to equal states."""
    inst = make(cf, 4, 32, 256, 8, True)
    assert inst.pressure_fused()
    inst.debug_stall_copies(True)
    inst.step(1)
    with pytest.raises(cf.ChanfastError) as e:
        inst.sync()
    assert e.value.status == cf.CF_ETIMEOUT
    inst.debug_stall_copies(False)
    inst.init_fields(3, 0.1, 0.01)
    inst.sync()
    a = make(cf, 4, 32, 256, 8, True)
    b = make(cf, 4, 32, 256, 8, True)
    a.step(3)
    b.step(3)
    for nm in "uvwcp":
        assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
    for x in (inst, a, b):
        x.close()


@pytest.mark.parametrize("scheme", ["chanfast", "channel"])
def test_set_dt_rebuilds_fused_records(cf, gpu, scheme):
    """cf_set_dt rebuilds the band tables, and with them the fused channel
    solves' precomputed records: an instance whose dt was changed steps as
    one created with that dt."""
    a = make(cf, 4, 64, 256, 10, True, scheme=scheme)
    b = make(cf, 4, 64, 256, 10, True, scheme=scheme, dt=5e-4)
    a.set_dt(5e-4)
    a.step(3)
    b.step(3)
    a.step_graph(1)
    b.step_graph(1)
    for nm in "uvwcp":
        assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
    a.close()
    b.close()


@pytest.mark.parametrize("ny", [64, 128])
def test_other_sizes_keep_separate_launches(cf, gpu, ny):
    a = make(cf, 4, 32, ny, 16, True)
    b = make(cf, 4, 32, ny, 16, False)
    assert a.launches_per_substep() == b.launches_per_substep()
    assert not a.pressure_fused() and not b.pressure_fused()
    a.close()
    b.close()


@pytest.mark.parametrize("ny", [256, 512])
def test_default_rule(cf, gpu, ny):
    """By default the fused launch is taken only where its one block per kx
    gives the GPU enough blocks: nx/2 + 1 at least half the SM count."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    nx_big = next(n for n in (64, 128, 256, 512) if 2 * (n // 2 + 1) >= sms)
    small = make(cf, 4, 32, ny, 8, None)
    big = make(cf, 4, nx_big, ny, 8, None)
    assert not small.pressure_fused()
    assert big.pressure_fused()
    small.close()
    big.close()


def test_batch_mixing_fused_and_separate(cf, gpu):
    """Members that fuse (power-of-two ny) and members that cannot (ny = 48)
    or chose not to share one batch; each ends where it ends alone."""
    # order, nx, ny, nz, fused, seed (members 0 and 3: one state, both paths)
    spec = [(4, 32, 512, 24, True, 20), (2, 64, 48, 20, True, 21), (2, 16, 256, 10, True, 22),
            (4, 32, 512, 24, False, 20), (2, 32, 128, 16, True, 24)]
    mixed = [make(cf, *m[:4], fused=m[4], seed=m[5]) for m in spec]
    alone = [make(cf, *m[:4], fused=m[4], seed=m[5]) for m in spec]
    cf.batch_step(mixed, 5)
    for inst in alone:
        cf.batch_step([inst], 5)
    for a, b in zip(alone, mixed):
        a.sync()
        b.sync()
        for nm in "uvwcp":
            assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
        assert np.array_equal(a.log(), b.log())
    # the fused and the separate member of the same configuration agree
    compare(mixed[0], mixed[3], "batch o4 32x512x24 fused vs separate")
    for inst in mixed + alone:
        inst.close()

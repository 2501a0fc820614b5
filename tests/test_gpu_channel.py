"""GPU parity of the fully implicit scheme (channel2 / channel4 of
channel.c): the CUDA engine with CF_SCHEME_CHANNEL against the compiled
reference replay of the same scheme (oracle/ref_driver.c, itself checked bit
for bit against the unmodified channel drivers in test_ref_driver.py).

Tolerances as for the z-implicit scheme: the engine differs from the
reference in FFT algorithm, summation order and the grouping of the band
coefficients, so u, v, w, c agree to relative L2 <= 1e-12 and p to 1e-10."""
import os

import numpy as np
import pytest

from test_gpu_parity import assert_stats_files_match, interior, logs_close, params, projected_state, rel

import ic

pytestmark = pytest.mark.gpu

CASES = [(2, 64, 24, 12), (4, 64, 32, 16), (4, 128, 20, 24)]


@pytest.mark.parametrize("order,nx,ny,nz", CASES)
def test_channel_substeps_match_reference(cf, ref, gpu, order, nx, ny, nz):
    prm = params(order, nx, ny, nz, nu=1 / 100.0)
    R, F = projected_state(ref, prm, 0, 0.1, 0.01)
    Z, _ = projected_state(ref, prm, 0, 0.1, 0.01)   # the z-implicit scheme, for contrast
    with cf.Instance(cf.Config.from_params(prm, scheme="channel")) as inst:
        for nm in "uvwc":
            inst.set_field(nm, F[nm])
        done = 0
        for n in (1, 3, 30):
            R.substeps(n - done, "channel")
            inst.step(n - done)
            done = n
            for nm in "uvwc":
                assert rel(interior(inst.get_field(nm), prm), interior(R.get(nm), prm)) < 1e-12, (nm, n)
            assert rel(interior(inst.get_field("p"), prm), interior(R.get("p"), prm)) < 1e-10, n
            assert logs_close(inst.log(), R.log())
        assert inst.max_divergence() < 1e-12
    # the two schemes differ by far more than the tolerance (rel 8e-9 .. 2e-7
    # here), so the test tells them apart
    Z.substeps(30, "chanfast")
    assert rel(interior(Z.get("u"), prm), interior(R.get("u"), prm)) > 1e-9
    R.close()
    Z.close()


def test_channel_graph_replay_equals_eager(cf, gpu):
    prm = params(4, 64, 24, 16)
    cfg = cf.Config.from_params(prm, scheme="channel")
    with cf.Instance(cfg) as a, cf.Instance(cfg) as b:
        a.init_fields(4, 0.1, 0.01)
        b.init_fields(4, 0.1, 0.01)
        a.step(1)
        b.step(1)
        a.step_graph(5)
        b.step(17)
        for nm in "uvwcp":
            assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
        assert np.array_equal(a.log(), b.log())
        assert a.launches_per_substep() == 20


@pytest.mark.parametrize("order", [2, 4])
def test_channel_drop_in_driver_matches_reference_driver(cf, ref, gpu, tmp_path, order):
    """channel2/channel4 of libchanfast.so against the reference drivers,
    through restart files and ASCII logs, 2 time steps."""
    prm = params(order, 64, 16, 12, setuframe=0.25, nu=1 / 100.0)
    R, F = projected_state(ref, prm, 3, 0.1, 0.01)
    R.close()
    outs = {}
    for who in ("ref", "gpu"):
        d = tmp_path / who
        os.makedirs(d / "outputdir")
        for nm in "uvwc":
            ic.write_restart(str(d / "outputdir" / f"{nm}_it0.dat"), F[nm], prm)
        if who == "ref":
            ref.run_chanfast(str(d), prm, 0, 2, scheme="channel")
        else:
            cwd = os.getcwd()
            os.chdir(d)
            try:
                rc = cf.channel(order, 1, 1, prm.nx, prm.ny, prm.nz, 0, 2, 2, 3, 3, 3, prm.lx, prm.ly, prm.lz,
                                prm.dt, 1.0, 0, prm.nu, prm.prandtl, prm.dpdx, prm.want_uvolavg,
                                prm.uvolavgmode, prm.want_cvolavg, prm.cvolavgmode, prm.setuframe,
                                prm.setvframe, prm.betg_x, prm.betg_y, prm.betg_z)
            finally:
                os.chdir(cwd)
            assert rc == 0
        outs[who] = d / "outputdir"
    for nm in "uvwc":
        a = ic.read_restart(str(outs["gpu"] / f"{nm}_it2.dat"), prm)
        b = ic.read_restart(str(outs["ref"] / f"{nm}_it2.dat"), prm)
        assert rel(a, b) < 1e-12, nm
    for f in ("cfl.dat", "pstat.dat", "cstat.dat"):
        a = np.loadtxt(str(outs["gpu"] / f))
        b = np.loadtxt(str(outs["ref"] / f))
        assert a.shape == b.shape and np.allclose(a, b, rtol=2e-6, atol=1e-12), f
    assert_stats_files_match(outs["gpu"], outs["ref"], 2)


@pytest.mark.slow
@pytest.mark.parametrize("order", [2, 4])
def test_channel_100_steps(cf, ref, gpu, order):
    """100 RK3 steps of channel2 / channel4 at 64 x 64 x 32 (Re_b 2800,
    dt 1e-3): u, v, w, c within 1e-12 relative L2 (measured 2e-13), max
    divergence <= 1e-12.  This scheme passes every velocity field through 2-D
    transforms each substep, and p, the inverse Laplacian of div(u*) / dt,
    amplifies their rounding by ~1/dt.  The reference itself moves by the
    same amount when only its FFT is replaced by another correct one
    (tests/test_oracle_fft_sensitivity.py): after these 100 steps its own p
    moves by 1.17e-10 (order 2) and 1.07e-10 (order 4), its u, v, w, c by
    3.6e-14 .. 2.0e-13 -- what the engine measures against it.  The bar for
    p is therefore twice that spread, 2.4e-10 (order 2) and 2.2e-10
    (order 4), in place of 1e-10."""
    prm = params(order, 64, 64, 32, lx=4 * np.pi, ly=4 * np.pi / 3, nu=1 / 2800.0, prandtl=1.0)
    R, F = projected_state(ref, prm, 0, 0.1, 0.01)
    with cf.Instance(cf.Config.from_params(prm, scheme="channel")) as inst:
        for nm in "uvwc":
            inst.set_field(nm, F[nm])
        inst.step_graph(100)
        R.substeps(300, "channel")
        worst = {}
        for nm in "uvwcp":
            worst[nm] = rel(interior(inst.get_field(nm), prm), interior(R.get(nm), prm))
        assert all(worst[nm] <= 1e-12 for nm in "uvwc"), worst
        fft_spread = {2: 1.17e-10, 4: 1.07e-10}[order]   # the reference's own, above
        assert worst["p"] <= 2.0 * fft_spread, worst
        assert inst.max_divergence() <= 1e-12
        assert logs_close(inst.log(), R.log())
    R.close()

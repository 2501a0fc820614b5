"""GPU parity: the CUDA engine (through its C ABI) against the compiled
reference (oracle/_ref) and the numpy restatement, on the same seeded inputs.

Tolerances: the engine reproduces the reference arithmetic except for the FFT
algorithm and the order of the xy-average sums, so u, v, w, c agree to a few
ulps (relative L2 <= 1e-13 here); the pressure is an inverse Laplacian of
those differences (<= 1e-10).  The end-to-end bar is relative L2 <= 1e-10 on
u, v, w, c, p after 100 RK3 steps and max discrete divergence <= 1e-12."""
import os

import numpy as np
import pytest

import chanfast_np as cn
import ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def logs_close(a, b):
    """Per-substep log rows (mdpdx, wall gradients, bulk, centreline, and the
    scalar's): the bulk means are summed in a different order than the
    reference's loop, so compare against each column's scale, not relatively
    (dcdt and the scalar centreline are differences of near-cancelling sums)."""
    scale = np.maximum(np.abs(b).max(axis=0), 1e-3)
    return a.shape == b.shape and np.all(np.abs(a - b) <= 1e-9 * scale)


def interior(a, p):
    return a[p.ngx:p.ngx + p.nx, p.ngy:p.ngy + p.ny, p.ngz:p.ngz + p.nz]


def projected_state(ref, prm, seed, amp, c_amp):
    """Raw seeded state made divergence-free by the reference's own projection."""
    g = cn.Grid(prm)
    R = ref.RefInstance(prm)
    u, v, w, c = ic.raw_state(prm, g.dz, seed, amp, c_amp)
    for nm, a in zip("uvwc", (u, v, w, c)):
        R.set(nm, a)
    R.project(1.0)
    u, v, w = R.get("u"), R.get("v"), R.get("w")
    for nm, a in zip("uvwc", (u, v, w, c)):
        R.set(nm, a)
    return R, dict(u=u, v=v, w=w, c=c)


def params(order, nx, ny, nz, **kw):
    base = dict(lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3, nu=1 / 2800.0, prandtl=0.71)
    base.update(kw)
    return cn.Params(order=order, nx=nx, ny=ny, nz=nz, **base)


# (2, 96, 96, 16) .. (4, 48, 320, 8) cover every fixed-size non-power-of-two
# transform (48, 96, 160, 192, 320, 384) in x and in y; the last two have odd
# nx and ny (no Nyquist column; the ky / ny - ky pairs of the band solves
# then have no self-paired column but ky = 0)
CASES = [(2, 16, 12, 10), (2, 32, 32, 32), (4, 18, 24, 12), (4, 64, 48, 40),
         (2, 96, 96, 16), (4, 192, 160, 12), (2, 384, 48, 8), (4, 48, 320, 8),
         (2, 15, 9, 10), (4, 25, 27, 12)]


@pytest.mark.parametrize("order,nx,ny,nz", CASES)
def test_substeps_match_reference(cf, ref, gpu, order, nx, ny, nz):
    prm = params(order, nx, ny, nz)
    R, F = projected_state(ref, prm, 0, 0.1, 0.01)
    with cf.Instance(cf.Config.from_params(prm)) as inst:
        for nm in "uvwc":
            inst.set_field(nm, F[nm])
        done = 0
        for n in (1, 3, 30):
            R.substeps(n - done)
            inst.step(n - done)
            done = n
            for nm in "uvwc":
                assert rel(interior(inst.get_field(nm), prm), interior(R.get(nm), prm)) < 1e-13, (nm, n)
            assert rel(interior(inst.get_field("p"), prm), interior(R.get("p"), prm)) < 1e-10, n
            assert logs_close(inst.log(), R.log())
        assert inst.max_divergence() < 1e-12
    R.close()


@pytest.mark.parametrize("order", [2, 4])
def test_graph_replay_equals_eager(cf, gpu, order):
    prm = params(order, 32, 24, 16)
    cfg = cf.Config.from_params(prm)
    with cf.Instance(cfg) as a, cf.Instance(cfg) as b:
        a.init_fields(4, 0.1, 0.01)
        b.init_fields(4, 0.1, 0.01)
        a.step(1)
        b.step(1)
        a.step_graph(5)   # 2 substeps to the step boundary, 2 graph replays, 1 eager step
        b.step(17)
        for nm in "uvwcp":
            assert np.array_equal(a.get_field(nm), b.get_field(nm)), nm
        assert np.array_equal(a.log(), b.log())
        assert a.substeps_done() == b.substeps_done() == 18


@pytest.mark.parametrize("order", [2, 4])
def test_device_initial_state_matches_reference(cf, ref, gpu, order):
    prm = params(order, 32, 24, 16, lx=2 * np.pi, ly=np.pi)
    R, F = projected_state(ref, prm, 1, 0.1, 0.01)
    with cf.Instance(cf.Config.from_params(prm)) as inst:
        inst.init_fields(1, 0.1, 0.01)
        assert np.array_equal(interior(inst.get_field("c"), prm), interior(F["c"], prm))
        for nm in "uvw":
            assert rel(interior(inst.get_field(nm), prm), interior(F[nm], prm)) < 1e-13, nm
        assert inst.max_divergence() < 1e-12
    R.close()


def test_layouts_round_trip(cf, gpu):
    prm = params(4, 16, 12, 10)
    cfg = cf.Config.from_params(prm)
    rng = np.random.default_rng(0)
    with cf.Instance(cfg) as inst:
        a = rng.standard_normal(cfg.interior_shape())
        inst.set_field("v", a, layout=cf.LAYOUT_INTERIOR)
        assert np.array_equal(inst.get_field("v", layout=cf.LAYOUT_INTERIOR), a)
        pad = inst.get_field("v")
        assert np.array_equal(interior(pad, prm), a)
        # x and y ghosts are periodic images
        assert np.array_equal(pad[0:3], pad[prm.nx:prm.nx + 3])
        assert np.array_equal(pad[:, -3:], pad[:, 3:6])


def test_matches_numpy_restatement(cf, gpu):
    prm = params(4, 24, 16, 12)
    g = cn.Grid(prm)
    u, v, w, c = ic.raw_state(prm, g.dz, 9, 0.1, 0.01)
    cn.project_initial(u, v, w, prm, g, 1.0)
    st = cn.new_state(u, v, w, c, g)
    with cf.Instance(cf.Config.from_params(prm)) as inst:
        for nm, a in zip("uvwc", (u, v, w, c)):
            inst.set_field(nm, a)
        inst.step(6)
        cn.run(st, prm, g, 6)
        for nm in "uvwc":
            assert rel(interior(inst.get_field(nm), prm), interior(getattr(st, nm), prm)) < 1e-13, nm


@pytest.mark.parametrize("order", [2, 4])
def test_drop_in_driver_matches_reference_driver(cf, ref, gpu, tmp_path, order):
    """chanfast2/chanfast4 of libchanfast.so against the reference drivers,
    through restart files and ASCII logs, 2 time steps."""
    prm = params(order, 24, 16, 12, setuframe=0.25)
    R, F = projected_state(ref, prm, 3, 0.1, 0.01)
    R.close()
    outs = {}
    for who in ("ref", "gpu"):
        d = tmp_path / who
        os.makedirs(d / "outputdir")
        for nm in "uvwc":
            ic.write_restart(str(d / "outputdir" / f"{nm}_it0.dat"), F[nm], prm)
        if who == "ref":
            ref.run_chanfast(str(d), prm, 0, 2)
        else:
            cwd = os.getcwd()
            os.chdir(d)
            try:
                rc = cf.chanfast(order, 1, 1, prm.nx, prm.ny, prm.nz, 0, 2, 2, 3, 3, 3, prm.lx, prm.ly, prm.lz,
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
        assert rel(a, b) < 1e-13, nm
    for f in ("cfl.dat", "pstat.dat", "cstat.dat"):
        a = np.loadtxt(str(outs["gpu"] / f))
        b = np.loadtxt(str(outs["ref"] / f))
        assert a.shape == b.shape and np.allclose(a, b, rtol=2e-6, atol=1e-12), f
    assert_stats_files_match(outs["gpu"], outs["ref"], 2)


STATS_FILES = ([f"{f}_avg" for f in "uvwcp"] + [f"{p}_corr" for p in ("uu", "vv", "ww", "cc", "pp", "wu", "uc", "wc")]
               + ["u_mom3", "u_mom4"]
               + [f"{p}_spec{d}" for p in ("uu", "vv", "ww", "cc", "pp", "wu", "uc", "wc") for d in "xy"])


def assert_stats_files_match(gpu_dir, ref_dir, it):
    """The istat statistics files (chanfast.c:658-843): %+e text, 7 digits.
    Entries agree to 2e-6 relative, or to 1e-12 absolute where the quantity
    is zero up to rounding on both sides (the xy mean of w, spectra of
    modes without energy) -- the fields themselves are O(1)."""
    for name in STATS_FILES:
        a = np.loadtxt(str(gpu_dir / f"{name}_it{it}.dat"))
        b = np.loadtxt(str(ref_dir / f"{name}_it{it}.dat"))
        assert a.shape == b.shape, name
        bad = np.abs(a - b) > 2e-6 * np.abs(b) + 1e-12
        assert not bad.any(), (name, int(np.argmax(bad)), a[bad][:3], b[bad][:3])
    for name in ("zp", "zw"):
        a = np.loadtxt(str(gpu_dir / f"{name}.dat"))
        b = np.loadtxt(str(ref_dir / f"{name}.dat"))
        assert np.allclose(a, b, rtol=2e-6, atol=1e-12), name


@pytest.mark.slow
def test_config0_100_steps(cf, ref, gpu):
    """The parity bar at the reference's own CPU-runnable case: 64^3, order 2,
    Re_b 2800, dt 1e-3, 100 RK3 steps from the seed-0 state."""
    prm = cn.Params(order=2, nx=64, ny=64, nz=64, lx=4 * np.pi, ly=4 * np.pi / 3, lz=2.0, dt=1e-3,
                    nu=1 / 2800.0, prandtl=1.0)
    R, F = projected_state(ref, prm, 0, 0.1, 0.0)
    with cf.Instance(cf.Config.from_params(prm)) as inst:
        for nm in "uvwc":
            inst.set_field(nm, F[nm])
        inst.step_graph(100)
        R.substeps(300)
        for nm in "uvwcp":
            r = rel(interior(inst.get_field(nm), prm), interior(R.get(nm), prm))
            assert r <= 1e-10, (nm, r)
        assert inst.max_divergence() <= 1e-12
        assert logs_close(inst.log(), R.log())
    R.close()
